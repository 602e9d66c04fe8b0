// graph.cu -- device graphs: construction from host / device CSR, coarsened
// levels, and the seeded R-MAT / SBM generators.
#include <cmath>
#include <vector>

#include "handles.cuh"

namespace mg {

namespace {

// pair k of a seeded R-MAT graph of 2^scale vertices: one quadrant choice per
// bit level, two levels per 64-bit random word
__device__ __forceinline__ void rmat_pair(int scale, uint64_t t1, uint64_t t2, uint64_t t3, uint64_t key, uint64_t k,
                                          uint32_t &u, uint32_t &v) {
    const int words = (scale + 1) / 2;
    uint32_t uu = 0, vv = 0;
    for (int wi = 0; wi < words; wi++) {
        uint64_t r = rng_at(key, k * (uint64_t)words + (uint64_t)wi);
#pragma unroll
        for (int h = 0; h < 2; h++) {
            int l = 2 * wi + h;
            if (l >= scale) break;
            uint64_t x = h ? (r >> 32) : (r & 0xFFFFFFFFull);
            uint32_t bu, bv;
            if (x < t1) { bu = 0; bv = 0; }
            else if (x < t2) { bu = 0; bv = 1; }
            else if (x < t3) { bu = 1; bv = 0; }
            else { bu = 1; bv = 1; }
            uu |= bu << (scale - 1 - l);
            vv |= bv << (scale - 1 - l);
        }
    }
    u = uu;
    v = vv;
}

__global__ void rmat_pairs_kernel(int scale, uint64_t m, uint64_t t1, uint64_t t2, uint64_t t3, uint64_t key,
                                  uint32_t *u, uint32_t *v) {
    for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < m; k += (uint64_t)gridDim.x * blockDim.x)
        rmat_pair(scale, t1, t2, t3, key, k, u[k], v[k]);
}

// pair k of a seeded SBM: the first min_ pairs join two vertices of one block,
// the rest two vertices of different blocks (block b holds [b*n/blocks,
// (b+1)*n/blocks))
__device__ __forceinline__ void sbm_pair(uint32_t n, uint32_t blocks, uint64_t min_, uint64_t kin, uint64_t kout,
                                         uint64_t k, uint32_t &u, uint32_t &v) {
    if (k < min_) {
        uint64_t r0 = rng_at(kin, 2 * k), r1 = rng_at(kin, 2 * k + 1);
        uint32_t bb = uni32((uint32_t)r0, blocks);
        uint32_t lo = (uint32_t)((uint64_t)bb * n / blocks), hi = (uint32_t)((uint64_t)(bb + 1) * n / blocks);
        u = lo + uni32((uint32_t)(r0 >> 32), hi - lo);
        v = lo + uni32((uint32_t)r1, hi - lo);
    } else {
        uint64_t j = k - min_;
        uint64_t r0 = rng_at(kout, 2 * j), r1 = rng_at(kout, 2 * j + 1);
        uint32_t b1 = uni32((uint32_t)r0, blocks);
        uint32_t b2 = uni32((uint32_t)(r0 >> 32), blocks - 1);
        if (b2 >= b1) b2++;
        uint32_t lo1 = (uint32_t)((uint64_t)b1 * n / blocks), hi1 = (uint32_t)((uint64_t)(b1 + 1) * n / blocks);
        uint32_t lo2 = (uint32_t)((uint64_t)b2 * n / blocks), hi2 = (uint32_t)((uint64_t)(b2 + 1) * n / blocks);
        u = lo1 + uni32((uint32_t)r1, hi1 - lo1);
        v = lo2 + uni32((uint32_t)(r1 >> 32), hi2 - lo2);
    }
}

__global__ void sbm_pairs_kernel(uint32_t n, uint32_t blocks, uint64_t min_, uint64_t m, uint64_t kin, uint64_t kout,
                                 uint32_t *u, uint32_t *v) {
    for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < m; k += (uint64_t)gridDim.x * blockDim.x)
        sbm_pair(n, blocks, min_, kin, kout, k, u[k], v[k]);
}

// Chung-Lu pair k: both endpoints drawn from the expected-degree distribution
// (first index whose 63-bit cumulative weight exceeds a 63-bit random draw);
// the pair's weight, when asked for, is lognormal(0, 1) rounded to float, a
// function of the unordered pair (Box-Muller on two hashes of it)
__global__ void chunglu_pairs_kernel(const uint64_t *cdf, uint32_t n, uint64_t m, uint64_t key, uint64_t kw,
                                     uint32_t *u, uint32_t *v, double *w) {
    for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < m; k += (uint64_t)gridDim.x * blockDim.x) {
        uint32_t ends[2];
        for (int side = 0; side < 2; side++) {
            const uint64_t x = rng_at(key, 2 * k + side) >> 1;
            uint32_t a = 0, b = n - 1;
            while (a < b) {
                const uint32_t mid = a + (b - a) / 2;
                if (cdf[mid] > x) b = mid;
                else a = mid + 1;
            }
            ends[side] = a;
        }
        u[k] = ends[0];
        v[k] = ends[1];
        if (w) {
            const uint32_t a = min(ends[0], ends[1]), b = max(ends[0], ends[1]);
            const uint64_t h1 = mix64(kw ^ (((uint64_t)a << 32) | b));
            const uint64_t h2 = mix64(h1);
            const double u1 = ((double)(h1 >> 11) + 1.0) * (1.0 / 9007199254740992.0);
            const double u2 = (double)(h2 >> 11) * (1.0 / 9007199254740992.0);
            const double z = sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2);
            w[k] = (double)(float)exp(z);
        }
    }
}

__global__ void to_f32_kernel(const double *x, uint64_t m, float *y) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += (uint64_t)gridDim.x * blockDim.x)
        y[i] = (float)x[i];
}

// per-graph parameters of a generated batch
struct GenDev {
    uint32_t kind, n, blocks, vbase;  // SBM: vertices, blocks; first vertex in the union
    int scale, pad;                   // R-MAT
    uint64_t min_, kin, kout;         // SBM: intra pairs, stream keys / R-MAT: key in kin
    uint64_t t1, t2, t3;              // R-MAT quadrant thresholds
    uint64_t pbase;                   // first pair of the graph
};

// all pairs of all graphs of a batch; graph of pair k by binary search over
// the pair bases (G + 1 entries)
__global__ void batch_pairs_kernel(const GenDev *gp, const uint64_t *pbase, uint32_t G, uint64_t M, uint32_t *u,
                                   uint32_t *v) {
    for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < M; k += (uint64_t)gridDim.x * blockDim.x) {
        uint32_t lo = 0, hi = G;  // last graph with pbase <= k
        while (hi - lo > 1) {
            uint32_t mid = (lo + hi) >> 1;
            if (pbase[mid] <= k) lo = mid;
            else hi = mid;
        }
        const GenDev &p = gp[lo];
        uint32_t a, b;
        if (p.kind == MG_GEN_RMAT) rmat_pair(p.scale, p.t1, p.t2, p.t3, p.kin, k - p.pbase, a, b);
        else sbm_pair(p.n, p.blocks, p.min_, p.kin, p.kout, k - p.pbase, a, b);
        u[k] = p.vbase + a;
        v[k] = p.vbase + b;
    }
}

// packed rows of a batch from the host: 64-bit row offsets -> 32-bit, local
// column ids -> union ids; flags non-monotone offsets (bit 0) and column ids
// outside the row's graph (bit 1).  One warp per row.
__global__ void batch_rows_kernel(const uint64_t *off64, uint32_t n, const uint32_t *voff, uint32_t G, uint32_t *cols,
                                  uint32_t *off32, int *bad) {
    const uint32_t lane = threadIdx.x & 31;
    int b = 0;
    for (uint64_t v = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; v <= n;
         v += ((uint64_t)gridDim.x * blockDim.x) >> 5) {
        const uint64_t o = off64[v];
        if (lane == 0) {
            off32[v] = (uint32_t)o;
            if (v > 0 && o < off64[v - 1]) b |= 1;
        }
        if (v == n) continue;
        uint32_t lo = 0, hi = G;  // graph of row v: last g with voff[g] <= v
        while (hi - lo > 1) {
            uint32_t mid = (lo + hi) >> 1;
            if (voff[mid] <= v) lo = mid;
            else hi = mid;
        }
        const uint32_t base = voff[lo], ng = voff[lo + 1] - base;
        const uint64_t e1 = off64[v + 1];
        for (uint64_t e = o + lane; e < e1; e += 32) {
            const uint32_t c = cols[e];
            if (c >= ng) b |= 2;
            else cols[e] = base + c;
        }
    }
    if (b) atomicOr(bad, b);
}

// 64-bit offsets -> 32-bit; flags non-monotone offsets (bit 0) and column ids
// out of range (bit 1)
__global__ void check_csr_kernel(const uint64_t *off64, uint32_t n, const uint32_t *cols, uint64_t nnz,
                                 uint32_t *off32, int *bad) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    int b = 0;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i <= n; i += stride) {
        uint64_t o = off64[i];
        off32[i] = (uint32_t)o;
        if (i > 0 && o < off64[i - 1]) b |= 1;
    }
    for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < nnz; e += stride)
        if (cols[e] >= n) b |= 2;
    if (b) atomicOr(bad, b);
}

// 64-bit finaliser of SplitMix64 (Steele, Lea and Flood, OOPSLA 2014)
__device__ __forceinline__ uint64_t mix64(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}

// hash of the entry (a, b) with integer weight x under one of two seeds
__device__ __forceinline__ uint64_t entry_hash(uint32_t a, uint32_t b, uint64_t x, uint64_t seed) {
    return mix64(mix64((((uint64_t)a << 32) | b) ^ seed) + x * 0x9e3779b97f4a7c15ull);
}

// A warp per row.  *unsorted |= 1 when a row is not strictly increasing.
// FP (integral weights): fp[0..3] += the sums over the entries (u, v, x) of
// h1(u, v, x), h1(v, u, x), h2(u, v, x), h2(v, u, x) (mod 2^64).  A graph
// whose entries are, as a multiset, their own transposes gives fp[0] ==
// fp[1] and fp[2] == fp[3]; any other graph gives two equal pairs only by a
// collision of two independent 64-bit sums.
template <int WK, bool FP>
__global__ void row_checks_kernel(const uint32_t *off, const uint32_t *col, const void *w, uint32_t n,
                                  int *unsorted, unsigned long long *fp) {
    constexpr uint64_t kSeed1 = 0x243f6a8885a308d3ull, kSeed2 = 0x13198a2e03707344ull;
    const uint32_t lane = threadIdx.x & 31u;
    int bad = 0;
    uint64_t f0 = 0, f1 = 0, f2 = 0, f3 = 0;
    for (uint32_t r = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < n; r += (gridDim.x * blockDim.x) >> 5) {
        const uint32_t lo = off[r], hi = off[r + 1];
        for (uint32_t e = lo + lane; e < hi; e += 32) {
            const uint32_t v = col[e];
            if (e + 1 < hi) bad |= v >= col[e + 1];
            if constexpr (FP) {
                uint64_t x = 1;
                if constexpr (WK == WK_F32) x = (uint64_t)((const float *)w)[e];
                else if constexpr (WK == WK_F64) x = (uint64_t)((const double *)w)[e];
                f0 += entry_hash(r, v, x, kSeed1);
                f1 += entry_hash(v, r, x, kSeed1);
                f2 += entry_hash(r, v, x, kSeed2);
                f3 += entry_hash(v, r, x, kSeed2);
            }
        }
    }
    if (__any_sync(0xffffffffu, bad) && lane == 0) atomicOr(unsorted, 1);
    if constexpr (FP) {
        f0 = warp_sum((unsigned long long)f0);
        f1 = warp_sum((unsigned long long)f1);
        f2 = warp_sum((unsigned long long)f2);
        f3 = warp_sum((unsigned long long)f3);
        if (lane == 0) {
            atomicAdd(fp + 0, (unsigned long long)f0);
            atomicAdd(fp + 1, (unsigned long long)f1);
            atomicAdd(fp + 2, (unsigned long long)f2);
            atomicAdd(fp + 3, (unsigned long long)f3);
        }
    }
}

// per-block partial sums of weights and integrality flags
template <class T>
__global__ void weight_stats_kernel(const T *w, uint64_t m, double *partial, int *nonintegral, int *nonunit) {
    double s = 0;
    int ni = 0, nu = 0;
    for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < m; e += (uint64_t)gridDim.x * blockDim.x) {
        double x = (double)w[e];
        s += x;
        ni |= (x < 0 || x != floor(x));
        nu |= (x != 1.0);
    }
    s = warp_sum(s);
    __shared__ double red[32];
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    if (__any_sync(0xffffffffu, ni) && (threadIdx.x & 31) == 0) atomicOr(nonintegral, 1);
    if (__any_sync(0xffffffffu, nu) && (threadIdx.x & 31) == 0) atomicOr(nonunit, 1);
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0;
        for (int i = 0; i < (int)(blockDim.x >> 5); i++) t += red[i];
        partial[blockIdx.x] = t;
    }
}

}  // namespace

// mass and integrality of a device weight array (deterministic block order)
template <class T>
static void device_weight_stats(const T *w, uint64_t m, double &mass, int &integral, int &unit, cudaStream_t s) {
    const unsigned blocks = 148 * 4;
    DBuf<double> part;
    DBuf<int> flags;
    double *p = part.ensure(blocks);
    int *f = flags.ensure(2);
    MG_CUDA(cudaMemsetAsync(f, 0, 2 * sizeof(int), s));
    weight_stats_kernel<T><<<blocks, 256, 0, s>>>(w, m, p, f, f + 1);
    MG_LAUNCH_CHECK();
    std::vector<double> hp(blocks);
    int hf[2];
    MG_CUDA(cudaMemcpyAsync(hp.data(), p, blocks * sizeof(double), cudaMemcpyDeviceToHost, s));
    MG_CUDA(cudaMemcpyAsync(hf, f, 2 * sizeof(int), cudaMemcpyDeviceToHost, s));
    MG_CUDA(cudaStreamSynchronize(s));
    double t = 0;
    for (double x : hp) t += x;
    mass = t;
    integral = !hf[0] && t < 4294967296.0;
    unit = !hf[1];
}

// An uploaded graph's row properties, in one pass over its entries: whether
// every row is strictly increasing, and (integral weights) whether it is
// symmetric as a multiset of entries (fingerprint above).
static void detect_row_properties(mg_graph *g, cudaStream_t s) {
    g->sorted_rows = 1;
    g->symmetric = g->integral;
    if (g->n == 0) return;
    DBuf<unsigned long long> flags;
    unsigned long long *d = flags.ensure(5);
    MG_CUDA(cudaMemsetAsync(d, 0, 5 * sizeof(unsigned long long), s));
    int *uns = (int *)(d + 4);
    const void *w = g->wk == WK_F32 ? (const void *)g->w32.get() : (const void *)g->w64.get();
    auto run = [&](auto kern) {
        kern<<<148 * 16, 256, 0, s>>>(g->off.get(), g->col.get(), w, g->n, uns, d);
        MG_LAUNCH_CHECK();
    };
    if (!g->integral) run(row_checks_kernel<WK_UNIT, false>);
    else if (g->wk == WK_F32) run(row_checks_kernel<WK_F32, true>);
    else if (g->wk == WK_F64) run(row_checks_kernel<WK_F64, true>);
    else run(row_checks_kernel<WK_UNIT, true>);
    unsigned long long h[5];
    MG_CUDA(cudaMemcpyAsync(h, d, sizeof h, cudaMemcpyDeviceToHost, s));
    MG_CUDA(cudaStreamSynchronize(s));
    g->sorted_rows = *(const int *)(h + 4) == 0;
    g->symmetric = g->integral && h[0] == h[1] && h[2] == h[3];
}

void graph_from_host_csr(mg_graph *g, uint32_t n, const uint64_t *offsets, const uint32_t *cols, const void *w,
                         int weight_type) {
    MG_CHECK(offsets != nullptr, MG_ERR_INVALID, "offsets is NULL");
    MG_CHECK(n < 0xFFFFFFFFu, MG_ERR_UNSUPPORTED, "too many vertices");
    MG_CHECK(offsets[0] == 0, MG_ERR_INVALID, "offsets[0] must be 0");
    const uint64_t nnz = offsets[n];
    MG_CHECK(nnz < 0xFFFFFFFFull, MG_ERR_UNSUPPORTED, "nnz must be below 2^32-1");
    MG_CHECK(nnz == 0 || cols != nullptr, MG_ERR_INVALID, "cols is NULL");
    MG_CHECK(weight_type >= MG_WEIGHT_UNIT && weight_type <= MG_WEIGHT_F64, MG_ERR_INVALID, "bad weight type");
    MG_CHECK(weight_type == MG_WEIGHT_UNIT || nnz == 0 || w != nullptr, MG_ERR_INVALID, "weights is NULL");
    // mass in CSR order (src/graph/host_graph.cpp:112-115), integrality, unit detection
    double mass = (double)nnz;
    bool nonint = false, unit = true;
    if (weight_type != MG_WEIGHT_UNIT) {
        mass = 0;
        for (uint64_t e = 0; e < nnz; e++) {
            double x = weight_type == MG_WEIGHT_F32 ? (double)((const float *)w)[e] : ((const double *)w)[e];
            mass += x;
            nonint |= (x < 0 || x != std::floor(x));
            unit &= (x == 1.0);
        }
    }
    cudaStream_t s = g->ctx->stream;
    g->n = n;
    g->nnz = nnz;
    // offsets and columns are checked on the device after the copy
    {
        DBuf<uint64_t> off64;
        DBuf<int> bad;
        uint64_t *d64 = off64.ensure((size_t)n + 1);
        int *dbad = bad.ensure(1);
        MG_CUDA(cudaMemsetAsync(dbad, 0, sizeof(int), s));
        MG_CUDA(cudaMemcpyAsync(d64, offsets, sizeof(uint64_t) * ((size_t)n + 1), cudaMemcpyHostToDevice, s));
        uint32_t *doff = g->off.ensure((size_t)n + 1);
        uint32_t *dcol = g->col.ensure(nnz + 1);
        MG_CUDA(cudaMemcpyAsync(dcol, cols, sizeof(uint32_t) * nnz, cudaMemcpyHostToDevice, s));
        check_csr_kernel<<<148 * 8, 256, 0, s>>>(d64, n, dcol, nnz, doff, dbad);
        MG_LAUNCH_CHECK();
        int hbad = 0;
        MG_CUDA(cudaMemcpyAsync(&hbad, dbad, sizeof(int), cudaMemcpyDeviceToHost, s));
        MG_CUDA(cudaStreamSynchronize(s));
        MG_CHECK(!(hbad & 1), MG_ERR_INVALID, "offsets must be non-decreasing");
        MG_CHECK(!(hbad & 2), MG_ERR_INVALID, "column index out of range");
    }
    if (unit) {
        g->wk = WK_UNIT;
    } else if (weight_type == MG_WEIGHT_F32) {
        g->wk = WK_F32;
        MG_CUDA(cudaMemcpyAsync(g->w32.ensure(nnz + 1), w, sizeof(float) * nnz, cudaMemcpyHostToDevice, s));
    } else {
        g->wk = WK_F64;
        MG_CUDA(cudaMemcpyAsync(g->w64.ensure(nnz + 1), w, sizeof(double) * nnz, cudaMemcpyHostToDevice, s));
    }
    g->mass = mass;
    g->integral = !nonint && mass < 4294967296.0;
    MG_CUDA(cudaStreamSynchronize(s));
    detect_row_properties(g, s);
}

void graph_from_device_csr(mg_graph *g, uint32_t n, uint64_t nnz, const uint32_t *d_off, const uint32_t *d_cols,
                           const void *d_w, int weight_type) {
    MG_CHECK(nnz < 0xFFFFFFFFull, MG_ERR_UNSUPPORTED, "nnz must be below 2^32-1");
    cudaStream_t s = g->ctx->stream;
    g->n = n;
    g->nnz = nnz;
    MG_CUDA(cudaMemcpyAsync(g->off.ensure((size_t)n + 1), d_off, sizeof(uint32_t) * ((size_t)n + 1),
                            cudaMemcpyDeviceToDevice, s));
    MG_CUDA(cudaMemcpyAsync(g->col.ensure(nnz + 1), d_cols, sizeof(uint32_t) * nnz, cudaMemcpyDeviceToDevice, s));
    g->wk = WK_UNIT;
    g->mass = (double)nnz;
    g->integral = nnz < 4294967296ull;
    if (weight_type != MG_WEIGHT_UNIT && nnz > 0) {
        int integral = 0, unit = 0;
        if (weight_type == MG_WEIGHT_F32) {
            device_weight_stats<float>((const float *)d_w, nnz, g->mass, integral, unit, s);
            if (!unit) {
                g->wk = WK_F32;
                MG_CUDA(cudaMemcpyAsync(g->w32.ensure(nnz + 1), d_w, sizeof(float) * nnz, cudaMemcpyDeviceToDevice, s));
            }
        } else {
            device_weight_stats<double>((const double *)d_w, nnz, g->mass, integral, unit, s);
            if (!unit) {
                g->wk = WK_F64;
                MG_CUDA(cudaMemcpyAsync(g->w64.ensure(nnz + 1), d_w, sizeof(double) * nnz, cudaMemcpyDeviceToDevice, s));
            }
        }
        g->integral = integral;
    }
    MG_CUDA(cudaStreamSynchronize(s));
    detect_row_properties(g, s);
}

void graph_from_level(mg_graph *g, LevelGraph &lv, int integral, double mass) {
    MG_CHECK(lv.wk == WK_F64, MG_ERR_INVALID, "graph_from_level: f64 level expected");
    cudaStream_t s = g->ctx->stream;
    g->n = lv.n;
    g->nnz = lv.nnz;
    MG_CUDA(cudaMemcpyAsync(g->off.ensure((size_t)lv.n + 1), lv.off.get(), sizeof(uint32_t) * ((size_t)lv.n + 1),
                            cudaMemcpyDeviceToDevice, s));
    MG_CUDA(cudaMemcpyAsync(g->col.ensure(lv.nnz + 1), lv.col.get(), sizeof(uint32_t) * lv.nnz,
                            cudaMemcpyDeviceToDevice, s));
    MG_CUDA(cudaMemcpyAsync(g->w64.ensure(lv.nnz + 1), lv.w.get(), sizeof(double) * lv.nnz,
                            cudaMemcpyDeviceToDevice, s));
    g->wk = WK_F64;
    g->integral = integral;
    g->mass = mass;
    g->sorted_rows = 1;  // levels have sorted, deduplicated rows
    g->symmetric = lv.symmetric && integral;
    MG_CUDA(cudaStreamSynchronize(s));
}

static void finish_generated(mg_graph *g, uint32_t n, uint64_t m, DBuf<uint32_t> &u, DBuf<uint32_t> &v) {
    mg_ctx *ctx = g->ctx;
    cudaStream_t s = ctx->stream;
    LevelGraph lv;
    csr_from_device_pairs(n, m, u.get(), v.get(), lv, ctx->cws, s);
    u.release();
    v.release();
    g->n = n;
    g->nnz = lv.nnz;
    // adopt the level's buffers
    std::swap(g->off.p, lv.off.p);
    std::swap(g->off.cap, lv.off.cap);
    std::swap(g->col.p, lv.col.p);
    std::swap(g->col.cap, lv.col.cap);
    g->wk = WK_UNIT;
    g->mass = (double)lv.nnz;
    g->integral = lv.nnz < 4294967296ull;
    g->sorted_rows = 1;  // sorted, deduplicated pairs
    g->symmetric = g->integral;  // both directions of every pair
    MG_CUDA(cudaStreamSynchronize(s));
}

void graph_generate_rmat(mg_graph *g, int scale, int edge_factor, double a, double b, double c, uint64_t seed) {
    MG_CHECK(scale >= 1 && scale <= 31 && edge_factor >= 1, MG_ERR_INVALID, "rmat: bad scale or edge factor");
    MG_CHECK(a >= 0 && b >= 0 && c >= 0 && a + b + c <= 1.0, MG_ERR_INVALID, "rmat: bad probabilities");
    const uint32_t n = 1u << scale;
    const uint64_t m = (uint64_t)edge_factor << scale;
    MG_CHECK(2 * m < 0xFFFFFFFFull, MG_ERR_UNSUPPORTED, "rmat: more than 2^32-1 directed entries");
    const uint64_t t1 = (uint64_t)(a * 4294967296.0);
    const uint64_t t2 = (uint64_t)((a + b) * 4294967296.0);
    const uint64_t t3 = (uint64_t)((a + b + c) * 4294967296.0);
    const uint64_t key = rng_key(seed, 0x524d4154ull);
    DBuf<uint32_t> u, v;
    u.ensure(m);
    v.ensure(m);
    cudaStream_t s = g->ctx->stream;
    rmat_pairs_kernel<<<148 * 16, 256, 0, s>>>(scale, m, t1, t2, t3, key, u.get(), v.get());
    MG_LAUNCH_CHECK();
    finish_generated(g, n, m, u, v);
}

void graph_generate_sbm(mg_graph *g, uint32_t n, uint32_t blocks, double mean_degree, double intra_frac,
                        uint64_t seed) {
    MG_CHECK(blocks >= 1 && n >= blocks && n < 0xFFFFFFFFu, MG_ERR_INVALID, "sbm: need 1 <= blocks <= n");
    const double din = mean_degree * intra_frac;
    const double dout = mean_degree - din;
    const uint64_t min_ = (uint64_t)std::llround((double)n * din / 2.0);
    const uint64_t mout = blocks > 1 ? (uint64_t)std::llround((double)n * dout / 2.0) : 0;
    const uint64_t m = min_ + mout;
    MG_CHECK(2 * m < 0xFFFFFFFFull, MG_ERR_UNSUPPORTED, "sbm: more than 2^32-1 directed entries");
    DBuf<uint32_t> u, v;
    u.ensure(m + 1);
    v.ensure(m + 1);
    cudaStream_t s = g->ctx->stream;
    if (m > 0) {
        sbm_pairs_kernel<<<148 * 16, 256, 0, s>>>(n, blocks, min_, m, rng_key(seed, 0x53424d31ull),
                                                  rng_key(seed, 0x53424d32ull), u.get(), v.get());
        MG_LAUNCH_CHECK();
    }
    finish_generated(g, n, m, u, v);
}

// Seeded Chung-Lu graph: expected degrees w_i = c * (i + i0)^(-1/(exponent-1)),
// i0 chosen so that w_0 / mean(w) = max_degree / mean_degree (integral
// approximation, bisection), scaled to mean_degree and capped at max_degree;
// n * mean_degree / 2 pairs with both ends drawn with probability
// proportional to w; self-loops dropped, duplicates merged.  The expected
// degrees and their cumulative table are computed on the host in the order
// written (the same table as the test oracle's generator); the pairs on the
// device from the same counter-based stream.
void graph_generate_chunglu(mg_graph *g, uint32_t n, double exponent, double mean_degree, double max_degree,
                            int lognormal, uint64_t seed) {
    MG_CHECK(n >= 2 && n < 0xFFFFFFFFu && exponent > 1.0 && mean_degree > 0 && max_degree > 0, MG_ERR_INVALID,
             "chung-lu: need n >= 2, exponent > 1, positive degrees");
    const double alpha = 1.0 / (exponent - 1.0);
    double lo = 1e-6, hi = (double)n;
    for (int it = 0; it < 200; it++) {
        const double i0 = 0.5 * (lo + hi);
        const double integ = (alpha == 1.0) ? std::log((n + i0) / i0)
                                            : (std::pow(n + i0, 1.0 - alpha) - std::pow(i0, 1.0 - alpha)) / (1.0 - alpha);
        const double ratio = std::pow(i0, -alpha) / (integ / n);
        if (ratio > max_degree / mean_degree) lo = i0;
        else hi = i0;
    }
    const double i0 = 0.5 * (lo + hi);
    std::vector<double> wd(n);
    double sum = 0;
    for (uint32_t i = 0; i < n; i++) {
        wd[i] = std::pow((double)i + i0, -alpha);
        sum += wd[i];
    }
    const double cst = mean_degree * n / sum;
    double tot = 0;
    for (uint32_t i = 0; i < n; i++) {
        wd[i] *= cst;
        if (wd[i] > max_degree) wd[i] = max_degree;
        tot += wd[i];
    }
    std::vector<uint64_t> cdf(n);
    double acc = 0;
    for (uint32_t i = 0; i < n; i++) {
        acc += wd[i];
        double f = acc / tot;
        if (f > 1.0) f = 1.0;
        cdf[i] = (uint64_t)(f * 9223372036854775808.0);
    }
    cdf[n - 1] = 0x8000000000000000ull;
    const uint64_t m = (uint64_t)std::llround((double)n * mean_degree / 2.0);
    MG_CHECK(2 * m < 0xFFFFFFFFull, MG_ERR_UNSUPPORTED, "chung-lu: more than 2^32-1 directed entries");
    mg_ctx *ctx = g->ctx;
    cudaStream_t s = ctx->stream;
    DBuf<uint64_t> dcdf;
    DBuf<uint32_t> u, v;
    DBuf<double> w;
    MG_CUDA(cudaMemcpyAsync(dcdf.ensure(n), cdf.data(), sizeof(uint64_t) * n, cudaMemcpyHostToDevice, s));
    u.ensure(m + 1);
    v.ensure(m + 1);
    double *dw = lognormal ? w.ensure(m + 1) : nullptr;
    if (m > 0) {
        chunglu_pairs_kernel<<<148 * 16, 256, 0, s>>>(dcdf.get(), n, m, rng_key(seed, 0x434c5547ull),
                                                      rng_key(seed, 0x4c4f474eull), u.get(), v.get(), dw);
        MG_LAUNCH_CHECK();
    }
    LevelGraph lv;
    csr_from_device_pairs(n, m, u.get(), v.get(), lv, ctx->cws, s, dw);
    g->n = n;
    g->nnz = lv.nnz;
    g->sorted_rows = 1;  // sorted, deduplicated pairs
    std::swap(g->off.p, lv.off.p);
    std::swap(g->off.cap, lv.off.cap);
    std::swap(g->col.p, lv.col.p);
    std::swap(g->col.cap, lv.col.cap);
    if (!lognormal) {
        g->wk = WK_UNIT;
        g->mass = (double)lv.nnz;
        g->integral = lv.nnz < 4294967296ull;
    } else {
        // every weight is a float value: keep them as f32
        if (lv.nnz) {
            float *w32 = g->w32.ensure(lv.nnz + 1);  // (allocations stay out of launch argument lists)
            to_f32_kernel<<<148 * 16, 256, 0, s>>>(lv.w.get(), lv.nnz, w32);
            MG_LAUNCH_CHECK();
        }
        g->wk = WK_F32;
        int integral = 0, unit = 0;
        device_weight_stats<float>(g->w32.get(), lv.nnz, g->mass, integral, unit, s);
        g->integral = integral;
    }
    g->symmetric = g->integral;  // both directions of every pair, with its weight
    MG_CUDA(cudaStreamSynchronize(s));
}

// ---- batches -----------------------------------------------------------------

namespace {
__global__ void gather_u32_kernel(const uint32_t *src, const uint32_t *idx, uint32_t m, uint32_t *dst) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < m) dst[i] = src[idx[i]];
}
}  // namespace

// entry offsets of the graphs of a packed union (offsets at the first vertex of
// each graph)
static void batch_entry_offsets(mg_batch *b) {
    cudaStream_t s = b->ctx->stream;
    const uint32_t G = b->graphs;
    uint32_t *idx = b->work.small.ensure(2 * (G + 1)), *out = idx + G + 1;
    MG_CUDA(cudaMemcpyAsync(idx, b->voff.data(), sizeof(uint32_t) * (G + 1), cudaMemcpyHostToDevice, s));
    gather_u32_kernel<<<(unsigned)ceil_div(G + 1, 256), 256, 0, s>>>(b->u.off.get(), idx, G + 1, out);
    MG_LAUNCH_CHECK();
    std::vector<uint32_t> h(G + 1);
    MG_CUDA(cudaMemcpyAsync(h.data(), out, sizeof(uint32_t) * (G + 1), cudaMemcpyDeviceToHost, s));
    MG_CUDA(cudaStreamSynchronize(s));
    b->eoff.assign(h.begin(), h.end());
}

void batch_generate(mg_batch *b, const mg_gen_params *params) {
    const uint32_t G = b->graphs;
    MG_CHECK(G >= 1 && params != nullptr, MG_ERR_INVALID, "batch: need at least one graph and its parameters");
    std::vector<GenDev> gp(G);
    std::vector<uint64_t> pbase(G + 1, 0);
    b->voff.assign(G + 1, 0);
    uint64_t nv = 0, M = 0;
    for (uint32_t g = 0; g < G; g++) {
        const mg_gen_params &p = params[g];
        GenDev &d = gp[g];
        d = GenDev{};
        d.kind = (uint32_t)p.kind;
        uint64_t m = 0;
        if (p.kind == MG_GEN_SBM) {
            MG_CHECK(p.blocks >= 1 && p.n >= p.blocks, MG_ERR_INVALID, "sbm: need 1 <= blocks <= n");
            // pair counts exactly as graph_generate_sbm
            const double din = p.mean_degree * p.intra_frac;
            const double dout = p.mean_degree - din;
            const uint64_t min_ = (uint64_t)std::llround((double)p.n * din / 2.0);
            const uint64_t mout = p.blocks > 1 ? (uint64_t)std::llround((double)p.n * dout / 2.0) : 0;
            d.n = p.n;
            d.blocks = p.blocks;
            d.min_ = min_;
            d.kin = rng_key(p.seed, 0x53424d31ull);
            d.kout = rng_key(p.seed, 0x53424d32ull);
            m = min_ + mout;
        } else if (p.kind == MG_GEN_RMAT) {
            // as graph_generate_rmat
            MG_CHECK(p.scale >= 1 && p.scale <= 31 && p.edge_factor >= 1, MG_ERR_INVALID, "rmat: bad scale or edge factor");
            MG_CHECK(p.a >= 0 && p.b >= 0 && p.c >= 0 && p.a + p.b + p.c <= 1.0, MG_ERR_INVALID,
                     "rmat: bad probabilities");
            d.n = 1u << p.scale;
            d.scale = p.scale;
            d.t1 = (uint64_t)(p.a * 4294967296.0);
            d.t2 = (uint64_t)((p.a + p.b) * 4294967296.0);
            d.t3 = (uint64_t)((p.a + p.b + p.c) * 4294967296.0);
            d.kin = rng_key(p.seed, 0x524d4154ull);
            m = (uint64_t)p.edge_factor << p.scale;
        } else {
            throw Error(MG_ERR_INVALID, "batch: unknown generator kind");
        }
        d.vbase = (uint32_t)nv;
        d.pbase = M;
        pbase[g] = M;
        b->voff[g] = (uint32_t)nv;
        nv += d.n;
        M += m;
        MG_CHECK(nv < 0xFFFFFFFFull, MG_ERR_UNSUPPORTED, "batch: more than 2^32-1 vertices in total");
        MG_CHECK(2 * M < 0xFFFFFFFFull, MG_ERR_UNSUPPORTED, "batch: more than 2^32-1 directed entries in total");
    }
    pbase[G] = M;
    b->voff[G] = (uint32_t)nv;
    cudaStream_t s = b->ctx->stream;
    BatchWork &W = b->work;
    uint32_t *u = W.pu.ensure(M + 1), *v = W.pv.ensure(M + 1);
    if (M > 0) {
        GenDev *dgp = (GenDev *)W.gen.ensure(sizeof(GenDev) * G);
        uint64_t *dpb = W.pbase.ensure(G + 1);
        MG_CUDA(cudaMemcpyAsync(dgp, gp.data(), sizeof(GenDev) * G, cudaMemcpyHostToDevice, s));
        MG_CUDA(cudaMemcpyAsync(dpb, pbase.data(), sizeof(uint64_t) * (G + 1), cudaMemcpyHostToDevice, s));
        batch_pairs_kernel<<<148 * 16, 256, 0, s>>>(dgp, dpb, G, M, u, v);
        MG_LAUNCH_CHECK();
    }
    // symmetric deduplicated CSR of the union; the union's previous buffers
    // are kept in W.built for the next batch
    csr_from_device_pairs((uint32_t)nv, M, u, v, W.built, b->ctx->cws, s);
    mg_graph *ug = &b->u;
    ug->n = (uint32_t)nv;
    ug->nnz = W.built.nnz;
    std::swap(ug->off.p, W.built.off.p);
    std::swap(ug->off.cap, W.built.off.cap);
    std::swap(ug->col.p, W.built.col.p);
    std::swap(ug->col.cap, W.built.col.cap);
    ug->wk = WK_UNIT;
    ug->mass = (double)ug->nnz;
    ug->integral = ug->nnz < 4294967296ull;
    MG_CUDA(cudaStreamSynchronize(s));
    batch_entry_offsets(b);
    b->mass.resize(G);
    b->integral.resize(G);
    for (uint32_t g = 0; g < G; g++) {
        b->mass[g] = (double)(b->eoff[g + 1] - b->eoff[g]);
        b->integral[g] = 1;
    }
}

void batch_from_host_csr(mg_batch *b, const uint64_t *voff, const uint64_t *offsets, const uint32_t *cols,
                         const void *w, int weight_type) {
    const uint32_t G = b->graphs;
    MG_CHECK(G >= 1 && voff != nullptr && offsets != nullptr, MG_ERR_INVALID, "batch: NULL offsets");
    MG_CHECK(voff[0] == 0, MG_ERR_INVALID, "batch: vertex_offsets[0] must be 0");
    for (uint32_t g = 0; g < G; g++)
        MG_CHECK(voff[g + 1] >= voff[g], MG_ERR_INVALID, "batch: vertex offsets must be non-decreasing");
    const uint64_t n = voff[G];
    MG_CHECK(n < 0xFFFFFFFFull, MG_ERR_UNSUPPORTED, "batch: more than 2^32-1 vertices in total");
    MG_CHECK(offsets[0] == 0, MG_ERR_INVALID, "offsets[0] must be 0");
    const uint64_t nnz = offsets[n];
    MG_CHECK(nnz < 0xFFFFFFFFull, MG_ERR_UNSUPPORTED, "batch: more than 2^32-1 directed entries in total");
    MG_CHECK(nnz == 0 || cols != nullptr, MG_ERR_INVALID, "cols is NULL");
    MG_CHECK(weight_type >= MG_WEIGHT_UNIT && weight_type <= MG_WEIGHT_F64, MG_ERR_INVALID, "bad weight type");
    MG_CHECK(weight_type == MG_WEIGHT_UNIT || nnz == 0 || w != nullptr, MG_ERR_INVALID, "weights is NULL");
    b->voff.resize(G + 1);
    b->eoff.resize(G + 1);
    for (uint32_t g = 0; g <= G; g++) {
        b->voff[g] = (uint32_t)voff[g];
        b->eoff[g] = offsets[voff[g]];
    }
    for (uint32_t g = 0; g < G; g++)
        MG_CHECK(b->eoff[g + 1] >= b->eoff[g], MG_ERR_INVALID, "offsets must be non-decreasing");
    // mass of each graph in its CSR order (src/graph/host_graph.cpp:112-115),
    // integrality, unit detection -- as graph_from_host_csr does per graph
    b->mass.assign(G, 0.0);
    b->integral.assign(G, 1);
    bool unit = true;
    for (uint32_t g = 0; g < G; g++) {
        const uint64_t e0 = b->eoff[g], e1 = b->eoff[g + 1];
        double mass = (double)(e1 - e0);
        bool nonint = false;
        if (weight_type != MG_WEIGHT_UNIT) {
            mass = 0;
            for (uint64_t e = e0; e < e1; e++) {
                double x = weight_type == MG_WEIGHT_F32 ? (double)((const float *)w)[e] : ((const double *)w)[e];
                mass += x;
                nonint |= (x < 0 || x != std::floor(x));
                unit &= (x == 1.0);
            }
        }
        b->mass[g] = mass;
        b->integral[g] = !nonint && mass < 4294967296.0;
    }
    mg_graph *u = &b->u;
    cudaStream_t s = b->ctx->stream;
    u->n = (uint32_t)n;
    u->nnz = nnz;
    {
        BatchWork &W = b->work;
        uint64_t *d64 = W.off64.ensure(n + 1);
        int *dbad = W.bad.ensure(1);
        uint32_t *dvoff = W.small.ensure(2 * (G + 1));
        MG_CUDA(cudaMemsetAsync(dbad, 0, sizeof(int), s));
        MG_CUDA(cudaMemcpyAsync(d64, offsets, sizeof(uint64_t) * (n + 1), cudaMemcpyHostToDevice, s));
        MG_CUDA(cudaMemcpyAsync(dvoff, b->voff.data(), sizeof(uint32_t) * (G + 1), cudaMemcpyHostToDevice, s));
        uint32_t *dcol = u->col.ensure(nnz + 1);
        if (nnz) MG_CUDA(cudaMemcpyAsync(dcol, cols, sizeof(uint32_t) * nnz, cudaMemcpyHostToDevice, s));
        uint32_t *uoff = u->off.ensure(n + 1);  // (allocations stay out of launch argument lists)
        batch_rows_kernel<<<148 * 16, 256, 0, s>>>(d64, (uint32_t)n, dvoff, G, dcol, uoff, dbad);
        MG_LAUNCH_CHECK();
        int hbad = 0;
        MG_CUDA(cudaMemcpyAsync(&hbad, dbad, sizeof(int), cudaMemcpyDeviceToHost, s));
        MG_CUDA(cudaStreamSynchronize(s));
        MG_CHECK(!(hbad & 1), MG_ERR_INVALID, "offsets must be non-decreasing");
        MG_CHECK(!(hbad & 2), MG_ERR_INVALID, "column index out of range");
    }
    if (weight_type == MG_WEIGHT_UNIT || unit) {
        u->wk = WK_UNIT;
    } else if (weight_type == MG_WEIGHT_F32) {
        u->wk = WK_F32;
        MG_CUDA(cudaMemcpyAsync(u->w32.ensure(nnz + 1), w, sizeof(float) * nnz, cudaMemcpyHostToDevice, s));
    } else {
        u->wk = WK_F64;
        MG_CUDA(cudaMemcpyAsync(u->w64.ensure(nnz + 1), w, sizeof(double) * nnz, cudaMemcpyHostToDevice, s));
    }
    double total = 0;
    int all_integral = 1;
    for (uint32_t g = 0; g < G; g++) {
        total += b->mass[g];
        all_integral &= b->integral[g];
    }
    u->mass = total;
    u->integral = all_integral;
    MG_CUDA(cudaStreamSynchronize(s));
}

}  // namespace mg
