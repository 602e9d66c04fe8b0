// noalloc.cu -- a local-move sweep that allocates nothing.
//
// Some callers cannot call cudaMalloc: a serving process that has handed its
// whole HBM budget to its own pool, or code that must not enter the CUDA
// allocator at all.  mg_local_move_noalloc gives them one local-move sweep on
// a graph they already hold in device memory.  The per-block hash tables,
// which every other sweep path takes from engine-owned allocations, live
// here in a fixed file-scope device array of kNoAllocScratchBytes.  Each
// block processes vertices in turn with its own slice of that array (room for
// pow2(2 * max degree + 2) slots); a vertex uses only the first
// pow2(2 * its degree + 2) slots of it as an open-addressing table, so the
// work per vertex follows its own degree, not the graph's maximum.  The arithmetic is the
// engine's FP64 gain (same tie-break, same version 1 / 2 rules), so for
// integral weights the result equals mg_local_move exactly.
#include <algorithm>
#include <mutex>

#include "handles.cuh"

namespace mg {
void set_orphan_error(const std::string &msg);
}

namespace {

using namespace mg;

constexpr size_t kNoAllocScratchBytes = 16u << 20;  // 16 MiB held by every GPU that loads the library
constexpr int kNoAllocThreads = 256;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

struct NoAllocArgs {
    const uint32_t *off, *col;
    const double *w;
    const uint32_t *C;
    const double *sigma, *k;
    uint32_t *C_new;
    uint32_t n;
    double m, two_m, r_m, r_two_m;
    int version, up;
};

// word 0 of the scratch: max degree (written by the first kernel)
__global__ void noalloc_maxdeg_kernel(const uint32_t *off, uint32_t n, uint32_t *out) {
    uint32_t mx = 0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        mx = max(mx, off[i + 1] - off[i]);
    mx = __reduce_max_sync(0xffffffffu, mx);
    if ((threadIdx.x & 31) == 0) atomicMax(out, mx);
}

__global__ void noalloc_clear_kernel(uint32_t *keys, double *vals, size_t slots) {
    for (size_t s = (size_t)blockIdx.x * blockDim.x + threadIdx.x; s < slots; s += (size_t)gridDim.x * blockDim.x) {
        keys[s] = kEmpty;
        vals[s] = 0.0;
    }
}

__device__ __forceinline__ bool nb_better(double g2, uint32_t c2, double g1, uint32_t c1, int up) {
    return g2 > g1 || (g2 == g1 && (up ? c2 < c1 : c2 > c1));
}

__global__ void __launch_bounds__(kNoAllocThreads) noalloc_move_kernel(NoAllocArgs A, uint32_t *tkeys,
                                                                       double *tvals, uint32_t tsize) {
    __shared__ double red_e[kNoAllocThreads / 32];
    __shared__ double red_g[kNoAllocThreads / 32];
    __shared__ uint32_t red_c[kNoAllocThreads / 32];
    uint32_t *keys = tkeys + (size_t)blockIdx.x * tsize;
    double *vals = tvals + (size_t)blockIdx.x * tsize;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (uint32_t v = blockIdx.x; v < A.n; v += gridDim.x) {
        const uint32_t src = A.C[v];
        const double ki = A.k[v];
        const double a = A.sigma[src] - ki;
        const uint32_t lo = A.off[v], hi = A.off[v + 1];
        // this vertex's table: the first ts slots of the block's slice, a
        // power of two >= 2 * degree + 2 (load <= 1/2); every slot it touches
        // lies below ts and is cleaned by its evaluation loop
        uint32_t ts = 32;
        while (ts < 2 * (hi - lo) + 2 && ts < tsize) ts <<= 1;
        double e_part = 0;
        for (uint32_t e = lo + threadIdx.x; e < hi; e += kNoAllocThreads) {
            const uint32_t j = A.col[e];
            const uint32_t c = A.C[j];
            const double w = A.w ? A.w[e] : 1.0;
            if (c != src) {
                const bool cand = A.version == 1 ? (A.up ? c < src : c > src) : true;
                if (!cand) continue;
                uint32_t s = hash_range(c, ts);
                for (uint32_t p = 0; p < ts; p++) {
                    uint32_t cur = ((volatile uint32_t *)keys)[s];
                    if (cur == c) break;
                    if (cur == kEmpty) {
                        uint32_t prev = atomicCAS(keys + s, kEmpty, c);
                        if (prev == kEmpty || prev == c) break;
                    }
                    s = s + 1 == ts ? 0 : s + 1;
                }
                atomicAdd(vals + s, w);
            } else if (j != v) {
                e_part += w;  // self-loops (j == v) stay out of e_src
            }
        }
        e_part = warp_sum(e_part);
        if (lane == 0) red_e[warp] = e_part;
        __syncthreads();
        double e_src = 0;
        for (int i = 0; i < kNoAllocThreads / 32; i++) e_src += red_e[i];
        double best = 0.0;
        uint32_t dst = src;
        for (uint32_t s = threadIdx.x; s < ts; s += kNoAllocThreads) {
            const uint32_t c = keys[s];
            if (c == kEmpty) continue;
            const double kic = vals[s];
            keys[s] = kEmpty;
            vals[s] = 0.0;
            double t = __dmul_rn(ki, __dsub_rn(a, A.sigma[c]));
            t = div_by(t, A.two_m, A.r_two_m);
            t = __dsub_rn(e_src, t);
            const double g = div_by(__dsub_rn(kic, t), A.m, A.r_m);
            if (nb_better(g, c, best, dst, A.up)) {
                best = g;
                dst = c;
            }
        }
        for (int o = 16; o > 0; o >>= 1) {
            double g2 = __shfl_xor_sync(0xffffffffu, best, o);
            uint32_t c2 = __shfl_xor_sync(0xffffffffu, dst, o);
            if (nb_better(g2, c2, best, dst, A.up)) {
                best = g2;
                dst = c2;
            }
        }
        __syncthreads();  // everyone has read red_e before it is reused
        if (lane == 0) {
            red_g[warp] = best;
            red_c[warp] = dst;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            for (int i = 0; i < kNoAllocThreads / 32; i++)
                if (nb_better(red_g[i], red_c[i], best, dst, A.up)) {
                    best = red_g[i];
                    dst = red_c[i];
                }
            uint32_t out = dst;
            if (A.version != 1) out = A.up ? (dst < src ? dst : src) : (dst > src ? dst : src);
            A.C_new[v] = out;
        }
        __syncthreads();  // table reset and red_* reads complete before the next vertex
    }
}

std::mutex g_noalloc_mu;
void *g_noalloc_addr[kMaxDevices] = {nullptr};

mg_status noalloc_fail(mg_status st, const std::string &msg) {
    set_orphan_error("mg_local_move_noalloc: " + msg);
    return st;
}

}  // namespace

extern "C" mg_status mg_local_move_noalloc(uint32_t n, const uint32_t *d_offsets, const uint32_t *d_cols,
                                           const double *d_weights, double mass, const uint32_t *d_C,
                                           const double *d_sigma, const double *d_k, uint32_t *d_C_new,
                                           int version, int up, void *stream) {
    if (!d_offsets || !d_cols || !d_C || !d_sigma || !d_k || !d_C_new)
        return noalloc_fail(MG_ERR_INVALID, "NULL argument");
    if (version < 0 || version > 2) return noalloc_fail(MG_ERR_INVALID, "version must be 0, 1 or 2");
    if (n == 0) return MG_OK;
    if (!(mass > 0)) return noalloc_fail(MG_ERR_INVALID, "mass must be positive");
    cudaStream_t s = (cudaStream_t)stream;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices)
        return noalloc_fail(MG_ERR_CUDA, "no current CUDA device");
    void *base = nullptr;
    {
        // once per device, with that device current: the device address of the
        // static array (its host-side name is only a stand-in)
        std::lock_guard<std::mutex> lock(g_noalloc_mu);
        if (!g_noalloc_addr[dev]) {
            cudaError_t e = cudaGetSymbolAddress(&g_noalloc_addr[dev], g_noalloc_scratch);
            if (e != cudaSuccess) {
                g_noalloc_addr[dev] = nullptr;
                return noalloc_fail(MG_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
            }
        }
        base = g_noalloc_addr[dev];
    }
    // word 0: max degree; tables start at byte 256
    uint32_t *d_maxdeg = (uint32_t *)base;
    if (cudaMemsetAsync(d_maxdeg, 0, sizeof(uint32_t), s) != cudaSuccess)
        return noalloc_fail(MG_ERR_CUDA, "memset failed");
    noalloc_maxdeg_kernel<<<148, 256, 0, s>>>(d_offsets, n, d_maxdeg);
    uint32_t maxdeg = 0;
    if (cudaMemcpyAsync(&maxdeg, d_maxdeg, sizeof maxdeg, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
        return noalloc_fail(MG_ERR_CUDA, cudaGetErrorString(cudaGetLastError()));
    const uint32_t tsize = pow2_at_least(2ull * maxdeg + 2, 32);
    const size_t table_bytes = (size_t)tsize * (sizeof(uint32_t) + sizeof(double));
    const size_t room = kNoAllocScratchBytes - 512;  // 256-byte header + alignment of the value array
    if (table_bytes > room)
        return noalloc_fail(MG_ERR_UNSUPPORTED, "max degree " + std::to_string(maxdeg) +
                                                    " needs a table larger than the static scratch (16 MiB)");
    uint32_t blocks = (uint32_t)std::min<size_t>({room / table_bytes, (size_t)148 * 4, (size_t)n});
    uint32_t *tkeys = (uint32_t *)((unsigned char *)base + 256);
    double *tvals = (double *)((unsigned char *)base + 256 + (((size_t)blocks * tsize * sizeof(uint32_t) + 255) & ~(size_t)255));
    const size_t slots = (size_t)blocks * tsize;
    // the array keeps the previous call's contents: clear the tables
    noalloc_clear_kernel<<<148 * 4, 256, 0, s>>>(tkeys, tvals, slots);
    NoAllocArgs A;
    A.off = d_offsets;
    A.col = d_cols;
    A.w = d_weights;
    A.C = d_C;
    A.sigma = d_sigma;
    A.k = d_k;
    A.C_new = d_C_new;
    A.n = n;
    A.m = mass / 2.0;
    A.two_m = 2.0 * A.m;
    A.r_m = 1.0 / A.m;
    A.r_two_m = 1.0 / A.two_m;
    A.version = version;
    A.up = up ? 1 : 0;
    noalloc_move_kernel<<<blocks, kNoAllocThreads, 0, s>>>(A, tkeys, tvals, tsize);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return noalloc_fail(MG_ERR_CUDA, cudaGetErrorString(e));
    return MG_OK;
}
