// coarsen.cu -- next-level graph from an assignment.
//
// Follows coarsen_graph_mg::coarsen_graph (src/coarsen_graph/coarsen_graph_mg.cu:2054-2240):
//   * dense, order-preserving relabel: flag used ids, scan, C' = scan[C]
//     (com_size_is_empty_all_range_cuda + InclusiveSum + renew_community_id_all_range_cuda,
//      :211-226, :267-286, :1330-1363);
//   * row r of the next level = every neighbour community c of the members of
//     r (r itself included, which carries the internal weight as a
//     self-loop) with the summed weight (aggregate_edges_and_weights_*,
//     :816-1125).
// The reference builds each row in a hash table (row order = slot order).
// Here every edge becomes a key (C'[u] << b) | C'[v], the keys are radix
// sorted and equal keys merged, so rows come out sorted by neighbour
// community.  For integral weights the merged sums are exact (prefix sums
// over 64-bit integers); for real weights they are double sums.  A symmetric
// integral graph is expanded from the transposed side in community order,
// which leaves only the high half of every key to sort.
#include <algorithm>
#include <type_traits>

#include "engine.cuh"

namespace mg {

namespace {

__global__ void mark_used_kernel(const uint32_t *C, uint32_t n, uint32_t *flags) {
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) flags[C[v]] = 1;
}

__global__ void apply_relabel_kernel(const uint32_t *C, uint32_t n, const uint32_t *newid, uint32_t *Cd) {
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) Cd[v] = newid[C[v]];
}

// key = (C'[u] << bc) | C'[v] per edge (u,v), payload = weight (if any).
// A block takes a tile of kExpandTile consecutive edges.  The rows that start
// inside the tile are marked at their first edge (a row id per position; of
// several rows starting at one position -- empty rows -- the largest, which is
// the non-empty one, wins), a prefix maximum over the tile then gives every
// edge its row, and the keys are written with coalesced loads and stores.
// One binary search per tile finds the row holding its first edge.
// TR (symmetric graphs): the rows are visited in member order -- off holds
// the offsets of the member-ordered expansion, member r's row starts at
// msrc[r] of the graph and its community is mcom[r] (non-decreasing in r) --
// and each entry (v, u) of member v's row is written as the key of its
// transpose, (C'[u] << bc) | C'[v].  The symmetric graph has the same keys
// either way, and this order has them sorted by their low half already.
// COMBINE (never with TR): the 32 edges a warp holds at a time are merged
// by key first (equal keys add their weights, a unit edge counting 1), and
// only one entry per distinct key is written, to the tile's own region of
// the output in arrival order; tcount[tile] receives the tile's entry count.
// Pays where communities repeat within rows (the end of a phase whose last
// sweep saw few distinct neighbour communities): the sort then sees far
// fewer keys.
constexpr int kExpandThreads = 256;
constexpr int kExpandPer = 16;
constexpr uint32_t kExpandTile = kExpandThreads * kExpandPer;

template <int WK, class PV, bool COMBINE = false, bool TR = false>
__global__ void __launch_bounds__(kExpandThreads)
    expand_keys_kernel(const uint32_t *off, const uint32_t *col, const void *w, uint32_t n, uint64_t m,
                       const uint32_t *Cd, int bc, uint64_t *keys, PV *vals, uint32_t *tcount,
                       const uint32_t *msrc, const uint32_t *mcom) {
    // tile position q lives at q + q/32 (one padding word per 32: the
    // per-thread runs of 16 positions then fall on distinct banks)
    __shared__ uint32_t rowat[kExpandTile + kExpandTile / 32];
    __shared__ uint32_t part[kExpandThreads];
    __shared__ uint32_t r0s, tcnt;
    __shared__ PV wstage[COMBINE ? kExpandThreads : 1];
    const uint32_t t = threadIdx.x;
    static_assert(!(COMBINE && TR), "the member-ordered expansion is not combined");
    if (COMBINE && t == 0) tcnt = 0;
    // the key and graph position of tile position q (edge e)
    auto entry = [&](uint32_t q, uint64_t e, uint64_t &key, uint64_t &p) {
        const uint32_t r = rowat[q + (q >> 5)];
        if constexpr (TR) {
            p = msrc[r] + (e - off[r]);
            key = ((uint64_t)Cd[__ldcs(col + p)] << bc) | mcom[r];
        } else {
            p = e;
            key = ((uint64_t)Cd[r] << bc) | Cd[__ldcs(col + e)];
        }
    };
    for (uint64_t E0 = (uint64_t)blockIdx.x * kExpandTile; E0 < m; E0 += (uint64_t)gridDim.x * kExpandTile) {
        const uint64_t E1 = E0 + kExpandTile < m ? E0 + kExpandTile : m;
        if (t == 0) {
            uint32_t lo = 0, hi = n - 1;  // last row with off[row] <= E0: the row of edge E0
            while (lo < hi) {
                const uint32_t mid = lo + ((hi - lo + 1) >> 1);
                if (off[mid] <= E0) lo = mid;
                else hi = mid - 1;
            }
            r0s = lo;
        }
        for (uint32_t q = t; q < kExpandTile + kExpandTile / 32; q += kExpandThreads) rowat[q] = 0;
        __syncthreads();
        const uint32_t r0 = r0s;
        if (t == 0) rowat[0] = r0;
        // rows r0+1, r0+2, ... that start inside the tile, 256 at a time
        for (uint32_t base = r0 + 1;; base += kExpandThreads) {
            const uint32_t j = base + t;
            bool inside = false;
            if (j < n) {
                const uint32_t st = off[j];
                inside = st < E1;
                if (inside) {
                    const uint32_t q = (uint32_t)(st - E0);
                    atomicMax(&rowat[q + (q >> 5)], j);
                }
            }
            // offsets are monotone: more rows can start inside only if the
            // batch's last one did
            if (!__syncthreads_or(t == kExpandThreads - 1 && inside)) break;
        }
        __syncthreads();
        // prefix maximum: 16 positions per thread, then across the threads
        uint32_t run = 0;
#pragma unroll
        for (int k = 0; k < kExpandPer; k++) {
            const uint32_t q = t * kExpandPer + k;
            run = max(run, rowat[q + (q >> 5)]);
            rowat[q + (q >> 5)] = run;
        }
        part[t] = run;
        __syncthreads();
        if (t < 32) {
            // exclusive prefix maximum of the 256 thread maxima: 8 per lane
            constexpr int L = kExpandThreads / 32;
            uint32_t loc[L], v = 0;
#pragma unroll
            for (int k = 0; k < L; k++) {
                v = max(v, part[t * L + k]);
                loc[k] = v;
            }
            uint32_t inc = v;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t y = __shfl_up_sync(0xffffffffu, inc, o);
                if ((int)t >= o) inc = max(inc, y);
            }
            uint32_t ex = __shfl_up_sync(0xffffffffu, inc, 1);
            if (t == 0) ex = 0;
#pragma unroll
            for (int k = 0; k < L; k++) part[t * L + k] = k ? max(ex, loc[k - 1]) : ex;
        }
        __syncthreads();
        {
            const uint32_t pre = part[t];
#pragma unroll
            for (int k = 0; k < kExpandPer; k++) {
                const uint32_t q = t * kExpandPer + k;
                rowat[q + (q >> 5)] = max(rowat[q + (q >> 5)], pre);
            }
        }
        __syncthreads();
        if constexpr (!COMBINE) {
#pragma unroll 4
            for (int k = 0; k < kExpandPer; k++) {
                const uint32_t q = k * kExpandThreads + t;
                const uint64_t e = E0 + q;
                if (e < E1) {
                    uint64_t key, p;
                    entry(q, e, key, p);
                    keys[e] = key;
                    if constexpr (WK == WK_F32) vals[e] = (PV)__ldcs((const float *)w + p);
                    else if constexpr (WK == WK_F64) vals[e] = (PV)__ldcs((const double *)w + p);
                    else if constexpr (WK == WK_U32) vals[e] = (PV)__ldcs((const uint32_t *)w + p);
                }
            }
        } else {
            const uint32_t lane = t & 31u;
            const uint64_t tile_base = E0;  // the tile's region of the output
#pragma unroll 2
            for (int k = 0; k < kExpandPer; k++) {
                const uint32_t q = k * kExpandThreads + t;
                const uint64_t e = E0 + q;
                uint64_t key = ~0ull;
                PV v = PV(0);
                if (e < E1) {
                    uint64_t p;
                    entry(q, e, key, p);
                    if constexpr (WK == WK_UNIT) v = PV(1);
                    else if constexpr (WK == WK_F32) v = (PV)__ldcs((const float *)w + p);
                    else if constexpr (WK == WK_F64) v = (PV)__ldcs((const double *)w + p);
                    else v = (PV)__ldcs((const uint32_t *)w + p);
                }
                const uint32_t peers = __match_any_sync(0xffffffffu, key);
                const bool lead = key != ~0ull && (uint32_t)(__ffs(peers) - 1) == lane;
                if constexpr (std::is_same<PV, uint32_t>::value) {
                    v = __reduce_add_sync(peers, v);
                } else {
                    wstage[t] = v;
                    __syncwarp();
                    if (lead) {
                        PV s = PV(0);
                        for (uint32_t mset = peers; mset; mset &= mset - 1) s += wstage[(t & ~31u) + __ffs(mset) - 1];
                        v = s;
                    }
                    __syncwarp();
                }
                const uint32_t lm = __ballot_sync(0xffffffffu, lead);
                if (lm) {
                    uint32_t pos = 0;
                    if (lane == (uint32_t)(__ffs(lm) - 1)) pos = atomicAdd(&tcnt, (uint32_t)__popc(lm));
                    pos = __shfl_sync(0xffffffffu, pos, __ffs(lm) - 1);
                    if (lead) {
                        const uint64_t o = tile_base + pos + __popc(lm & ((1u << lane) - 1u));
                        keys[o] = key;
                        vals[o] = v;
                    }
                }
            }
            __syncthreads();
            if (t == 0) {
                tcount[E0 / kExpandTile] = tcnt;
                tcnt = 0;
            }
        }
        __syncthreads();  // rowat (and the tile counter) are reused by the next tile
    }
}

// gather the tiles' combined entries into one dense array
template <class PV>
__global__ void compact_tiles_kernel(const uint64_t *keys, const PV *vals, const uint32_t *toff, uint64_t tiles,
                                     uint64_t *okeys, PV *ovals) {
    for (uint64_t tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
        const uint32_t a = toff[tile], b = toff[tile + 1];
        const uint64_t src = tile * kExpandTile;
        for (uint32_t i = threadIdx.x; i < b - a; i += blockDim.x) {
            okeys[a + i] = keys[src + i];
            ovals[a + i] = vals[src + i];
        }
    }
}

// member order of a symmetric coarsening: mkey[v] = (C'[v] << 32) | v, sorted
// on its community bits, gives the vertices grouped by community
__global__ void member_keys_kernel(const uint32_t *Cd, uint32_t n, uint64_t *mkey) {
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x)
        mkey[v] = ((uint64_t)Cd[v] << 32) | v;
}

// per member r: its row start in the graph, its community, its degree (the
// exclusive scan of the degrees gives the member-ordered expansion offsets)
__global__ void member_rows_kernel(const uint64_t *mkey, const uint32_t *off, uint32_t n, uint32_t *msrc,
                                   uint32_t *mcom, uint32_t *mdeg) {
    for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
        const uint64_t k = mkey[r];
        const uint32_t v = (uint32_t)k;
        const uint32_t lo = off[v];
        msrc[r] = lo;
        mcom[r] = (uint32_t)(k >> 32);
        mdeg[r] = off[v + 1] - lo;
    }
}

// head[i] = 1 where a run of equal keys starts
__global__ void run_heads_kernel(const uint64_t *keys, size_t m, uint32_t *head) {
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += (size_t)gridDim.x * blockDim.x)
        head[i] = (i == 0 || keys[i] != keys[i - 1]) ? 1u : 0u;
}

// compact run heads: ukey[s] = key, ustart[s] = position
__global__ void compact_runs_kernel(const uint64_t *keys, size_t m, const uint32_t *head, const uint32_t *seg,
                                    uint64_t *ukey, uint32_t *ustart) {
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += (size_t)gridDim.x * blockDim.x) {
        if (head[i]) {
            uint32_t s = seg[i];
            ukey[s] = keys[i];
            ustart[s] = (uint32_t)i;
        }
    }
}

// cols of the new CSR from the sorted unique keys
__global__ void emit_cols_kernel(const uint64_t *ukey, uint32_t u, int bc, uint32_t *col) {
    const uint64_t mask = (1ull << bc) - 1ull;
    for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < u; s += gridDim.x * blockDim.x)
        col[s] = (uint32_t)(ukey[s] & mask);
}
// off[r] = first unique key whose row is >= r (binary search; empty rows allowed)
__global__ void emit_offsets_kernel(const uint64_t *ukey, uint32_t u, int bc, uint32_t n_rows, uint32_t *off) {
    for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r <= n_rows; r += gridDim.x * blockDim.x) {
        uint32_t lo = 0, hi = u;
        while (lo < hi) {
            uint32_t mid = lo + ((hi - lo) >> 1);
            if ((uint32_t)(ukey[mid] >> bc) < r) lo = mid + 1;
            else hi = mid;
        }
        off[r] = lo;
    }
}

void emit_rows(const uint64_t *ukey, uint32_t u, int bc, uint32_t n_rows, uint32_t *off, uint32_t *col,
               cudaStream_t s);

// run weights as run lengths (unit weights)
template <class W>
__global__ void run_lengths_kernel(const uint32_t *ustart, uint32_t u, uint32_t m, W *w) {
    for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < u; s += gridDim.x * blockDim.x) {
        uint32_t end = s + 1 < u ? ustart[s + 1] : m;
        w[s] = (W)(end - ustart[s]);
    }
}

// integral weights: exact prefix sums over uint64, run sum = prefix difference
template <class T>
__global__ void to_u64_kernel(const T *v, size_t m, uint64_t *o) {
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += (size_t)gridDim.x * blockDim.x)
        o[i] = (uint64_t)v[i];
}
// (the sums of an integral graph are below its mass < 2^32: exact as uint32)
__global__ void run_diff_kernel(const uint32_t *ustart, uint32_t u, uint32_t m, const uint64_t *pre, uint32_t *w) {
    for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < u; s += gridDim.x * blockDim.x) {
        uint32_t end = s + 1 < u ? ustart[s + 1] : m;
        w[s] = (uint32_t)(pre[end] - pre[ustart[s]]);
    }
}

__global__ void u32_to_f64_kernel(const uint32_t *a, uint64_t m, double *o) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += (uint64_t)gridDim.x * blockDim.x)
        o[i] = (double)a[i];
}

// real weights: each thread sums 8 consecutive sorted entries run by run and
// adds each run piece to its run total
constexpr int kSegItems = 8;
__global__ void run_sums_kernel(const double *v, size_t m, const uint32_t *seg, const uint32_t *head, double *w) {
    size_t base = ((size_t)blockIdx.x * blockDim.x + threadIdx.x) * kSegItems;
    if (base >= m) return;
    size_t end = base + kSegItems < m ? base + kSegItems : m;
    uint32_t cur = seg[base] - (head[base] ? 0u : 1u);
    double acc = 0;
    for (size_t i = base; i < end; i++) {
        uint32_t s = seg[i] - (head[i] ? 0u : 1u);
        if (s != cur) {
            atomicAdd(w + cur, acc);
            acc = 0;
            cur = s;
        }
        acc += v[i];
    }
    atomicAdd(w + cur, acc);
}

__global__ void upper_degree_kernel(const uint32_t *off, const uint32_t *Cd, uint32_t n, uint64_t *up) {
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x)
        atomicAdd((unsigned long long *)up + Cd[v], (unsigned long long)(off[v + 1] - off[v]));
}

__global__ void pair_keys_kernel(const uint32_t *u, const uint32_t *v, uint64_t m, int bc, uint64_t *keys) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += (uint64_t)gridDim.x * blockDim.x) {
        uint32_t a = u[i], b = v[i];
        if (a == b) {
            keys[2 * i] = 1ull << (2 * bc);
            keys[2 * i + 1] = 1ull << (2 * bc);
        } else {
            keys[2 * i] = ((uint64_t)a << bc) | b;
            keys[2 * i + 1] = ((uint64_t)b << bc) | a;
        }
    }
}

// weighted pairs: both directions carry the pair's weight
__global__ void pair_weights_kernel(const double *w, uint64_t m, double *vals) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += (uint64_t)gridDim.x * blockDim.x) {
        vals[2 * i] = w[i];
        vals[2 * i + 1] = w[i];
    }
}

// weight of each unique key: the first of its run (duplicate pairs of a
// generator carry equal weights)
__global__ void run_first_values_kernel(const uint32_t *ustart, uint32_t u, const double *vals, double *w) {
    for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < u; s += gridDim.x * blockDim.x) w[s] = vals[ustart[s]];
}

__global__ void gather_compose_kernel(uint32_t *assign, const uint32_t *map, uint32_t n0) {
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n0; v += gridDim.x * blockDim.x)
        assign[v] = map[assign[v]];
}

__global__ void identity_kernel(uint32_t *C, uint32_t n) {
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) C[v] = v;
}

inline unsigned grid_for(uint64_t n, int threads = 256, uint64_t cap = 148ull * 16) {
    uint64_t g = ceil_div(n, threads);
    if (g > cap) g = cap;
    return (unsigned)(g ? g : 1);
}

void emit_rows(const uint64_t *ukey, uint32_t u, int bc, uint32_t n_rows, uint32_t *off, uint32_t *col,
               cudaStream_t s) {
    emit_cols_kernel<<<grid_for(u), 256, 0, s>>>(ukey, u, bc, col);
    MG_LAUNCH_CHECK();
    emit_offsets_kernel<<<grid_for((uint64_t)n_rows + 1), 256, 0, s>>>(ukey, u, bc, n_rows, off);
    MG_LAUNCH_CHECK();
}

// Sorted unique keys -> CSR (off, col) and per-run starts; returns the count.
uint32_t unique_runs(const uint64_t *keys, size_t m, int bc, uint32_t n_rows, LevelGraph &out, CoarsenWorkspace &ws,
                     cudaStream_t s, uint32_t **ustart_out, uint32_t **seg_out, uint32_t **head_out) {
    uint32_t *head = ws.rowcnt.ensure(m + 1);
    uint32_t *seg = ws.seg.ensure(m + 1);
    run_heads_kernel<<<grid_for(m), 256, 0, s>>>(keys, m, head);
    MG_LAUNCH_CHECK();
    exclusive_scan<uint32_t>(head, seg, m, seg + m, s, ws.prim);
    uint32_t u = 0;
    MG_CUDA(cudaMemcpyAsync(&u, seg + m, sizeof u, cudaMemcpyDeviceToHost, s));
    MG_CUDA(cudaStreamSynchronize(s));
    uint64_t *ukey = ws.u64tmp.ensure(u + 1);
    uint32_t *ustart = ws.u32tmp.ensure(u + 1);
    compact_runs_kernel<<<grid_for(m), 256, 0, s>>>(keys, m, head, seg, ukey, ustart);
    MG_LAUNCH_CHECK();
    out.n = n_rows;
    out.nnz = u;
    uint32_t *off = out.off.ensure((size_t)n_rows + 1);
    uint32_t *col = out.col.ensure(u + 1);
    if (u == 0) {
        MG_CUDA(cudaMemsetAsync(off, 0, sizeof(uint32_t) * ((size_t)n_rows + 1), s));
    } else {
        emit_rows(ukey, u, bc, n_rows, off, col, s);
    }
    *ustart_out = ustart;
    *seg_out = seg;
    *head_out = head;
    return u;
}

// ---- sorted keys -> CSR in two tiled passes (integral weights) -------------
// A tile of kRunTile sorted keys: each thread takes kRunPer consecutive keys
// (staged in shared memory); a key starts a run when it differs from the one
// before it.  Pass 1 counts the runs of every tile; pass 2, given the tiles'
// run offsets, writes every run's column and first position and the row
// offsets (a run whose row differs from the previous key's opens that row and
// every empty row before it).
constexpr int kRunThreads = 256;
constexpr int kRunPer = 16;
constexpr uint32_t kRunTile = kRunThreads * kRunPer;

__global__ void __launch_bounds__(kRunThreads) run_count_kernel(const uint64_t *keys, size_t m, uint32_t *tcount) {
    __shared__ uint32_t wsum[kRunThreads / 32];
    const uint32_t t = threadIdx.x;
    for (size_t tile = blockIdx.x; tile * kRunTile < m; tile += gridDim.x) {
        const size_t t0 = tile * kRunTile;
        uint32_t c = 0;
#pragma unroll 4
        for (int k = 0; k < kRunPer; k++) {
            const size_t i = t0 + (size_t)k * kRunThreads + t;  // coalesced; heads need no order here
            if (i < m) c += (i == 0 || keys[i] != keys[i - 1]) ? 1u : 0u;
        }
        c = warp_sum(c);
        if ((t & 31) == 0) wsum[t >> 5] = c;
        __syncthreads();
        if (t == 0) {
            uint32_t s = 0;
            for (int w = 0; w < kRunThreads / 32; w++) s += wsum[w];
            tcount[tile] = s;
        }
        __syncthreads();
    }
}

// rows [r0, r1] of a long gap of empty rows all start at p (filled by
// fill_gaps_kernel, so that no thread walks millions of empty rows)
struct RowGap {
    uint32_t r0, r1, p;
};
constexpr uint32_t kInlineRows = 64;

__device__ __forceinline__ void set_rows(uint32_t *off, uint32_t r0, uint32_t r1, uint32_t p, RowGap *gaps,
                                         uint32_t *ngaps) {
    if (r0 > r1) return;
    if (r1 - r0 < kInlineRows) {
        for (uint32_t r = r0; r <= r1; r++) off[r] = p;
    } else {
        gaps[atomicAdd(ngaps, 1u)] = RowGap{r0, r1, p};
    }
}

__global__ void fill_gaps_kernel(const RowGap *gaps, const uint32_t *ngaps, uint32_t *off) {
    const uint32_t ng = *ngaps;
    for (uint32_t gi = blockIdx.x; gi < ng; gi += gridDim.x) {
        const RowGap gp = gaps[gi];
        for (uint32_t r = gp.r0 + threadIdx.x; r <= gp.r1; r += blockDim.x) off[r] = gp.p;
    }
}

// Pass 2.  A thread holds its 16 keys (and the one before them) in
// registers; the tile's runs are staged in shared memory (column, first
// position) and written out with coalesced stores.  LEN (unit weights): also
// the run lengths, each the distance to the next run's start; the last run
// of a tile ends in a later tile and gets its length from
// run_tail_lengths_kernel.
template <bool LEN>
__global__ void __launch_bounds__(kRunThreads) run_emit_kernel(const uint64_t *keys, size_t m, int bc,
                                                               uint32_t n_rows, const uint32_t *toff, uint32_t u,
                                                               uint32_t *col, uint32_t *ustart, uint32_t *len,
                                                               uint32_t *off, RowGap *gaps, uint32_t *ngaps) {
    // logical position x (0: the key before the tile, q + 1: the tile's q-th
    // key) lives at x + x/16: a thread's 16 consecutive keys then fall on
    // different banks than its neighbours'.  Reused for the staged runs.
    constexpr uint32_t kSk = kRunTile + 1 + (kRunTile + 1) / 16 + 1;
    static_assert(kSk * sizeof(uint64_t) >= 2 * kRunTile * sizeof(uint32_t), "staging fits in the key buffer");
    __shared__ uint64_t sk[kSk];
    __shared__ uint32_t wsum[kRunThreads / 32];
    uint32_t *scol = (uint32_t *)sk, *sst = scol + kRunTile;
    const uint32_t t = threadIdx.x, lane = t & 31u, warp = t >> 5;
    const uint64_t mask = (1ull << bc) - 1ull;
    for (size_t tile = blockIdx.x; tile * kRunTile < m; tile += gridDim.x) {
        const size_t t0 = tile * kRunTile;
        const uint32_t tn = (uint32_t)(m - t0 < kRunTile ? m - t0 : kRunTile);
        for (uint32_t q = t; q < tn; q += kRunThreads) sk[(q + 1) + ((q + 1) >> 4)] = keys[t0 + q];
        if (t == 0) sk[0] = t0 ? keys[t0 - 1] : ~0ull;
        __syncthreads();
        // this thread's keys: positions [t * kRunPer, (t + 1) * kRunPer) of the tile
        uint64_t kk[kRunPer + 1];
        uint32_t c = 0;
#pragma unroll
        for (int k = 0; k <= kRunPer; k++) {
            const uint32_t x = t * kRunPer + k;  // logical position (key q = x - 1)
            kk[k] = x <= tn ? sk[x + (x >> 4)] : ~0ull;
        }
#pragma unroll
        for (int k = 0; k < kRunPer; k++) {
            const uint32_t q = t * kRunPer + k;
            if (q < tn && ((t0 == 0 && q == 0) || kk[k + 1] != kk[k])) c++;
        }
        // exclusive prefix of the heads over the tile's threads
        uint32_t inc = c;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, inc, o);
            if ((int)lane >= o) inc += y;
        }
        if (lane == 31) wsum[warp] = inc;
        __syncthreads();  // every thread's keys are in registers: sk becomes the staging area
        uint32_t before = 0, nr = 0;
        for (uint32_t w = 0; w < kRunThreads / 32; w++) {
            if (w < warp) before += wsum[w];
            nr += wsum[w];
        }
        const uint32_t base = toff[tile];
        uint32_t lp = before + inc - c;  // this thread's first run, within the tile
#pragma unroll
        for (int k = 0; k < kRunPer; k++) {
            const uint32_t q = t * kRunPer + k;
            if (q >= tn) break;
            const uint64_t key = kk[k + 1], prev = kk[k];
            const bool first = t0 == 0 && q == 0;
            if (!first && key == prev) continue;
            scol[lp] = (uint32_t)(key & mask);
            sst[lp] = (uint32_t)(t0 + q);
            // rows (previous key's row, this row] start at this run
            const uint32_t row = (uint32_t)(key >> bc);
            const uint32_t r0 = first ? 0u : (uint32_t)(prev >> bc) + 1u;
            set_rows(off, r0, row, base + lp, gaps, ngaps);
            lp++;
        }
        // after the last key: the remaining rows (and off[n_rows]) end at u
        if (t0 + tn == m && tn > 0 && t == (tn - 1) / kRunPer) {
            set_rows(off, (uint32_t)(keys[t0 + tn - 1] >> bc) + 1u, n_rows, u, gaps, ngaps);
        }
        __syncthreads();
        for (uint32_t i = t; i < nr; i += kRunThreads) {
            const uint32_t st = sst[i];
            col[base + i] = scol[i];
            ustart[base + i] = st;
            if (LEN && i + 1 < nr) len[base + i] = sst[i + 1] - st;
        }
        __syncthreads();  // sk and wsum are reused by the next tile
    }
}

// LEN: the length of each tile's last run, which ends at the next run's start
// (or at the end of the keys)
__global__ void run_tail_lengths_kernel(const uint32_t *toff, uint64_t tiles, uint32_t u, uint32_t m,
                                        const uint32_t *ustart, uint32_t *len) {
    for (uint64_t tile = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; tile < tiles;
         tile += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t a = toff[tile], b = toff[tile + 1];
        if (a == b) continue;  // no run starts in this tile
        const uint32_t end = b < u ? ustart[b] : m;
        len[b - 1] = end - ustart[b - 1];
    }
}

}  // namespace

// Sorted keys -> CSR (off, col) and per-run starts; returns the count.  For
// callers that need no per-entry run index (integral weights).
uint32_t unique_runs_tiled(const uint64_t *keys, size_t m, int bc, uint32_t n_rows, LevelGraph &out,
                           CoarsenWorkspace &ws, cudaStream_t s, uint32_t **ustart_out, bool lengths) {
    const uint64_t tiles = ceil_div(m, kRunTile);
    uint32_t *tcount = ws.tcount.ensure(tiles + 1);
    const unsigned grid = (unsigned)std::min<uint64_t>(tiles, 148ull * 8);
    run_count_kernel<<<grid, kRunThreads, 0, s>>>(keys, m, tcount);
    MG_LAUNCH_CHECK();
    exclusive_scan<uint32_t>(tcount, tcount, tiles, tcount + tiles, s, ws.prim);
    uint32_t u = 0;
    MG_CUDA(cudaMemcpyAsync(&u, tcount + tiles, sizeof u, cudaMemcpyDeviceToHost, s));
    MG_CUDA(cudaStreamSynchronize(s));
    uint32_t *ustart = ws.u32tmp.ensure((size_t)u + 1);
    out.n = n_rows;
    out.nnz = u;
    uint32_t *off = out.off.ensure((size_t)n_rows + 1);
    uint32_t *col = out.col.ensure((size_t)u + 1);
    // at most one gap per run, plus the rows after the last key
    RowGap *gaps = (RowGap *)ws.u64tmp.ensure(((size_t)u + 2) * sizeof(RowGap) / sizeof(uint64_t) + 2);
    uint32_t *ngaps = ws.rowcnt.ensure(1);
    MG_CUDA(cudaMemsetAsync(ngaps, 0, sizeof(uint32_t), s));
    if (lengths) {
        uint32_t *len = out.wi.ensure((size_t)u + 1);
        run_emit_kernel<true><<<grid, kRunThreads, 0, s>>>(keys, m, bc, n_rows, tcount, u, col, ustart, len, off,
                                                           gaps, ngaps);
        MG_LAUNCH_CHECK();
        run_tail_lengths_kernel<<<grid_for(tiles), 256, 0, s>>>(tcount, tiles, u, (uint32_t)m, ustart, len);
        MG_LAUNCH_CHECK();
    } else {
        run_emit_kernel<false><<<grid, kRunThreads, 0, s>>>(keys, m, bc, n_rows, tcount, u, col, ustart, nullptr,
                                                            off, gaps, ngaps);
        MG_LAUNCH_CHECK();
    }
    fill_gaps_kernel<<<148 * 8, 256, 0, s>>>(gaps, ngaps, off);
    MG_LAUNCH_CHECK();
    *ustart_out = ustart;
    return u;
}

void level_weights_f64(const GraphView &g, double *out, cudaStream_t s) {
    if (g.nnz == 0) return;
    if (g.wk == WK_F64) {
        MG_CUDA(cudaMemcpyAsync(out, g.w, sizeof(double) * g.nnz, cudaMemcpyDeviceToDevice, s));
        return;
    }
    MG_CHECK(g.wk == WK_U32, MG_ERR_INVALID, "level_weights_f64: unexpected weight kind");
    u32_to_f64_kernel<<<grid_for(g.nnz), 256, 0, s>>>((const uint32_t *)g.w, g.nnz, out);
    MG_LAUNCH_CHECK();
}

uint32_t relabel_dense(const uint32_t *C, uint32_t n, uint32_t *C_dense, CoarsenWorkspace &ws, cudaStream_t s) {
    if (n == 0) return 0;
    uint32_t *flags = ws.flags.ensure((size_t)n + 1);
    uint32_t *newid = ws.newid.ensure((size_t)n + 1);
    MG_CUDA(cudaMemsetAsync(flags, 0, sizeof(uint32_t) * n, s));
    mark_used_kernel<<<grid_for(n), 256, 0, s>>>(C, n, flags);
    MG_LAUNCH_CHECK();
    exclusive_scan<uint32_t>(flags, newid, n, newid + n, s, ws.prim);
    apply_relabel_kernel<<<grid_for(n), 256, 0, s>>>(C, n, newid, C_dense);
    MG_LAUNCH_CHECK();
    uint32_t nn = 0;
    MG_CUDA(cudaMemcpyAsync(&nn, newid + n, sizeof nn, cudaMemcpyDeviceToHost, s));
    MG_CUDA(cudaStreamSynchronize(s));
    return nn;
}

void coarsen_level(const GraphView &g, const uint32_t *Cd, uint32_t n_new, int integral, LevelGraph &out,
                   CoarsenWorkspace &ws, cudaStream_t s, uint64_t *upper_degree_off, bool combine) {
    const size_t m = g.nnz;
    const int bc = bits_for(n_new);
    if (upper_degree_off) {
        MG_CUDA(cudaMemsetAsync(upper_degree_off, 0, sizeof(uint64_t) * ((size_t)n_new + 1), s));
        upper_degree_kernel<<<grid_for(g.n), 256, 0, s>>>(g.off, Cd, g.n, upper_degree_off);
        MG_LAUNCH_CHECK();
        exclusive_scan<uint64_t>(upper_degree_off, upper_degree_off, n_new, upper_degree_off + n_new, s, ws.prim);
    }
    // integral graphs: the next level's weights as exact 32-bit integers
    out.wk = integral ? WK_U32 : WK_F64;
    out.symmetric = g.symmetric && integral;
    if (m == 0) {
        out.n = n_new;
        out.nnz = 0;
        MG_CUDA(cudaMemsetAsync(out.off.ensure((size_t)n_new + 1), 0, sizeof(uint32_t) * ((size_t)n_new + 1), s));
        out.col.ensure(1);
        out.w.ensure(1);
        out.wi.ensure(1);
        return;
    }
    if (g.wk == WK_UNIT && !integral) combine = false;  // (a unit graph is always integral)
    // Symmetric integral graphs: expand from the transposed side in member
    // order (vertices grouped by community, communities ascending), so the
    // keys arrive sorted by their low half and the stable sort needs only the
    // high half's passes; equal keys merge into exact integer sums in any
    // order, so the CSR is the same as the full sort's.  Not with combining:
    // the combined keys are few, and the member order costs more than the
    // passes it saves (R-MAT-24 level 1 -> 2: 17.8 ms full sort, 20.4 ms
    // member order).
    const bool tr = g.symmetric && integral && !combine;
    const uint32_t *msrc = nullptr, *mcom = nullptr, *eoff = g.off;
    if (tr) {
        // vertices sorted by community (stable: ascending ids inside one)
        uint64_t *mk = ws.keys.ensure(std::max<size_t>(m, g.n) + 1);
        uint64_t *mk2 = ws.keys_alt.ensure(std::max<size_t>(m, g.n) + 1);
        member_keys_kernel<<<grid_for(g.n), 256, 0, s>>>(Cd, g.n, mk);
        MG_LAUNCH_CHECK();
        const bool mf = radix_sort<NoVal>(mk, (NoVal *)nullptr, mk2, (NoVal *)nullptr, g.n, 32 + bc, s, ws.prim, 32);
        uint32_t *ms = ws.msrc.ensure((size_t)g.n + 1), *mc = ws.mcom.ensure((size_t)g.n + 1);
        uint32_t *vo = ws.voff.ensure((size_t)g.n + 1);
        member_rows_kernel<<<grid_for(g.n), 256, 0, s>>>(mf ? mk2 : mk, g.off, g.n, ms, mc, vo);
        MG_LAUNCH_CHECK();
        exclusive_scan<uint32_t>(vo, vo, g.n, vo + g.n, s, ws.prim);
        msrc = ms;
        mcom = mc;
        eoff = vo;
    }
    uint64_t *keys = ws.keys.ensure(m);
    uint64_t *keys2 = ws.keys_alt.ensure(m);
    // combined entries carry their summed weight (unit edges count 1)
    const bool weighted = g.wk != WK_UNIT || combine;
    double *vals = weighted ? ws.vals.ensure(m + 1) : nullptr;
    double *vals2 = weighted ? ws.vals_alt.ensure(m + 1) : nullptr;
    // integral weights travel through the sort as 32-bit integers (exact:
    // every weight of an integral graph is below 2^32), real ones as double
    const bool ipay = weighted && integral;
    uint32_t *ivals = (uint32_t *)vals, *ivals2 = (uint32_t *)vals2;
    // one block per tile, at most 8 resident per SM (grid-stride over tiles)
    const uint64_t tiles = ceil_div(m, kExpandTile);
    const unsigned gw = grid_for(tiles, 1, 148ull * 8);
    uint32_t *tcount = combine ? ws.tcount.ensure(tiles + 1) : nullptr;
    auto expand = [&](auto *pv, auto comb, auto trv) {
        using PV = typename std::remove_pointer<decltype(pv)>::type;
        constexpr bool CB = decltype(comb)::value, TR = decltype(trv)::value;
        if (g.wk == WK_UNIT)
            expand_keys_kernel<WK_UNIT, PV, CB, TR><<<gw, kExpandThreads, 0, s>>>(eoff, g.col, g.w, g.n, m, Cd, bc,
                                                                                   keys, pv, tcount, msrc, mcom);
        else if (g.wk == WK_F32)
            expand_keys_kernel<WK_F32, PV, CB, TR><<<gw, kExpandThreads, 0, s>>>(eoff, g.col, g.w, g.n, m, Cd, bc,
                                                                                  keys, pv, tcount, msrc, mcom);
        else if (g.wk == WK_U32)
            expand_keys_kernel<WK_U32, PV, CB, TR><<<gw, kExpandThreads, 0, s>>>(eoff, g.col, g.w, g.n, m, Cd, bc,
                                                                                  keys, pv, tcount, msrc, mcom);
        else
            expand_keys_kernel<WK_F64, PV, CB, TR><<<gw, kExpandThreads, 0, s>>>(eoff, g.col, g.w, g.n, m, Cd, bc,
                                                                                  keys, pv, tcount, msrc, mcom);
        MG_LAUNCH_CHECK();
    };
    // the sort's input: every edge (mm = m), or the combined entries gathered
    // densely into the alternate buffers (mm = their count)
    size_t mm = m;
    if (combine) {
        if (ipay) expand(ivals, std::true_type(), std::false_type());
        else expand(vals, std::true_type(), std::false_type());
        exclusive_scan<uint32_t>(tcount, tcount, tiles, tcount + tiles, s, ws.prim);
        uint32_t d = 0;
        MG_CUDA(cudaMemcpyAsync(&d, tcount + tiles, sizeof d, cudaMemcpyDeviceToHost, s));
        MG_CUDA(cudaStreamSynchronize(s));
        const unsigned gc = grid_for(tiles, 1, 148ull * 16);
        if (ipay) compact_tiles_kernel<uint32_t><<<gc, 256, 0, s>>>(keys, ivals, tcount, tiles, keys2, ivals2);
        else compact_tiles_kernel<double><<<gc, 256, 0, s>>>(keys, vals, tcount, tiles, keys2, vals2);
        MG_LAUNCH_CHECK();
        std::swap(keys, keys2);
        std::swap(vals, vals2);
        std::swap(ivals, ivals2);
        mm = d;
    } else {
        if (tr && ipay) expand(ivals, std::false_type(), std::true_type());
        else if (tr) expand(vals, std::false_type(), std::true_type());
        else if (ipay) expand(ivals, std::false_type(), std::false_type());
        else expand(vals, std::false_type(), std::false_type());
    }
    // the member-ordered expansion is sorted by the low half already
    const int lo = tr ? bc : 0;
    bool flipped;
    if (ipay) flipped = radix_sort<uint32_t>(keys, ivals, keys2, ivals2, mm, 2 * bc, s, ws.prim, lo);
    else if (weighted) flipped = radix_sort<double>(keys, vals, keys2, vals2, mm, 2 * bc, s, ws.prim, lo);
    else flipped = radix_sort<NoVal>(keys, (NoVal *)nullptr, keys2, (NoVal *)nullptr, mm, 2 * bc, s, ws.prim, lo);
    const uint64_t *sk = flipped ? keys2 : keys;
    const double *sv = flipped ? vals2 : vals;
    uint32_t *ustart, *seg = nullptr, *head = nullptr;
    // integral weights need only each run's first position; real weights
    // also the run index of every entry (segmented sums)
    // (unit weights of an integral graph: the run lengths come with the runs)
    uint32_t u = integral ? unique_runs_tiled(sk, mm, bc, n_new, out, ws, s, &ustart, !weighted)
                          : unique_runs(sk, mm, bc, n_new, out, ws, s, &ustart, &seg, &head);
    if (integral && !weighted) {
        // weights written by unique_runs_tiled
    } else if (!weighted) {
        double *w = out.w.ensure(u + 1);
        run_lengths_kernel<double><<<grid_for(u), 256, 0, s>>>(ustart, u, (uint32_t)mm, w);
        MG_LAUNCH_CHECK();
    } else if (integral) {
        // exact: 64-bit prefix sums over the sorted weights, run sum = difference
        uint64_t *pre = (uint64_t *)(flipped ? vals : vals2);
        to_u64_kernel<uint32_t><<<grid_for(mm), 256, 0, s>>>(flipped ? ivals2 : ivals, mm, pre);
        MG_LAUNCH_CHECK();
        exclusive_scan<uint64_t>(pre, pre, mm, pre + mm, s, ws.prim);
        uint32_t *wi = out.wi.ensure(u + 1);
        run_diff_kernel<<<grid_for(u), 256, 0, s>>>(ustart, u, (uint32_t)mm, pre, wi);
        MG_LAUNCH_CHECK();
    } else {
        double *w = out.w.ensure(u + 1);
        MG_CUDA(cudaMemsetAsync(w, 0, sizeof(double) * u, s));
        run_sums_kernel<<<(unsigned)ceil_div(ceil_div(mm, kSegItems), 256), 256, 0, s>>>(sv, mm, seg, head, w);
        MG_LAUNCH_CHECK();
    }
}

void csr_from_device_pairs(uint32_t n, uint64_t m, const uint32_t *u, const uint32_t *v, LevelGraph &out,
                           CoarsenWorkspace &ws, cudaStream_t s, const double *w) {
    const size_t mm = 2 * m;
    MG_CHECK(mm < 0xFFFFFFFFull, MG_ERR_UNSUPPORTED, "graph has more than 2^32-1 directed entries");
    out.wk = WK_F64;
    if (m == 0) {
        out.n = n;
        out.nnz = 0;
        MG_CUDA(cudaMemsetAsync(out.off.ensure((size_t)n + 1), 0, sizeof(uint32_t) * ((size_t)n + 1), s));
        out.col.ensure(1);
        out.w.ensure(1);
        return;
    }
    const int bc = bits_for(n);
    uint64_t *keys = ws.keys.ensure(mm + 1);
    uint64_t *keys2 = ws.keys_alt.ensure(mm + 1);
    pair_keys_kernel<<<grid_for(m), 256, 0, s>>>(u, v, m, bc, keys);
    MG_LAUNCH_CHECK();
    // self-loop markers (bit 2*bc set) sort last and are dropped below
    bool flipped;
    const double *sv = nullptr;
    if (w) {
        double *vals = ws.vals.ensure(mm + 1), *vals2 = ws.vals_alt.ensure(mm + 1);
        pair_weights_kernel<<<grid_for(m), 256, 0, s>>>(w, m, vals);
        MG_LAUNCH_CHECK();
        flipped = radix_sort<double>(keys, vals, keys2, vals2, mm, 2 * bc + 1, s, ws.prim);
        sv = flipped ? vals2 : vals;
    } else {
        flipped = radix_sort<NoVal>(keys, (NoVal *)nullptr, keys2, (NoVal *)nullptr, mm, 2 * bc + 1, s, ws.prim);
    }
    const uint64_t *sk = flipped ? keys2 : keys;
    uint32_t *head = ws.rowcnt.ensure(mm + 1);
    uint32_t *seg = ws.seg.ensure(mm + 1);
    run_heads_kernel<<<grid_for(mm), 256, 0, s>>>(sk, mm, head);
    MG_LAUNCH_CHECK();
    exclusive_scan<uint32_t>(head, seg, mm, seg + mm, s, ws.prim);
    uint32_t nu = 0;
    uint64_t last = 0;
    MG_CUDA(cudaMemcpyAsync(&nu, seg + mm, sizeof nu, cudaMemcpyDeviceToHost, s));
    MG_CUDA(cudaMemcpyAsync(&last, sk + mm - 1, sizeof last, cudaMemcpyDeviceToHost, s));
    MG_CUDA(cudaStreamSynchronize(s));
    uint64_t *ukey = ws.u64tmp.ensure((size_t)nu + 1);
    uint32_t *ustart = ws.u32tmp.ensure((size_t)nu + 1);
    compact_runs_kernel<<<grid_for(mm), 256, 0, s>>>(sk, mm, head, seg, ukey, ustart);
    MG_LAUNCH_CHECK();
    uint32_t uu = nu - (last == (1ull << (2 * bc)) ? 1u : 0u);
    out.n = n;
    out.nnz = uu;
    uint32_t *off = out.off.ensure((size_t)n + 1);
    uint32_t *col = out.col.ensure((size_t)uu + 1);
    if (uu == 0) {
        MG_CUDA(cudaMemsetAsync(off, 0, sizeof(uint32_t) * ((size_t)n + 1), s));
    } else {
        emit_rows(ukey, uu, bc, n, off, col, s);
        if (w) {
            double *w = out.w.ensure((size_t)uu + 1);
            run_first_values_kernel<<<grid_for(uu), 256, 0, s>>>(ustart, uu, sv, w);
            MG_LAUNCH_CHECK();
        }
    }
}

void gather_compose(uint32_t *assign, const uint32_t *map, uint32_t n0, cudaStream_t s) {
    if (n0 == 0) return;
    gather_compose_kernel<<<grid_for(n0), 256, 0, s>>>(assign, map, n0);
    MG_LAUNCH_CHECK();
}

void fill_identity(uint32_t *C, uint32_t n, cudaStream_t s) {
    if (n == 0) return;
    identity_kernel<<<grid_for(n), 256, 0, s>>>(C, n);
    MG_LAUNCH_CHECK();
}

}  // namespace mg
