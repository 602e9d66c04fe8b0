// lm_kernels.cuh -- the local-move sweep kernels and their launcher, shared by
// the single-graph sweep (local_move.cu) and the batched sweep
// (local_move_batch.cu).  Included by exactly those two translation units.
#pragma once

#include <cooperative_groups.h>

#include <algorithm>
#include <map>
#include <mutex>
#include <set>
#include <tuple>
#include <utility>
#include <vector>

#include "engine.cuh"

namespace mg {
namespace lmk {

struct LMArgs {
    const uint32_t *__restrict__ off;
    const uint32_t *__restrict__ col;
    const void *__restrict__ w;
    const uint32_t *__restrict__ P;
    uint32_t *__restrict__ N;
    const double *__restrict__ k;
    const double *__restrict__ sigma;
    const uint32_t *__restrict__ perm;
    // single-graph sweeps: the row range of every class-list entry, read
    // beside perm so that a vertex's edges do not wait for its id (NULL in
    // batched sweeps)
    const uint2 *__restrict__ rows;
    GainK K;             // gain constants of the graph
    int up;
    int integral;
    int agg;             // communities repeat among neighbours: lane-local run combining (table kernels)
    int split;           // cluster tables: split rows over the CTAs, combine in the warp, insert via DSMEM
    int first;           // the level's first sweep (P = identity, sigma = k): table-free kernels
    SweepAcc *acc;
    // batched sweeps: graph of each vertex, per-graph control word and gain
    // constants, the three assignment buffers, sum_in per vertex, and the
    // sweep direction in device memory
    const uint32_t *__restrict__ gid;
    const uint32_t *__restrict__ pgid;  // graph of each entry of perm
    const uint32_t *__restrict__ gword;
    const GainK *__restrict__ gk;
    uint32_t *Cb0, *Cb1, *Cb2;
    double *__restrict__ sinv;
    const int *__restrict__ up_dev;
};

// Per-vertex view of a sweep: the assignment read (P) and written (N) and the
// gain constants.  A batched sweep takes them from the vertex's graph and
// skips the vertices of graphs that are not active.
struct VView {
    const uint32_t *P;
    uint32_t *N;
    GainK K;
};

__device__ __forceinline__ uint32_t *buf_sel(const LMArgs &A, uint32_t b) {
    return b == 0 ? A.Cb0 : b == 1 ? A.Cb1 : A.Cb2;
}

template <int BT>
__device__ __forceinline__ bool vview_g(const LMArgs &A, uint32_t g, VView &v) {
    if constexpr (BT == 0) {
        v.P = A.P;
        v.N = A.N;
        return true;
    } else {
        const uint32_t w = A.gword[g];
        if (!(w & kGwActive)) return false;
        v.P = buf_sel(A, gw_p(w));
        v.N = buf_sel(A, gw_n(w));
        v.K = A.gk[g];
        return true;
    }
}

// vertex i, graph from the per-vertex table
template <int BT>
__device__ __forceinline__ bool vview(const LMArgs &A, uint32_t i, VView &v) {
    return vview_g<BT>(A, BT ? A.gid[i] : 0u, v);
}

// entry pos of the bins list, graph from the list's own table
template <int BT>
__device__ __forceinline__ bool vview_at(const LMArgs &A, uint32_t pos, VView &v) {
    return vview_g<BT>(A, BT ? A.pgid[pos] : 0u, v);
}

template <int BT>
__device__ __forceinline__ const GainK &kref(const LMArgs &A, const VView &v) {
    if constexpr (BT == 0) return A.K;
    else return v.K;
}

template <int BT>
__device__ __forceinline__ int load_up(const LMArgs &A) {
    if constexpr (BT == 0) return A.up;
    else return *A.up_dev;
}

// sum_in contribution of vertex i: into the thread's running sum (single
// graph) or into the per-vertex array (batched; summed per graph later)
template <int BT>
__device__ __forceinline__ void put_sin(const LMArgs &A, uint32_t i, double &sin, double x) {
    if constexpr (BT == 0) sin += x;
    else A.sinv[i] = x;
}

template <int WK>
__device__ __forceinline__ double wload(const void *w, uint32_t e) {
    if constexpr (WK == WK_UNIT) return 1.0;
    else if constexpr (WK == WK_U32) return u2d(__ldcs((const uint32_t *)w + e));
    else if constexpr (WK == WK_F32 || WK == WK_F32I) return (double)__ldcs((const float *)w + e);
    else return __ldcs((const double *)w + e);
}

// ---- gain in the three precision modes -------------------------------------
template <int PREC>
struct Prec;
template <>
struct Prec<MG_PREC_FP64> {
    using G = double;
    // (k_ic - (e - k_i*(a - s_c)/(2m))) / m, each operation rounded as written;
    // both quotients are correctly rounded (div_by), so the value is the one a
    // divide instruction gives
    __device__ static __forceinline__ G gain(double kic, double e, double ki, double a, double sc,
                                             const GainK &K) {
        double t = __dmul_rn(ki, __dsub_rn(a, sc));
        t = div_by(t, K.two_m, K.r_two_m);
        t = __dsub_rn(e, t);
        return div_by(__dsub_rn(kic, t), K.m, K.r_m);
    }
};
template <>
struct Prec<MG_PREC_FP32> {
    using G = float;
    __device__ static __forceinline__ G gain(double kic, double e, double ki, double a, double sc,
                                             const GainK &K) {
        float t = __fmul_rn((float)ki, __fsub_rn((float)a, (float)sc));
        t = div_by(t, K.two_m_f, K.r_two_m_f);
        t = __fsub_rn((float)e, t);
        return div_by(__fsub_rn((float)kic, t), K.m_f, K.r_m_f);
    }
};
template <>
struct Prec<MG_PREC_INT64> {
    using G = long long;
    // 2m*m*gain = 2m*(k_ic - e) + k_i*(a - s_c), exact for integral weights
    __device__ static __forceinline__ G gain(double kic, double e, double ki, double a, double sc,
                                             const GainK &K) {
        return K.mass_i * ((long long)kic - (long long)e) + (long long)ki * ((long long)a - (long long)sc);
    }
};

template <class G>
__device__ __forceinline__ bool better(G g2, uint32_t c2, G g1, uint32_t c1, int up) {
    return g2 > g1 || (g2 == g1 && (up ? c2 < c1 : c2 > c1));
}

template <int VER>
__device__ __forceinline__ bool is_candidate(uint32_t c, uint32_t src, int up) {
    if constexpr (VER == 1) return up ? c < src : c > src;
    else return c != src;
}

template <int VER>
__device__ __forceinline__ uint32_t final_choice(uint32_t dst, uint32_t src, int up) {
    if constexpr (VER == 1) return dst;
    else return up ? (dst < src ? dst : src) : (dst > src ? dst : src);
}

template <class G>
__device__ __forceinline__ G shfl_xor_g(G v, int o) {
    return __shfl_xor_sync(0xffffffffu, v, o);
}

// Block-level accumulation of sum_in / distinct into the sweep accumulators.
__device__ __forceinline__ void flush_acc(SweepAcc *acc, int integral, double sin, unsigned dcnt) {
    __shared__ double s_f;
    __shared__ unsigned long long s_d;
    if (threadIdx.x == 0) {
        s_f = 0;
        s_d = 0;
    }
    __syncthreads();
    double v = warp_sum(sin);
    unsigned long long d = warp_sum((unsigned long long)dcnt);
    if ((threadIdx.x & 31) == 0) {
        if (v != 0) atomicAdd(&s_f, v);
        if (d) atomicAdd(&s_d, d);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        if (integral) {
            if (s_f != 0) atomicAdd(&acc->sin_u, (unsigned long long)s_f);
        } else if (s_f != 0) {
            atomicAdd(&acc->sin_f, s_f);
        }
        if (s_d) atomicAdd(&acc->distinct, s_d);
    }
}

// ============================================================================
// bins 0-4: T lanes per vertex, deg <= T
// ============================================================================
template <int T, int WK, int PREC, int VER, int BT>
__global__ void __launch_bounds__(256) lm_tile_kernel(LMArgs A, uint32_t bin_off, uint32_t bin_size) {
    using G = typename Prec<PREC>::G;
    const int up = load_up<BT>(A);
    __shared__ double wbuf[8][32];
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    const uint32_t gl = lane & (T - 1), gbase = lane & ~(uint32_t)(T - 1);
    const uint32_t gmask = T == 32 ? 0xffffffffu : (((1u << T) - 1u) << gbase);
    constexpr uint32_t GPW = 32 / T;
    double sin = 0;
    unsigned dcnt = 0;
    const uint32_t gwarp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nwarp = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t wb = gwarp * GPW; wb < bin_size; wb += nwarp * GPW) {
        const uint32_t idx = wb + lane / T;
        bool active = idx < bin_size;
        uint32_t i = 0, src = 0, lo = 0, hi = 0;
        double ki = 0, a = 0;
        VView vv;
        if (active) {
            i = A.perm[bin_off + idx];
            if constexpr (BT == 0) {
                const uint2 r = A.rows[bin_off + idx];
                lo = r.x;
                hi = r.y;
            }
            active = vview_at<BT>(A, bin_off + idx, vv);
        }
        if (active) {
            if constexpr (BT != 0) {
                lo = A.off[i];
                hi = A.off[i + 1];
            }
            src = vv.P[i];
        }
        const uint32_t e = lo + gl;
        const bool has = active && e < hi;
        uint32_t j = kEmpty, c = kEmpty;
        double w = 0;
        if (has) {
            j = __ldcs(A.col + e);
            w = wload<WK>(A.w, e);
            c = vv.P[j];
        }
        if (active) {
            ki = A.k[i];
            a = A.sigma[src] - ki;
        }
        const bool self = has && j == i;
        const bool inner = has && !self && c == src;
        const bool cand = has && c != src && is_candidate<VER>(c, src, up);
        const uint32_t key = cand ? c : kEmpty;
        const uint32_t peers = __match_any_sync(0xffffffffu, key) & gmask;
        const bool leader = cand && (uint32_t)(__ffs(peers) - 1) == lane;
        double kic, e_src, selfw;
        if constexpr (WK == WK_UNIT) {
            kic = u2d(__popc(peers));
            e_src = u2d(__popc(__ballot_sync(0xffffffffu, inner) & gmask));
            selfw = u2d(__popc(__ballot_sync(0xffffffffu, self) & gmask));
        } else {
            wbuf[warp][lane] = w;
            __syncwarp();
            kic = 0;
            if (leader) {
                uint32_t mset = peers;
                while (mset) {
                    int l = __ffs(mset) - 1;
                    kic += wbuf[warp][l];
                    mset &= mset - 1;
                }
            }
            __syncwarp();
            e_src = inner ? w : 0.0;
            selfw = self ? w : 0.0;
#pragma unroll
            for (int o = T / 2; o > 0; o >>= 1) {
                e_src += __shfl_xor_sync(0xffffffffu, e_src, o);
                selfw += __shfl_xor_sync(0xffffffffu, selfw, o);
            }
        }
        G best = G(0);
        uint32_t dst = src;
        if (leader) {
            G g = Prec<PREC>::gain(kic, e_src, ki, a, A.sigma[c], kref<BT>(A, vv));
            if (better(g, c, best, dst, up)) {
                best = g;
                dst = c;
            }
            dcnt++;
        }
#pragma unroll
        for (int o = T / 2; o > 0; o >>= 1) {
            G g2 = shfl_xor_g(best, o);
            uint32_t c2 = __shfl_xor_sync(0xffffffffu, dst, o);
            if (better(g2, c2, best, dst, up)) {
                best = g2;
                dst = c2;
            }
        }
        if (active && gl == 0) {
            vv.N[i] = final_choice<VER>(dst, src, up);
            put_sin<BT>(A, i, sin, e_src + selfw);
        }
    }
    flush_acc(A.acc, A.integral, sin, dcnt);
}

// ============================================================================
// classes up to 4096: GT threads per vertex, shared-memory table
// ============================================================================
// table value type: 32-bit integer sums for integral weights, else double
template <int WK>
struct ValT {
    using type = typename std::conditional<kIntg<WK>, uint32_t, double>::type;
};

template <int GT>
__device__ __forceinline__ void group_sync() {
    if constexpr (GT == 32) __syncwarp();
    else __syncthreads();
}

// argmax over a group of GT threads; the result is valid in the group's first
// thread (the only one its callers read it from)
template <int GT, class G>
__device__ __forceinline__ void group_argmax(G &best, uint32_t &dst, int up, G *rg, uint32_t *rc) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        G g2 = shfl_xor_g(best, o);
        uint32_t c2 = __shfl_xor_sync(0xffffffffu, dst, o);
        if (better(g2, c2, best, dst, up)) {
            best = g2;
            dst = c2;
        }
    }
    if constexpr (GT > 32) {
        // the group's warps are [w0, w0 + GT/32) of the block (several groups
        // may share a block)
        const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
        const int w0 = (threadIdx.x / GT) * (GT / 32);
        if (lane == 0) {
            rg[warp] = best;
            rc[warp] = dst;
        }
        __syncthreads();
        if (threadIdx.x % GT == 0) {
#pragma unroll 8
            for (int w2 = 1; w2 < GT / 32; w2++) {
                if (better(rg[w0 + w2], rc[w0 + w2], best, dst, up)) {
                    best = rg[w0 + w2];
                    dst = rc[w0 + w2];
                }
            }
        }
        __syncthreads();
    }
}

// table bits for a vertex of degree d: 2*d slots rounded up to a power of
// two, at least 32, at most the group's table (2^max_bits slots)
__device__ __forceinline__ int table_bits(uint32_t d, int max_bits) {
    const int want = d <= 16 ? 5 : 33 - __clz(2 * d - 1);
    return want < max_bits ? want : max_bits;
}

// weight of edge e as the table's value type: exact 32-bit integer for
// integral graphs (no float->int conversion instruction: the f64 value plus
// 2^52 carries the integer in its low mantissa word), double otherwise
template <int WK>
__device__ __forceinline__ typename ValT<WK>::type wget(const void *w, uint32_t e) {
    if constexpr (WK == WK_UNIT) return 1u;
    else if constexpr (WK == WK_U32) return __ldcs((const uint32_t *)w + e);
    else if constexpr (WK == WK_F64I)
        return (uint32_t)__double2loint(__dadd_rn(__ldcs((const double *)w + e), 4503599627370496.0));
    else if constexpr (WK == WK_F32I) return __float2uint_rn(__ldcs((const float *)w + e));
    else return wload<WK>(w, e);
}

// an edge weight (double) as a table value: exact 32-bit integer for integral
// weights (the f64 value plus 2^52 carries it in its low mantissa word)
template <class V>
__device__ __forceinline__ V wcast(double w) {
    if constexpr (std::is_same<V, uint32_t>::value) return (uint32_t)__double2loint(__dadd_rn(w, 4503599627370496.0));
    else return w;
}

template <class V>
__device__ __forceinline__ double v2d(V v) {
    if constexpr (std::is_same<V, uint32_t>::value) return u2d(v);
    else return v;
}

constexpr uint64_t kEmpty64 = 0xFFFFFFFF00000000ull;

// Shared-memory hash table of 2^slots_log2 slots per group of GT threads (a
// power of two >= 2 * the largest degree of the launch, load <= 1/2): a key
// array and a value array (32-bit integer sums for integral weights, doubles
// otherwise).  Newly inserted slots are appended to a per-table list, so the
// evaluation runs densely over the distinct candidates only (and resets
// exactly those slots).
template <int GT, int WK, int PREC, int VER, int BLOCK, int BT>
__global__ void __launch_bounds__(BLOCK, 1024 / BLOCK)
    lm_hash_kernel(LMArgs A, uint32_t bin_off, uint32_t bin_size, int slots_log2) {
    using G = typename Prec<PREC>::G;
    const int up = load_up<BT>(A);
    using V = typename ValT<WK>::type;
    constexpr int GPB = BLOCK / GT;
    constexpr int BATCH = 4;
    constexpr int EB = 4;
    const uint32_t S = 1u << slots_log2;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    // values V [S * GPB] | keys u32 [S * GPB] | used u16 [S/2 * GPB]
    V *vals_all = (V *)smem_raw;
    uint32_t *keys_all = (uint32_t *)(smem_raw + sizeof(V) * S * GPB);
    uint16_t *used_all = (uint16_t *)(smem_raw + (sizeof(V) + sizeof(uint32_t)) * S * GPB);
    // per-vertex sums and candidate counters, double-buffered by the parity
    // of the group's vertex: the next vertex starts before they are cleared
    __shared__ V acc_e[2][GPB], acc_s[2][GPB];
    __shared__ uint32_t cnt[2][GPB];
    __shared__ G red_g[32];
    __shared__ uint32_t red_c[32];
    const int g = threadIdx.x / GT, t = threadIdx.x % GT;
    V *vals = vals_all + g * S;
    uint32_t *keys = keys_all + g * S;
    uint16_t *used = used_all + g * (S / 2);
    for (uint32_t s2 = threadIdx.x; s2 < S * GPB; s2 += BLOCK) {
        keys_all[s2] = kEmpty;
        vals_all[s2] = V(0);
    }
    if (threadIdx.x < GPB) {
        for (int q = 0; q < 2; q++) {
            acc_e[q][threadIdx.x] = V(0);
            acc_s[q][threadIdx.x] = V(0);
            cnt[q][threadIdx.x] = 0;
        }
    }
    __syncthreads();
    double sin = 0;
    unsigned dcnt = 0;
    int par = 0;
    for (uint32_t idx = blockIdx.x * GPB + g; idx - g < bin_size; idx += gridDim.x * GPB, par ^= 1) {
        // the loop condition is uniform inside a group (GT == 32) or block (GT > 32)
        bool active = idx < bin_size;
        uint32_t i = 0, src = 0, lo = 0, hi = 0;
        double ki = 0, a = 0;
        VView vv;
        if (active) {
            i = A.perm[bin_off + idx];
            if constexpr (BT == 0) {
                const uint2 r = A.rows[bin_off + idx];
                lo = r.x;
                hi = r.y;
            }
            active = vview_at<BT>(A, bin_off + idx, vv);
        }
        if (active) {
            if constexpr (BT != 0) {
                lo = A.off[i];
                hi = A.off[i + 1];
            }
            src = vv.P[i];  // needed first by the edge pass's community tests
            ki = A.k[i];
        }
        const int tb = table_bits(hi - lo, slots_log2);
        const uint32_t mask = (1u << tb) - 1u;
        V e_part = V(0), s_part = V(0);
        // warp-uniform loop bound (lanes past the row's end take part with no
        // edge), so that the warp can append its new slots with one atomic
        const uint32_t lane = threadIdx.x & 31u;
        // add `val` to community `key`'s slot (kEmpty: nothing); called by
        // every lane of the warp at the same point, so that the warp's new
        // slots join the table's candidate list with one atomic
        auto insert = [&](uint32_t key, V val) {
            uint32_t hnew = kEmpty;  // slot this lane claimed for a new key
            if (key != kEmpty) {
                // one compare-and-swap per probe: claims an empty slot or
                // finds the key (load <= 1/2, so the loop ends long before S)
                uint32_t h = hash_slot(key, tb);
                for (uint32_t p = 0; p < S; p++) {
                    const uint32_t prev = atomicCAS(keys + h, kEmpty, key);
                    if (prev == kEmpty) {
                        hnew = h;
                        break;
                    }
                    if (prev == key) break;
                    h = (h + 1) & mask;
                }
                atomicAdd(vals + h, val);
            }
            const uint32_t m = __ballot_sync(0xffffffffu, hnew != kEmpty);
            if (m) {
                const uint32_t leader = __ffs(m) - 1;
                uint32_t pos = 0;
                if (lane == leader) pos = atomicAdd(&cnt[par][g], (uint32_t)__popc(m));
                pos = __shfl_sync(0xffffffffu, pos, leader);
                if (hnew != kEmpty) used[pos + __popc(m & ((1u << lane) - 1u))] = (uint16_t)hnew;
            }
        };
        // run combining (A.agg: sweeps where communities repeat): a lane adds
        // the weights of its consecutive edges into one community in a
        // register and inserts the sum when its community changes, so rows
        // whose neighbours sit in a few communities make few shared-memory
        // adds to the same slot
        uint32_t rk = kEmpty;
        V rs = V(0);
        for (uint32_t wbase = lo + (t & ~31u); wbase < hi; wbase += GT * BATCH) {
            const uint32_t base = wbase + lane;
            uint32_t jj[BATCH], cc[BATCH];
            V ww[BATCH];
            // rows shorter than the batch: whole sub-steps past the row's end
            // are skipped by the warp (uniform test)
#pragma unroll
            for (int b = 0; b < BATCH; b++) {
                uint32_t e = base + b * GT;
                jj[b] = e < hi ? __ldcs(A.col + e) : kEmpty;
                ww[b] = e < hi ? wget<WK>(A.w, e) : V(0);
            }
#pragma unroll
            for (int b = 0; b < BATCH; b++) cc[b] = jj[b] != kEmpty ? vv.P[jj[b]] : kEmpty;
#pragma unroll
            for (int b = 0; b < BATCH; b++) {
                if (wbase + b * GT >= hi) break;
                const uint32_t c = cc[b];
                const bool cand = jj[b] != kEmpty && c != src && is_candidate<VER>(c, src, up);
                if (A.agg) {  // uniform: a kernel argument
                    const bool same = cand && c == rk;
                    const uint32_t fk = cand && !same ? rk : kEmpty;
                    const V fv = rs;
                    if (cand) {
                        rs = same ? rs + ww[b] : ww[b];
                        rk = c;
                    }
                    insert(fk, fv);
                } else {
                    insert(cand ? c : kEmpty, ww[b]);
                }
                if (!cand && jj[b] != kEmpty && c == src) {
                    if (jj[b] != i) e_part += ww[b];
                    else s_part += ww[b];
                }
            }
        }
        if (A.agg) insert(rk, rs);  // every lane's last run
        // group totals of e and self weight, folded into the barrier that
        // publishes the table
        e_part = warp_sum(e_part);
        s_part = warp_sum(s_part);
        if ((threadIdx.x & 31) == 0) {
            if (e_part != V(0)) atomicAdd(&acc_e[par][g], e_part);
            if (s_part != V(0)) atomicAdd(&acc_s[par][g], s_part);
        }
        group_sync<GT>();
        // sigma of the vertex's own community: loaded here, beside the
        // candidates' sigma, so that the edge loads above need not wait for
        // the vertex's community id
        if (active) a = A.sigma[src] - ki;
        const double e_src = v2d(acc_e[par][g]), selfw = v2d(acc_s[par][g]);
        const uint32_t nd = cnt[par][g];
        G best = G(0);
        uint32_t dst = src;
        for (uint32_t ub = t & ~31u; ub < nd; ub += GT * EB) {  // warp-uniform
            const uint32_t u0 = ub + lane;
            uint32_t kk[EB];
            double sc[EB], kv[EB];
            // sub-steps wholly past the candidates are skipped by the warp
            // (uniform tests: few candidates is the common case once
            // communities form)
#pragma unroll
            for (int b = 0; b < EB; b++) {
                kk[b] = kEmpty;
                if (ub + b * GT >= nd) break;
                const uint32_t u = u0 + b * GT;
                if (u < nd) {
                    const uint32_t h = used[u];
                    kk[b] = keys[h];
                    kv[b] = v2d(vals[h]);
                    keys[h] = kEmpty;
                    vals[h] = V(0);
                }
            }
#pragma unroll
            for (int b = 0; b < EB; b++) {
                if (ub + b * GT >= nd) break;
                if (kk[b] != kEmpty) sc[b] = A.sigma[kk[b]];
            }
#pragma unroll
            for (int b = 0; b < EB; b++) {
                if (ub + b * GT >= nd) break;
                if (kk[b] != kEmpty) {
                    G gn = Prec<PREC>::gain(kv[b], e_src, ki, a, sc[b], kref<BT>(A, vv));
                    if (better(gn, kk[b], best, dst, up)) {
                        best = gn;
                        dst = kk[b];
                    }
                }
            }
        }
        // argmax over the group: warp shuffles, then (wider groups) the
        // warps' winners meet in shared memory behind one barrier and thread 0
        // of the group takes the best.  The table was cleaned during the
        // evaluation, before that barrier, so the next vertex may start.
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            G g2 = shfl_xor_g(best, o);
            uint32_t c2 = __shfl_xor_sync(0xffffffffu, dst, o);
            if (better(g2, c2, best, dst, up)) {
                best = g2;
                dst = c2;
            }
        }
        if constexpr (GT > 32) {
            const int warp = threadIdx.x >> 5;
            if ((threadIdx.x & 31) == 0) {
                red_g[warp] = best;
                red_c[warp] = dst;
            }
            __syncthreads();
            if (t == 0) {
#pragma unroll
                for (int w2 = 1; w2 < GT / 32; w2++) {
                    if (better(red_g[warp + w2], red_c[warp + w2], best, dst, up)) {
                        best = red_g[warp + w2];
                        dst = red_c[warp + w2];
                    }
                }
            }
        }
        if (t == 0) {
            if (active) {
                vv.N[i] = final_choice<VER>(dst, src, up);
                put_sin<BT>(A, i, sin, e_src + selfw);
                dcnt += nd;
            }
            // used again two vertices on, after at least one more barrier
            cnt[par][g] = 0;
            acc_e[par][g] = V(0);
            acc_s[par][g] = V(0);
        }
        if constexpr (GT == 32) __syncwarp();
    }
    flush_acc(A.acc, A.integral, sin, dcnt);
}

// ============================================================================
// classes 5-10: a warp works a batch of K vertices at once (K * D <= 256,
// D = 2^logd the class's largest degree), each vertex with its own table of
// 2D slots in the warp's slice of shared memory.  Batch position f = r * 256
// + p * 32 + lane (round r, step p) is edge f mod D of vertex f / D, so one
// step belongs to one vertex (D >= 32) and every lane has kWarpP edges -- and
// later kWarpP candidates -- in flight at once.  Warp-level synchronisation
// only: no block barrier, no table shared between warps.
// ============================================================================
constexpr int kWarpP = 8;                  // entries per lane per round
constexpr int kWarpF = 32 * kWarpP;        // batch entries per round
constexpr int kWarpThreads = 256;
constexpr int kWarpMaxLogD = 10;           // classes up to 10 (degree <= 1024)

// slots of a warp's slice for classes of largest degree 2^logd
__host__ __device__ constexpr uint32_t warp_slots(int logd) {
    return 2u * ((1u << logd) > (uint32_t)kWarpF ? (1u << logd) : (uint32_t)kWarpF);
}
// bytes of a warp's slice: values V | keys u32 | candidate lists u16 (half
// the slots) | counters u32[16] | internal and self weights V[8] each
template <int WK>
__host__ __device__ constexpr size_t warp_slice_bytes(int logd) {
    return ((size_t)warp_slots(logd) * (sizeof(typename ValT<WK>::type) + sizeof(uint32_t) + sizeof(uint16_t) / 2) +
            3 * 8 * 8 + 15) & ~(size_t)15;
}

template <int WK, int PREC, int VER, int BT>
__global__ void __launch_bounds__(kWarpThreads) lm_warp_kernel(LMArgs A, uint32_t bin_off, uint32_t bin_size,
                                                                int logd) {
    using G = typename Prec<PREC>::G;
    using V = typename ValT<WK>::type;
    const int up = load_up<BT>(A);
    const uint32_t D = 1u << logd;
    const uint32_t K = D >= (uint32_t)kWarpF ? 1u : (uint32_t)kWarpF / D;  // vertices per batch (<= 8)
    const uint32_t rounds = D >= (uint32_t)kWarpF ? D / kWarpF : 1u;
    const uint32_t TS = 2 * D;  // slots per vertex table
    const int tb = logd + 1;
    const uint32_t WS = K * TS;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    unsigned char *slice = smem_raw + warp * warp_slice_bytes<WK>(logd);
    V *vals = (V *)slice;
    uint32_t *keys = (uint32_t *)(slice + sizeof(V) * WS);
    uint16_t *used = (uint16_t *)(slice + (sizeof(V) + sizeof(uint32_t)) * WS);
    uint32_t *cnt = (uint32_t *)(slice + (sizeof(V) + sizeof(uint32_t) + sizeof(uint16_t) / 2) * WS);
    V *acc_e = (V *)(cnt + 16), *acc_s = acc_e + 8;
    for (uint32_t s = lane; s < WS; s += 32) {
        keys[s] = kEmpty;
        vals[s] = V(0);
    }
    if (lane < 8) {
        cnt[lane] = 0;
        acc_e[lane] = V(0);
        acc_s[lane] = V(0);
    }
    __syncwarp();
    double sin = 0;
    unsigned dcnt = 0;
    const uint32_t gwarp = blockIdx.x * (kWarpThreads / 32) + warp;
    const uint32_t nwarp = gridDim.x * (kWarpThreads / 32);
    for (uint32_t b0 = gwarp * K; b0 < bin_size; b0 += nwarp * K) {  // warp-uniform
        // lane k < K holds vertex k of the batch
        uint32_t i = 0, lo = 0, hi = 0, src = kEmpty;
        double ki = 0;
        bool act = false;
        VView vv;
        vv.P = A.P;
        vv.N = A.N;
        if (lane < K && b0 + lane < bin_size) {
            const uint32_t pos = bin_off + b0 + lane;
            i = A.perm[pos];
            if constexpr (BT == 0) {
                const uint2 r = A.rows[pos];
                lo = r.x;
                hi = r.y;
            }
            act = vview_at<BT>(A, pos, vv);
            if (act) {
                if constexpr (BT != 0) {
                    lo = A.off[i];
                    hi = A.off[i + 1];
                }
                src = vv.P[i];
                ki = A.k[i];
            } else {
                hi = lo;
            }
        }
        // ---- edge pass: neighbour communities into the vertices' tables ----
        V e_part = V(0), s_part = V(0);
        for (uint32_t r = 0; r < rounds; r++) {
            uint32_t jj[kWarpP], cc[kWarpP];
            V ww[kWarpP];
#pragma unroll
            for (int p = 0; p < kWarpP; p++) {
                const uint32_t f = r * kWarpF + p * 32 + lane;
                const uint32_t k = f >> logd;  // uniform over the step
                const uint32_t lk = __shfl_sync(0xffffffffu, lo, k), hk = __shfl_sync(0xffffffffu, hi, k);
                const uint32_t e = lk + (f & (D - 1));
                jj[p] = e < hk ? __ldcs(A.col + e) : kEmpty;
                ww[p] = e < hk ? wget<WK>(A.w, e) : V(0);
            }
#pragma unroll
            for (int p = 0; p < kWarpP; p++) {
                const uint32_t k = (r * kWarpF + p * 32) >> logd;
                const uint32_t *Pk;
                if constexpr (BT == 0) Pk = A.P;
                else Pk = (const uint32_t *)__shfl_sync(0xffffffffu, (unsigned long long)vv.P, k);
                cc[p] = jj[p] != kEmpty ? Pk[jj[p]] : kEmpty;
            }
#pragma unroll
            for (int p = 0; p < kWarpP; p++) {
                const uint32_t f0 = r * kWarpF + p * 32;
                const uint32_t k = f0 >> logd;
                const uint32_t sk = __shfl_sync(0xffffffffu, src, k);
                const uint32_t ik = __shfl_sync(0xffffffffu, i, k);
                const uint32_t c = cc[p];
                uint32_t hnew = kEmpty;
                if (jj[p] != kEmpty) {
                    if (c != sk) {
                        if (is_candidate<VER>(c, sk, up)) {
                            uint32_t *tk = keys + k * TS;
                            uint32_t h = hash_slot(c, tb);
                            for (uint32_t q = 0; q < TS; q++) {
                                const uint32_t cur = ((volatile uint32_t *)tk)[h];
                                if (cur == c) break;
                                if (cur == kEmpty) {
                                    const uint32_t prev = atomicCAS(tk + h, kEmpty, c);
                                    if (prev == kEmpty) {
                                        hnew = h;
                                        break;
                                    }
                                    if (prev == c) break;
                                }
                                h = (h + 1) & (TS - 1);
                            }
                            atomicAdd(vals + k * TS + h, ww[p]);
                        }
                    } else if (jj[p] != ik) {
                        e_part += ww[p];
                    } else {
                        s_part += ww[p];
                    }
                }
                // the step's new slots join vertex k's candidate list
                const uint32_t m = __ballot_sync(0xffffffffu, hnew != kEmpty);
                if (m) {
                    uint32_t pos = 0;
                    if (lane == 0) {
                        pos = cnt[k];
                        cnt[k] = pos + __popc(m);
                    }
                    pos = __shfl_sync(0xffffffffu, pos, 0);
                    if (hnew != kEmpty) used[k * D + pos + __popc(m & ((1u << lane) - 1u))] = (uint16_t)hnew;
                }
                // last step of vertex k: its internal and self weight
                if (((f0 + 32) & (D - 1)) == 0) {
                    const V te = warp_sum(e_part), ts = warp_sum(s_part);
                    if (lane == 0) {
                        acc_e[k] += te;
                        acc_s[k] += ts;
                    }
                    e_part = V(0);
                    s_part = V(0);
                }
            }
        }
        __syncwarp();
        // sigma of the vertex's own community, loaded after the edge pass
        const double a = act ? A.sigma[src] - ki : 0.0;
        // ---- candidate pass: score every distinct candidate, argmax per vertex ----
        G best = G(0);
        uint32_t dst = 0;
        for (uint32_t r = 0; r < rounds; r++) {
            uint32_t kk[kWarpP];
            double kv[kWarpP], sc[kWarpP];
#pragma unroll
            for (int p = 0; p < kWarpP; p++) {
                const uint32_t f = r * kWarpF + p * 32 + lane;
                const uint32_t k = f >> logd, u = f & (D - 1);
                kk[p] = kEmpty;
                if (u < cnt[k]) {
                    const uint32_t h = k * TS + used[k * D + u];
                    kk[p] = keys[h];
                    kv[p] = v2d(vals[h]);
                    keys[h] = kEmpty;
                    vals[h] = V(0);
                }
            }
#pragma unroll
            for (int p = 0; p < kWarpP; p++)
                if (kk[p] != kEmpty) sc[p] = A.sigma[kk[p]];
#pragma unroll
            for (int p = 0; p < kWarpP; p++) {
                const uint32_t f0 = r * kWarpF + p * 32;
                const uint32_t k = f0 >> logd;
                if ((f0 & (D - 1)) == 0) {  // first step of vertex k
                    best = G(0);
                    dst = __shfl_sync(0xffffffffu, src, k);
                }
                const double kik = __shfl_sync(0xffffffffu, ki, k);
                const double ak = __shfl_sync(0xffffffffu, a, k);
                if (kk[p] != kEmpty) {
                    const double ek = v2d(acc_e[k]);
                    GainK Kk;
                    if constexpr (BT == 0) Kk = A.K;
                    else Kk = A.gk[A.pgid[bin_off + b0 + k]];
                    const G gn = Prec<PREC>::gain(kv[p], ek, kik, ak, sc[p], Kk);
                    if (better(gn, kk[p], best, dst, up)) {
                        best = gn;
                        dst = kk[p];
                    }
                }
                if (((f0 + 32) & (D - 1)) == 0) {  // last step of vertex k: argmax, result
#pragma unroll
                    for (int o = 16; o > 0; o >>= 1) {
                        const G g2 = shfl_xor_g(best, o);
                        const uint32_t c2 = __shfl_xor_sync(0xffffffffu, dst, o);
                        if (better(g2, c2, best, dst, up)) {
                            best = g2;
                            dst = c2;
                        }
                    }
                    if (lane == k && act) {
                        vv.N[i] = final_choice<VER>(dst, src, up);
                        put_sin<BT>(A, i, sin, v2d(acc_e[k]) + v2d(acc_s[k]));
                        dcnt += cnt[k];
                    }
                }
            }
        }
        __syncwarp();
        if (lane < K) {
            cnt[lane] = 0;
            acc_e[lane] = V(0);
            acc_s[lane] = V(0);
        }
        __syncwarp();
    }
    flush_acc(A.acc, A.integral, sin, dcnt);
}

// ============================================================================
// classes 13-17: one vertex per thread-block cluster of CS CTAs, the
// cluster's shared memory holding one hash table of CS * kSegSlots<WK> slots.
// A neighbour community hashes to (owner CTA, slot); the owner's segment
// collects its sum (see the two fill modes below), each CTA evaluates the
// candidates of its segment, and rank 0 reduces the CS winners through
// distributed shared memory.  Two cluster barriers per
// vertex (accumulators double-buffered).  Slots are a 32-bit key and a sum:
// 32-bit integer for integral weights (shared-memory 32-bit adds; 64-bit
// packed slots were slower under contention), else double.
// ============================================================================
namespace cg = cooperative_groups;
constexpr int kClusterThreads = 1024;  // one CTA per SM with a 16K-slot segment
// CTA size of heavy tier t: tier 0 of an integral graph (degrees <= 8,192)
// runs 512-thread CTAs with half a dense segment, two per SM, so that one
// vertex's barriers and argmax overlap another's edge pass
template <int WK>
constexpr int tier_threads(int t) {
    return kDenseTier<WK>(t) && t == 0 ? kClusterThreads / 2 : kClusterThreads;
}

template <int CS>
__device__ __forceinline__ void cluster_barrier() {
    if constexpr (CS == 1) __syncthreads();
    else cg::this_cluster().sync();
}

template <int CS, class T>
__device__ __forceinline__ T *rank_ptr(T *p, unsigned r) {
    if constexpr (CS == 1) return p;
    else return cg::this_cluster().map_shared_rank(p, r);
}

template <int CS, int WK, int PREC, int VER, int BT, bool DENSE = false, int NT = kClusterThreads>
__global__ void __launch_bounds__(NT, kClusterThreads / NT) lm_cluster_kernel(LMArgs A, const uint32_t *verts,
                                                                        uint32_t count) {
    using G = typename Prec<PREC>::G;
    const int up = load_up<BT>(A);
    static_assert(!DENSE || kIntg<WK>, "dense segments hold 32-bit sums");
    constexpr int S = DENSE ? kDenseSlots / (kClusterThreads / NT) : kSegSlots<WK>;
    constexpr int BATCH = 4;
    constexpr int EB = 4;  // slots per thread per evaluation batch
    extern __shared__ __align__(16) unsigned char smem_raw[];
    // keys u32 [S] | sums [S] (u32 for integral weights, else double) | used u16 [S]
    // (DENSE: no insertion list; the evaluation scans the segment)
    using CV = typename ValT<WK>::type;
    uint32_t *keys = (uint32_t *)smem_raw;
    CV *vals = (CV *)(smem_raw + sizeof(uint32_t) * S);
    // slots of this CTA's segment that received a new key, in insertion order
    uint16_t *used = (uint16_t *)(smem_raw + (sizeof(uint32_t) + sizeof(CV)) * S);
    __shared__ uint32_t ucnt;
    __shared__ double acc_e[2], acc_s[2];
    __shared__ G best_g[2][CS];
    __shared__ uint32_t best_c[2][CS];
    __shared__ G red_g[32];
    __shared__ uint32_t red_c[32];
    unsigned rank = 0;
    if constexpr (CS > 1) rank = cg::this_cluster().block_rank();
    for (int s = threadIdx.x; s < S; s += NT) {
        keys[s] = kEmpty;
        vals[s] = CV(0);
    }
    if (threadIdx.x < 2) {
        acc_e[threadIdx.x] = 0;
        acc_s[threadIdx.x] = 0;
    }
    if (threadIdx.x == 0) ucnt = 0;
    cluster_barrier<CS>();
    const uint32_t cluster_id = blockIdx.x / CS, nclusters = gridDim.x / CS;
    double sin = 0;
    unsigned dcnt = 0;
    int par = 0;
    for (uint32_t vi = cluster_id; vi < count; vi += nclusters) {
        const uint32_t i = verts[vi];
        VView vv;
        // uniform over the cluster: every CTA works on the same vertex
        if (!vview<BT>(A, i, vv)) continue;
        const uint32_t lo = A.off[i], hi = A.off[i + 1], src = vv.P[i];
        const double ki = A.k[i];
        double e_part = 0, s_part = 0;
        // Two ways to fill the cluster's table (mg_sweep_options; own by default,
        // measured faster on R-MAT-24 at every level):
        //  * own fill: every CTA reads the whole row
        //    (it stays in cache) and inserts only the communities whose slots
        //    it owns, so all table atomics are local;
        //  * split fill (A.split): the CTAs split the row and the inserts go to
        //    the owner CTA, through distributed shared memory when it is
        //    another.
        const bool own = CS > 1 && !A.split;
        const uint32_t t0 = own ? threadIdx.x : rank * NT + threadIdx.x;
        const uint32_t step = own ? NT : CS * NT;
        // add `val` to community `key`'s slot in the segment of its owner CTA
        // (this CTA's own shared memory, or another's through DSMEM)
        auto ins = [&](uint32_t key, CV val) {
            const uint32_t h = hash_range(key, (uint32_t)CS * S);
            const unsigned owner = h / S;
            uint32_t s = h - owner * S;
            uint32_t *ks = owner == rank ? keys : rank_ptr<CS>(keys, owner);
            CV *vs = owner == rank ? vals : rank_ptr<CS>(vals, owner);
            uint16_t *useg = owner == rank ? used : rank_ptr<CS>(used, owner);
            uint32_t *uc = owner == rank ? &ucnt : rank_ptr<CS>(&ucnt, owner);
            bool placed = false;
            for (int p = 0; p < S; p++) {
                const uint32_t prev = atomicCAS(ks + s, kEmpty, key);
                if (prev == kEmpty) {
                    if constexpr (!DENSE) useg[atomicAdd(uc, 1u)] = (uint16_t)s;
                    placed = true;
                    break;
                }
                if (prev == key) {
                    placed = true;
                    break;
                }
                s = s + 1 == S ? 0 : s + 1;
            }
            if (placed) atomicAdd(vs + s, val);
            else atomicAdd(&A.acc->overflow, 1ull);
        };
        // run combining (A.agg: sweeps where communities repeat): a thread adds
        // the weights of its consecutive edges into one community and inserts
        // the sum when its community changes
        uint32_t rk = kEmpty;
        CV rs = CV(0);
        for (uint32_t wbase = lo + (t0 & ~31u); wbase < hi; wbase += step * BATCH) {
            const uint32_t base = wbase + (t0 & 31u);
            uint32_t jj[BATCH], cc[BATCH];
            double ww[BATCH];
#pragma unroll
            for (int b = 0; b < BATCH; b++) {
                uint32_t e = base + b * step;
                jj[b] = e < hi ? (own ? __ldg(A.col + e) : __ldcs(A.col + e)) : kEmpty;
                ww[b] = e < hi ? wload<WK>(A.w, e) : 0.0;
            }
#pragma unroll
            for (int b = 0; b < BATCH; b++) cc[b] = jj[b] != kEmpty ? vv.P[jj[b]] : kEmpty;
#pragma unroll
            for (int b = 0; b < BATCH; b++) {
                if (wbase + b * step >= hi) break;  // uniform over the warp
                const uint32_t c = cc[b];
                bool cand = jj[b] != kEmpty && c != src && is_candidate<VER>(c, src, up);
                if (cand && own) cand = hash_range(c, (uint32_t)CS * S) / S == rank;
                if ((!own || rank == 0) && jj[b] != kEmpty && c == src) {
                    if (jj[b] != i) e_part += ww[b];
                    else s_part += ww[b];
                }
                if (!cand) continue;
                const CV wv = wcast<CV>(ww[b]);
                if (A.agg) {  // uniform: a kernel argument
                    if (c == rk) {
                        rs += wv;
                    } else {
                        if (rk != kEmpty) ins(rk, rs);
                        rk = c;
                        rs = wv;
                    }
                } else {
                    ins(c, wv);
                }
            }
        }
        if (rk != kEmpty) ins(rk, rs);  // the thread's last run
        e_part = warp_sum(e_part);
        s_part = warp_sum(s_part);
        if ((threadIdx.x & 31) == 0) {
            if (e_part != 0) atomicAdd(rank_ptr<CS>(&acc_e[par], 0), e_part);
            if (s_part != 0) atomicAdd(rank_ptr<CS>(&acc_s[par], 0), s_part);
        }
        cluster_barrier<CS>();  // all inserts and partial sums are in
        const double a = A.sigma[src] - ki;  // loaded after the edge pass, beside the candidates' sigma
        const double e_src = *rank_ptr<CS>(&acc_e[par], 0);
        G best = G(0);
        uint32_t dst = src;
        const uint32_t nd = ucnt;
        if constexpr (DENSE) {
            // every slot of the segment, EB per thread per step (S is a
            // multiple of NT * EB); the non-empty ones are this
            // CTA's candidates, reset as they are read
            static_assert(S % (NT * EB) == 0, "whole evaluation steps");
            for (uint32_t sb = threadIdx.x; sb < (uint32_t)S; sb += NT * EB) {
                uint32_t kk[EB];
                double kv[EB], sc[EB];
#pragma unroll
                for (int b = 0; b < EB; b++) {
                    const uint32_t s = sb + b * NT;
                    kk[b] = keys[s];
                    if (kk[b] != kEmpty) {
                        kv[b] = v2d(vals[s]);
                        keys[s] = kEmpty;
                        vals[s] = CV(0);
                        dcnt++;
                    }
                }
#pragma unroll
                for (int b = 0; b < EB; b++)
                    if (kk[b] != kEmpty) sc[b] = A.sigma[kk[b]];
#pragma unroll
                for (int b = 0; b < EB; b++) {
                    if (kk[b] != kEmpty) {
                        G gn = Prec<PREC>::gain(kv[b], e_src, ki, a, sc[b], kref<BT>(A, vv));
                        if (better(gn, kk[b], best, dst, up)) {
                            best = gn;
                            dst = kk[b];
                        }
                    }
                }
            }
        }
        for (uint32_t ub = threadIdx.x & ~31u; !DENSE && ub < nd; ub += NT * EB) {  // warp-uniform
            const uint32_t u0 = ub + (threadIdx.x & 31u);
            uint32_t kk[EB];
            double kv[EB], sc[EB];
            // sub-steps wholly past the candidates are skipped (uniform tests)
#pragma unroll
            for (int b = 0; b < EB; b++) {
                kk[b] = kEmpty;
                if (ub + b * NT >= nd) break;
                const uint32_t u = u0 + b * NT;
                if (u < nd) {
                    const uint32_t s = used[u];
                    kk[b] = keys[s];
                    kv[b] = v2d(vals[s]);
                    keys[s] = kEmpty;
                    vals[s] = CV(0);
                }
            }
#pragma unroll
            for (int b = 0; b < EB; b++) {
                if (ub + b * NT >= nd) break;
                if (kk[b] != kEmpty) sc[b] = A.sigma[kk[b]];
            }
#pragma unroll
            for (int b = 0; b < EB; b++) {
                if (ub + b * NT >= nd) break;
                if (kk[b] != kEmpty) {
                    G gn = Prec<PREC>::gain(kv[b], e_src, ki, a, sc[b], kref<BT>(A, vv));
                    if (better(gn, kk[b], best, dst, up)) {
                        best = gn;
                        dst = kk[b];
                    }
                }
            }
        }
        group_argmax<NT, G>(best, dst, up, red_g, red_c);
        if (threadIdx.x == 0) {
            if constexpr (!DENSE) dcnt += nd;
            ucnt = 0;  // every thread of this CTA has read it (barriers in group_argmax)
            rank_ptr<CS>(&best_g[par][0], 0)[rank] = best;
            rank_ptr<CS>(&best_c[par][0], 0)[rank] = dst;
        }
        cluster_barrier<CS>();  // winners of every CTA are with rank 0
        if (rank == 0 && threadIdx.x == 0) {
            G bg = G(0);
            uint32_t bc = src;
            for (int r = 0; r < CS; r++)
                if (better(best_g[par][r], best_c[par][r], bg, bc, up)) {
                    bg = best_g[par][r];
                    bc = best_c[par][r];
                }
            vv.N[i] = final_choice<VER>(bc, src, up);
            put_sin<BT>(A, i, sin, e_src + acc_s[par]);
            acc_e[par] = 0;
            acc_s[par] = 0;
        }
        par ^= 1;
    }
    cluster_barrier<CS>();  // no CTA leaves while others may still touch its memory
    flush_acc(A.acc, A.integral, sin, dcnt);
}

// ============================================================================
// bin 9, last tier (giants): global tables, many CTAs per vertex
// ============================================================================
constexpr int kHeavyThreads = 256;
constexpr uint32_t kHeavyChunkE = 4096;  // edges per insert item
constexpr uint32_t kHeavyChunkS = 4096;  // slots per evaluate item

__device__ __forceinline__ uint32_t find_item(const uint32_t *item_off, uint32_t H, uint32_t q) {
    // last h with item_off[h] <= q
    uint32_t lo = 0, hi = H;
    while (hi - lo > 1) {
        uint32_t mid = (lo + hi) >> 1;
        if (item_off[mid] <= q) lo = mid;
        else hi = mid;
    }
    return lo;
}


template <int WK, int VER, int BT>
__global__ void __launch_bounds__(kHeavyThreads) heavy_insert_kernel(LMArgs A, const uint32_t *hv, uint32_t H,
                                                                      const uint32_t *ins_off,
                                                                      const uint64_t *toff,
                                                                      const uint32_t *tsize, uint32_t *tkeys,
                                                                      double *tvals, double *hacc) {
    constexpr int BATCH = 4;
    __shared__ double red[2][kHeavyThreads / 32];
    const uint32_t q = blockIdx.x;
    const uint32_t h = find_item(ins_off, H, q);
    const uint32_t v = hv[h];
    VView vv;
    if (!vview<BT>(A, v, vv)) return;  // uniform over the block
    const int up = load_up<BT>(A);
    const uint32_t chunk = q - ins_off[h];
    const uint32_t vlo = A.off[v], vhi = A.off[v + 1];
    const uint32_t lo = vlo + chunk * kHeavyChunkE;
    const uint32_t hi = min(vhi, lo + kHeavyChunkE);
    const uint32_t src = vv.P[v];
    const uint32_t ts = tsize[h];
    uint32_t *keys = tkeys + toff[h];
    double *vals = tvals + toff[h];
    double e_part = 0, s_part = 0;
    auto ins = [&](uint32_t key, double val) {
        uint32_t s = hash_range(key, ts);
        for (uint32_t p = 0; p < ts; p++) {
            const uint32_t prev = atomicCAS(keys + s, kEmpty, key);
            if (prev == kEmpty || prev == key) break;
            s = s + 1 == ts ? 0 : s + 1;
        }
        atomicAdd(vals + s, val);
    };
    // run combining (A.agg: sweeps where communities repeat), as in the
    // shared-memory tables: one global atomic per run of equal communities
    uint32_t rk = kEmpty;
    double rs = 0;
    for (uint32_t base = lo + threadIdx.x; base < hi; base += kHeavyThreads * BATCH) {
        uint32_t jj[BATCH], cc[BATCH];
        double ww[BATCH];
#pragma unroll
        for (int b = 0; b < BATCH; b++) {
            uint32_t e = base + b * kHeavyThreads;
            jj[b] = e < hi ? __ldcs(A.col + e) : kEmpty;
            ww[b] = e < hi ? wload<WK>(A.w, e) : 0.0;
        }
#pragma unroll
        for (int b = 0; b < BATCH; b++) cc[b] = jj[b] != kEmpty ? vv.P[jj[b]] : kEmpty;
#pragma unroll
        for (int b = 0; b < BATCH; b++) {
            if (jj[b] == kEmpty) continue;
            const uint32_t c = cc[b];
            if (c != src) {
                if (is_candidate<VER>(c, src, up)) {
                    if (A.agg) {
                        if (c == rk) {
                            rs += ww[b];
                        } else {
                            if (rk != kEmpty) ins(rk, rs);
                            rk = c;
                            rs = ww[b];
                        }
                    } else {
                        ins(c, ww[b]);
                    }
                }
            } else if (jj[b] != v) {
                e_part += ww[b];
            } else {
                s_part += ww[b];
            }
        }
    }
    if (rk != kEmpty) ins(rk, rs);
    e_part = warp_sum(e_part);
    s_part = warp_sum(s_part);
    if ((threadIdx.x & 31) == 0) {
        red[0][threadIdx.x >> 5] = e_part;
        red[1][threadIdx.x >> 5] = s_part;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0, b = 0;
        for (int w2 = 0; w2 < kHeavyThreads / 32; w2++) {
            a += red[0][w2];
            b += red[1][w2];
        }
        if (a != 0) atomicAdd(hacc + 2 * h, a);
        if (b != 0) atomicAdd(hacc + 2 * h + 1, b);
    }
}

// per evaluate item: packed winner {gain bits, id}
template <int PREC, int BT>
__global__ void __launch_bounds__(kHeavyThreads) heavy_eval_kernel(LMArgs A, const uint32_t *hv, uint32_t H,
                                                                    const uint32_t *eval_off,
                                                                    const uint64_t *toff, const uint32_t *tsize,
                                                                    uint32_t *tkeys, double *tvals,
                                                                    const double *hacc,
                                                                    unsigned long long *item_best) {
    using G = typename Prec<PREC>::G;
    __shared__ G rg[32];
    __shared__ uint32_t rc[32];
    __shared__ unsigned long long s_d;
    const uint32_t q = blockIdx.x;
    const uint32_t h = find_item(eval_off, H, q);
    const uint32_t v = hv[h];
    VView vv;
    if (!vview<BT>(A, v, vv)) return;  // uniform over the block
    const int up = load_up<BT>(A);
    const uint32_t part = q - eval_off[h];
    const uint32_t ts = tsize[h];
    const uint32_t lo = part * kHeavyChunkS, hi = min(ts, lo + kHeavyChunkS);
    uint32_t *keys = tkeys + toff[h];
    double *vals = tvals + toff[h];
    const uint32_t src = vv.P[v];
    const double ki = A.k[v];
    const double a = A.sigma[src] - ki;
    const double e_src = hacc[2 * h];
    if (threadIdx.x == 0) s_d = 0;
    G best = G(0);
    uint32_t dst = src;
    unsigned dcnt = 0;
    for (uint32_t s = lo + threadIdx.x; s < hi; s += kHeavyThreads) {
        uint32_t c = keys[s];
        if (c != kEmpty) {
            double kv = vals[s];
            keys[s] = kEmpty;
            vals[s] = 0.0;
            G gn = Prec<PREC>::gain(kv, e_src, ki, a, A.sigma[c], kref<BT>(A, vv));
            if (better(gn, c, best, dst, up)) {
                best = gn;
                dst = c;
            }
            dcnt++;
        }
    }
    group_argmax<kHeavyThreads, G>(best, dst, up, rg, rc);
    unsigned long long d = warp_sum((unsigned long long)dcnt);
    if ((threadIdx.x & 31) == 0 && d) atomicAdd(&s_d, d);
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long bits;
        if constexpr (sizeof(G) == 8) bits = *(unsigned long long *)&best;
        else bits = (unsigned long long)(*(uint32_t *)&best);
        item_best[2 * q] = bits;
        item_best[2 * q + 1] = dst;
        if (s_d) atomicAdd(&A.acc->distinct, s_d);
    }
}

template <int PREC, int VER, int BT>
__global__ void heavy_final_kernel(LMArgs A, const uint32_t *hv, uint32_t H, const uint32_t *eval_off,
                                   double *hacc, const unsigned long long *item_best) {
    using G = typename Prec<PREC>::G;
    const uint32_t h = blockIdx.x * blockDim.x + threadIdx.x;
    const int up = load_up<BT>(A);
    double sin = 0;
    VView vv;
    if (h < H && vview<BT>(A, hv[h], vv)) {
        const uint32_t v = hv[h];
        const uint32_t src = vv.P[v];
        G best = G(0);
        uint32_t dst = src;
        for (uint32_t q = eval_off[h]; q < eval_off[h + 1]; q++) {
            unsigned long long bits = item_best[2 * q];
            uint32_t c = (uint32_t)item_best[2 * q + 1];
            G g;
            if constexpr (sizeof(G) == 8) g = *(G *)&bits;
            else {
                uint32_t b32 = (uint32_t)bits;
                g = *(G *)&b32;
            }
            if (better(g, c, best, dst, up)) {
                best = g;
                dst = c;
            }
        }
        vv.N[v] = final_choice<VER>(dst, src, up);
        put_sin<BT>(A, v, sin, hacc[2 * h] + hacc[2 * h + 1]);
        hacc[2 * h] = 0;
        hacc[2 * h + 1] = 0;
    }
    flush_acc(A.acc, A.integral, sin, 0);
}

template <int CS, int WK, int PREC, int VER, int BT, bool DENSE, int NT = kClusterThreads>
size_t cluster_smem() {
    if constexpr (DENSE)
        return (size_t)(kDenseSlots / (kClusterThreads / NT)) * (sizeof(uint32_t) + sizeof(typename ValT<WK>::type));
    else return (size_t)kSegSlots<WK> * (sizeof(uint32_t) + sizeof(typename ValT<WK>::type) + sizeof(uint16_t));
}

template <int CS, int WK, int PREC, int VER, int BT, int NT = kClusterThreads>
cudaLaunchConfig_t cluster_config(size_t smem, unsigned grid, cudaStream_t s, cudaLaunchAttribute *attr) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid, 1, 1);
    cfg.blockDim = dim3(NT, 1, 1);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = CS;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cfg;
}

// Maximum co-resident clusters of a cluster kernel (0 when the shape cannot
// run) on the current device.  The first call per device also raises the
// kernel's shared-memory limit there (a per-device setting); the result is
// cached per device, under a lock, since serving workers launch concurrently.
template <int CS, int WK, int PREC, int VER, int BT, bool DENSE = false, int NT = kClusterThreads>
int cluster_capacity() {
    static std::mutex mu;
    static std::map<int, int> caps;  // device -> co-resident clusters
    int dev = 0;
    MG_CUDA(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lk(mu);
    const auto it = caps.find(dev);
    if (it != caps.end()) return it->second;
    auto kern = lm_cluster_kernel<CS, WK, PREC, VER, BT, DENSE, NT>;
    const size_t smem = cluster_smem<CS, WK, PREC, VER, BT, DENSE, NT>();
    MG_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    if (CS > 8) MG_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
    cudaLaunchAttribute attr[1];
    cudaLaunchConfig_t cfg = cluster_config<CS, WK, PREC, VER, BT, NT>(smem, CS * 148, nullptr, attr);
    int n = 0;
    if (cudaOccupancyMaxActiveClusters(&n, (void *)kern, &cfg) != cudaSuccess) {
        cudaGetLastError();
        n = 0;
    }
    caps[dev] = n;
    return n;
}

template <int CS, int WK, int PREC, int VER, int BT, bool DENSE, int NT = kClusterThreads>
void launch_cluster(const LMArgs &A, const uint32_t *verts, uint32_t count, cudaStream_t s) {
    auto kern = lm_cluster_kernel<CS, WK, PREC, VER, BT, DENSE, NT>;
    const size_t smem = cluster_smem<CS, WK, PREC, VER, BT, DENSE, NT>();
    int cap = cluster_capacity<CS, WK, PREC, VER, BT, DENSE, NT>();
    MG_CHECK(cap > 0, MG_ERR_UNSUPPORTED, "cluster shape cannot be scheduled on this device");
    unsigned clusters = (unsigned)std::min<uint64_t>(count, (uint64_t)cap);
    cudaLaunchAttribute attr[1];
    cudaLaunchConfig_t cfg = cluster_config<CS, WK, PREC, VER, BT, NT>(smem, clusters * CS, s, attr);
    MG_CUDA(cudaLaunchKernelEx(&cfg, kern, A, verts, count));
    MG_LAUNCH_CHECK();
}

// Bytes of dynamic shared memory of a hash launch with 2^slots_log2 slots per group.
template <int WK>
size_t hash_smem(int gpb, int slots_log2) {
    const size_t per_slot = sizeof(typename ValT<WK>::type) + sizeof(uint32_t) + 1;
    return ((size_t)1 << slots_log2) * (size_t)gpb * per_slot;
}

// The dynamic shared-memory limit of a kernel is a per-function setting, so it
// is raised once per device to the largest table the kernel is launched with
// (setting it per launch would race between threads launching different
// table sizes).
inline void raise_smem_limit(const void *kern, size_t smem) {
    static std::mutex mu;
    static std::set<std::pair<const void *, int>> done;  // (kernel, device)
    int dev = 0;
    MG_CUDA(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lk(mu);
    if (done.count({kern, dev})) return;
    MG_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    done.insert({kern, dev});
}

// Shared-memory carveout (percent of the SM's 228 KB) that holds `blocks`
// resident blocks of `smem` dynamic and `stat` static bytes each (plus the
// per-block reserve); the rest of the SM's 256 KB stays L1, which the sweep
// kernels' community and sigma gathers go through.  The hint pays when the
// sweep's two streams run kernels concurrently (a kernel running alone gets
// the same configuration with or without it).
inline unsigned carveout_pct(size_t smem, size_t stat, int blocks) {
    const size_t need = (size_t)blocks * (smem + stat + 1024);
    return (unsigned)std::min<size_t>(100, (need * 100 + 233471) / 233472 + 1);
}

// The carveout of a kernel launched with `block` threads and `smem` dynamic
// bytes: the smallest that keeps its full occupancy (occupancy calculator,
// which assumes the largest carveout), cached per device under a lock since
// serving workers launch concurrently.
inline unsigned launch_carveout(const void *kern, unsigned block, size_t smem) {
    static std::mutex mu;
    static std::map<std::tuple<const void *, unsigned, size_t, int>, unsigned> cache;
    int dev = 0;
    MG_CUDA(cudaGetDevice(&dev));
    const auto key = std::make_tuple(kern, block, smem, dev);
    std::lock_guard<std::mutex> lk(mu);
    auto it = cache.find(key);
    if (it != cache.end()) return it->second;
    int blocks = 0;
    MG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, kern, (int)block, smem));
    cudaFuncAttributes fa;
    MG_CUDA(cudaFuncGetAttributes(&fa, kern));
    const unsigned pct = blocks > 0 ? carveout_pct(smem, fa.sharedSizeBytes, blocks) : 100u;
    cache.emplace(key, pct);
    return pct;
}

// Launch of a single-graph sweep kernel with its carveout hint (batched sweeps
// launch plainly: they are captured into CUDA graphs).
template <int BT, class... P, class... Args>
void launch_l1(void (*kern)(P...), unsigned grid, unsigned block, size_t smem, cudaStream_t s, Args... args) {
    if constexpr (BT == 0) {
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(grid);
        cfg.blockDim = dim3(block);
        cfg.dynamicSmemBytes = smem;
        cfg.stream = s;
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributePreferredSharedMemoryCarveout;
        at[0].val.sharedMemCarveout = launch_carveout((const void *)kern, block, smem);
        cfg.attrs = at;
        cfg.numAttrs = 1;
        MG_CUDA(cudaLaunchKernelEx(&cfg, kern, args...));
    } else {
        kern<<<grid, block, smem, s>>>(args...);
    }
    MG_LAUNCH_CHECK();
}

// One light class (degrees <= 2^cls) with the given shape.
template <int WK, int PREC, int VER, int BT>
void launch_light(int shape, int cls, const LMArgs &A, uint32_t off, uint32_t size, cudaStream_t s) {
    if (size == 0) return;
    auto tile = [&](auto kern, int T) {
        const uint64_t per_block = 256 / T;
        const unsigned grid = (unsigned)std::min<uint64_t>(ceil_div(size, per_block), 148ull * 32);
        launch_l1<BT>(kern, grid, 256, 0, s, A, off, size);
    };
    auto hash = [&](auto kern, int gt, int block) {
        const int gpb = block / gt;
        const int sl = std::max(5, cls + 1);  // 2 * 2^cls slots, at least 32
        const size_t smem = hash_smem<WK>(gpb, sl);
        // the largest table of the shape: 2 * its capacity
        int max_sl = 5;
        while ((1u << max_sl) < 2 * shape_capacity(shape)) max_sl++;
        raise_smem_limit((const void *)kern, hash_smem<WK>(gpb, max_sl));
        const unsigned grid = (unsigned)std::min<uint64_t>(ceil_div(size, gpb), 148ull * 64);
        launch_l1<BT>(kern, grid, block, smem, s, A, off, size, sl);
    };
    auto warpk = [&](auto kern) {
        const int logd = std::max(5, cls);
        const size_t smem = (kWarpThreads / 32) * warp_slice_bytes<WK>(logd);
        raise_smem_limit((const void *)kern, (kWarpThreads / 32) * warp_slice_bytes<WK>(kWarpMaxLogD));
        const uint32_t K = (1u << logd) >= (uint32_t)kWarpF ? 1u : (uint32_t)kWarpF >> logd;
        const unsigned grid = (unsigned)std::min<uint64_t>(ceil_div(size, (kWarpThreads / 32) * K), 148ull * 8);
        launch_l1<BT>(kern, grid, kWarpThreads, smem, s, A, off, size, logd);
    };
    switch (shape) {
        case SH_T2: tile(lm_tile_kernel<2, WK, PREC, VER, BT>, 2); break;
        case SH_T4: tile(lm_tile_kernel<4, WK, PREC, VER, BT>, 4); break;
        case SH_T8: tile(lm_tile_kernel<8, WK, PREC, VER, BT>, 8); break;
        case SH_T16: tile(lm_tile_kernel<16, WK, PREC, VER, BT>, 16); break;
        case SH_T32: tile(lm_tile_kernel<32, WK, PREC, VER, BT>, 32); break;
        case SH_H32: hash(lm_hash_kernel<32, WK, PREC, VER, 256, BT>, 32, 256); break;
        case SH_H64: hash(lm_hash_kernel<64, WK, PREC, VER, 256, BT>, 64, 256); break;
        case SH_H128: hash(lm_hash_kernel<128, WK, PREC, VER, 128, BT>, 128, 128); break;
        case SH_H256: hash(lm_hash_kernel<256, WK, PREC, VER, 256, BT>, 256, 256); break;
        case SH_H512: hash(lm_hash_kernel<512, WK, PREC, VER, 512, BT>, 512, 512); break;
        case SH_W: warpk(lm_warp_kernel<WK, PREC, VER, BT>); break;
        default: throw Error(MG_ERR_INVALID, "unknown sweep shape");
    }
}

// ============================================================================
// the first sweep of a level (single graph): every community is one vertex
// (P = identity, sigma = k) and rows hold no repeated neighbour, so every
// neighbour j != i is a candidate community of its own with k_ic = w_ij and
// e = 0 -- no table.  The gain is the same FP64 expression with the same
// operands as the table kernels', so the result is bit-identical.  T lanes
// per vertex (T <= 32), or BLOCK threads per vertex for long rows.
// ============================================================================
constexpr int kFirstU = 4;  // edges in flight per thread

template <int T, int WK, int PREC, int VER>
__global__ void __launch_bounds__(256) lm_first_kernel(LMArgs A, uint32_t bin_off, uint32_t bin_size) {
    using G = typename Prec<PREC>::G;
    const int up = A.up;
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t gl = lane & (T - 1);
    constexpr uint32_t GPW = 32 / T;
    double sin = 0;
    unsigned dcnt = 0;
    const uint32_t gwarp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nwarp = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t wb = gwarp * GPW; wb < bin_size; wb += nwarp * GPW) {  // warp-uniform
        const uint32_t idx = wb + lane / T;
        const bool active = idx < bin_size;
        uint32_t i = 0, lo = 0, hi = 0;
        if (active) {
            i = A.perm[bin_off + idx];
            const uint2 r = A.rows[bin_off + idx];
            lo = r.x;
            hi = r.y;
        }
        const double ki = active ? A.k[i] : 0.0;
        const double a = active ? A.sigma[i] - ki : 0.0;
        G best = G(0);
        uint32_t dst = i;
        double selfw = 0;
        for (uint32_t e0 = lo + gl; e0 < hi; e0 += T * kFirstU) {
            uint32_t jj[kFirstU];
            double ww[kFirstU], sc[kFirstU];
#pragma unroll
            for (int u = 0; u < kFirstU; u++) {
                const uint32_t e = e0 + u * T;
                jj[u] = e < hi ? __ldcs(A.col + e) : kEmpty;
                ww[u] = e < hi ? wload<WK>(A.w, e) : 0.0;
            }
#pragma unroll
            for (int u = 0; u < kFirstU; u++) sc[u] = jj[u] != kEmpty && jj[u] != i ? A.sigma[jj[u]] : 0.0;
#pragma unroll
            for (int u = 0; u < kFirstU; u++) {
                const uint32_t j = jj[u];
                if (j == kEmpty) continue;
                if (j == i) {
                    selfw += ww[u];
                    continue;
                }
                if (!is_candidate<VER>(j, i, up)) continue;
                dcnt++;
                const G gn = Prec<PREC>::gain(ww[u], 0.0, ki, a, sc[u], A.K);
                if (better(gn, j, best, dst, up)) {
                    best = gn;
                    dst = j;
                }
            }
        }
#pragma unroll
        for (int o = T / 2; o > 0; o >>= 1) {
            const G g2 = shfl_xor_g(best, o);
            const uint32_t c2 = __shfl_xor_sync(0xffffffffu, dst, o);
            if (better(g2, c2, best, dst, up)) {
                best = g2;
                dst = c2;
            }
            selfw += __shfl_xor_sync(0xffffffffu, selfw, o);
        }
        if (active && gl == 0) {
            A.N[i] = final_choice<VER>(dst, i, up);
            sin += selfw;
        }
    }
    flush_acc(A.acc, A.integral, sin, dcnt);
}

template <int BLOCK, int WK, int PREC, int VER>
__global__ void __launch_bounds__(BLOCK) lm_first_block_kernel(LMArgs A, uint32_t bin_off, uint32_t bin_size) {
    using G = typename Prec<PREC>::G;
    const int up = A.up;
    __shared__ G red_g[BLOCK / 32];
    __shared__ uint32_t red_c[BLOCK / 32];
    __shared__ double red_s[BLOCK / 32];
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    double sin = 0;
    unsigned dcnt = 0;
    for (uint32_t idx = blockIdx.x; idx < bin_size; idx += gridDim.x) {  // uniform over the block
        const uint32_t i = A.perm[bin_off + idx];
        const uint2 r = A.rows[bin_off + idx];
        const uint32_t lo = r.x, hi = r.y;
        const double ki = A.k[i];
        const double a = A.sigma[i] - ki;
        G best = G(0);
        uint32_t dst = i;
        double selfw = 0;
        for (uint32_t e0 = lo + threadIdx.x; e0 < hi; e0 += BLOCK * kFirstU) {
            uint32_t jj[kFirstU];
            double ww[kFirstU], sc[kFirstU];
#pragma unroll
            for (int u = 0; u < kFirstU; u++) {
                const uint32_t e = e0 + u * BLOCK;
                jj[u] = e < hi ? __ldcs(A.col + e) : kEmpty;
                ww[u] = e < hi ? wload<WK>(A.w, e) : 0.0;
            }
#pragma unroll
            for (int u = 0; u < kFirstU; u++) sc[u] = jj[u] != kEmpty && jj[u] != i ? A.sigma[jj[u]] : 0.0;
#pragma unroll
            for (int u = 0; u < kFirstU; u++) {
                const uint32_t j = jj[u];
                if (j == kEmpty) continue;
                if (j == i) {
                    selfw += ww[u];
                    continue;
                }
                if (!is_candidate<VER>(j, i, up)) continue;
                dcnt++;
                const G gn = Prec<PREC>::gain(ww[u], 0.0, ki, a, sc[u], A.K);
                if (better(gn, j, best, dst, up)) {
                    best = gn;
                    dst = j;
                }
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const G g2 = shfl_xor_g(best, o);
            const uint32_t c2 = __shfl_xor_sync(0xffffffffu, dst, o);
            if (better(g2, c2, best, dst, up)) {
                best = g2;
                dst = c2;
            }
            selfw += __shfl_xor_sync(0xffffffffu, selfw, o);
        }
        if (lane == 0) {
            red_g[warp] = best;
            red_c[warp] = dst;
            red_s[warp] = selfw;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            double s = red_s[0];
            for (int w2 = 1; w2 < BLOCK / 32; w2++) {
                if (better(red_g[w2], red_c[w2], best, dst, up)) {
                    best = red_g[w2];
                    dst = red_c[w2];
                }
                s += red_s[w2];
            }
            A.N[i] = final_choice<VER>(dst, i, up);
            sin += s;
        }
        __syncthreads();  // red_* are reused by the next vertex
    }
    flush_acc(A.acc, A.integral, sin, dcnt);
}

template <int WK, int PREC, int VER>
void launch_first(int cls, const LMArgs &A, uint32_t off, uint32_t size, cudaStream_t s) {
    if (size == 0) return;
    auto lanes = [&](auto kern, int T) {
        const unsigned grid = (unsigned)std::min<uint64_t>(ceil_div(size, 256 / T), 148ull * 32);
        launch_l1<0>(kern, grid, 256, 0, s, A, off, size);
    };
    auto block = [&](auto kern, int bs) {
        const unsigned grid = (unsigned)std::min<uint64_t>(size, 148ull * (2048 / bs) * 4);
        launch_l1<0>(kern, grid, (unsigned)bs, 0, s, A, off, size);
    };
    if (cls <= 1) lanes(lm_first_kernel<2, WK, PREC, VER>, 2);
    else if (cls == 2) lanes(lm_first_kernel<4, WK, PREC, VER>, 4);
    else if (cls == 3) lanes(lm_first_kernel<8, WK, PREC, VER>, 8);
    else if (cls == 4) lanes(lm_first_kernel<16, WK, PREC, VER>, 16);
    else if (cls <= 9) lanes(lm_first_kernel<32, WK, PREC, VER>, 32);
    else if (cls < kFirstHeavyClass) block(lm_first_block_kernel<256, WK, PREC, VER>, 256);
    else block(lm_first_block_kernel<1024, WK, PREC, VER>, 1024);
}

template <int WK, int PREC, int VER, int BT>
void launch_sweep(const GraphView &g, const MoveLevel &lvl, MoveWorkspace &ws, const LMArgs &A, cudaStream_t s) {
    const Bins &B = lvl.bins;
    if constexpr (BT == 0) {
        if (A.first) {
            // the level's first sweep: no tables (every class, heavy ones included)
            MG_CUDA(cudaEventRecord(ws.ev_fork, s));
            const int ns = 1 + std::max(1, std::min(ws.light_streams, MoveWorkspace::kStreams - 1));
            for (int q = 0; q < ns; q++) MG_CUDA(cudaStreamWaitEvent(ws.streams[q], ws.ev_fork, 0));
            for (int c = kSweepClasses - 1; c >= 0; c--)
                launch_first<WK, PREC, VER>(c, A, B.offset[c], B.size[c], ws.streams[c % ns]);
            for (int q = 0; q < ns; q++) {
                MG_CUDA(cudaEventRecord(ws.ev_join[q], ws.streams[q]));
                MG_CUDA(cudaStreamWaitEvent(s, ws.ev_join[q], 0));
            }
            return;
        }
    }
    // fork: heavy path on its own stream, the light classes on two others
    MG_CUDA(cudaEventRecord(ws.ev_fork, s));
    const int ns = 1 + std::max(1, std::min(ws.light_streams, MoveWorkspace::kStreams - 1));
    for (int q = 0; q < ns; q++) MG_CUDA(cudaStreamWaitEvent(ws.streams[q], ws.ev_fork, 0));
    cudaStream_t sh = ws.streams[0], sm = ws.streams[1];
    const uint32_t *hl = lvl.heavy_list;
    // heavy tiers, largest clusters first
    if (lvl.tier_off[5] > lvl.tier_off[4])
        launch_cluster<tier_ctas<WK>(4), WK, PREC, VER, BT, kDenseTier<WK>(4)>(A, hl + lvl.tier_off[4], lvl.tier_off[5] - lvl.tier_off[4],
                                                             sh);
    if (lvl.tier_off[4] > lvl.tier_off[3])
        launch_cluster<tier_ctas<WK>(3), WK, PREC, VER, BT, kDenseTier<WK>(3)>(A, hl + lvl.tier_off[3], lvl.tier_off[4] - lvl.tier_off[3],
                                                             sh);
    if (lvl.tier_off[3] > lvl.tier_off[2])
        launch_cluster<tier_ctas<WK>(2), WK, PREC, VER, BT, kDenseTier<WK>(2)>(A, hl + lvl.tier_off[2], lvl.tier_off[3] - lvl.tier_off[2],
                                                             sh);
    if (lvl.tier_off[2] > lvl.tier_off[1])
        launch_cluster<tier_ctas<WK>(1), WK, PREC, VER, BT, kDenseTier<WK>(1)>(A, hl + lvl.tier_off[1], lvl.tier_off[2] - lvl.tier_off[1],
                                                             sh);
    if (lvl.tier_off[1] > lvl.tier_off[0])
        launch_cluster<tier_ctas<WK>(0), WK, PREC, VER, BT, kDenseTier<WK>(0), tier_threads<WK>(0)>(A, hl + lvl.tier_off[0], lvl.tier_off[1] - lvl.tier_off[0],
                                                             sm);
    if (lvl.giants > 0) {
        const uint32_t H = lvl.giants;
        const uint32_t *hv = hl + lvl.tier_off[kTiers - 1];
        launch_l1<BT>(heavy_insert_kernel<WK, VER, BT>, lvl.ins_items, kHeavyThreads, 0, sh, A, hv, H,
                      ws.h_ins.get(), ws.h_toff.get(), ws.h_tsize.get(), ws.h_keys.get(), ws.h_vals.get(),
                      ws.h_acc.get());
        launch_l1<BT>(heavy_eval_kernel<PREC, BT>, lvl.eval_items, kHeavyThreads, 0, sh, A, hv, H,
                      ws.h_eval.get(), ws.h_toff.get(), ws.h_tsize.get(), ws.h_keys.get(), ws.h_vals.get(),
                      ws.h_acc.get(), ws.h_best.get());
        heavy_final_kernel<PREC, VER, BT><<<(unsigned)ceil_div(H, 256), 256, 0, sh>>>(A, hv, H, ws.h_eval.get(),
                                                                                  ws.h_acc.get(), ws.h_best.get());
        MG_LAUNCH_CHECK();
    }
    // light classes, heaviest first, spread over the light streams
    for (int c = kLightClasses - 1; c >= 0; c--) {
        const int sh_c = lvl.shape[c];
        launch_light<WK, PREC, VER, BT>(sh_c, c, A, B.offset[c], B.size[c], ws.streams[1 + c % (ns - 1)]);
    }
    for (int q = 0; q < ns; q++) {
        MG_CUDA(cudaEventRecord(ws.ev_join[q], ws.streams[q]));
        MG_CUDA(cudaStreamWaitEvent(s, ws.ev_join[q], 0));
    }
}

// The kernel weight kind a sweep of g uses (integral graphs: integer slots).
inline int sweep_wk(const GraphView &g, const SweepParams &p) {
    return p.integral ? (g.wk == WK_F32 ? (int)WK_F32I : g.wk == WK_F64 ? (int)WK_F64I : g.wk) : g.wk;
}

// Weight kind / precision / version dispatch: f.run<WK, PREC, VER>().
template <class F>
void dispatch_kind(const GraphView &g, const SweepParams &p, F &f) {
    MG_CHECK(p.version == 1 || p.version == 2, MG_ERR_INVALID, "version must be 0, 1 or 2");
    const int wk = sweep_wk(g, p);
#define MG_SWEEP_CASE(WKV, PRECV)                                                                  \
    if (wk == WKV && p.precision == PRECV) {                                                       \
        if (p.version == 1) f.template run<WKV, PRECV, 1>();                                       \
        else f.template run<WKV, PRECV, 2>();                                                      \
        return;                                                                                    \
    }
    MG_SWEEP_CASE(WK_UNIT, MG_PREC_FP64)
    MG_SWEEP_CASE(WK_F32I, MG_PREC_FP64)
    MG_SWEEP_CASE(WK_F64I, MG_PREC_FP64)
    MG_SWEEP_CASE(WK_U32, MG_PREC_FP64)
    MG_SWEEP_CASE(WK_F32, MG_PREC_FP64)
    MG_SWEEP_CASE(WK_F64, MG_PREC_FP64)
    MG_SWEEP_CASE(WK_UNIT, MG_PREC_INT64)
    MG_SWEEP_CASE(WK_F32I, MG_PREC_INT64)
    MG_SWEEP_CASE(WK_F64I, MG_PREC_INT64)
    MG_SWEEP_CASE(WK_U32, MG_PREC_INT64)
    MG_SWEEP_CASE(WK_UNIT, MG_PREC_FP32)
    MG_SWEEP_CASE(WK_F32I, MG_PREC_FP32)
    MG_SWEEP_CASE(WK_F64I, MG_PREC_FP32)
    MG_SWEEP_CASE(WK_U32, MG_PREC_FP32)
    MG_SWEEP_CASE(WK_F32, MG_PREC_FP32)
    MG_SWEEP_CASE(WK_F64, MG_PREC_FP32)
#undef MG_SWEEP_CASE
    throw Error(MG_ERR_INVALID, "unknown weight kind or precision");
}

template <int BT>
struct SweepF {
    const GraphView &g;
    const MoveLevel &lvl;
    MoveWorkspace &ws;
    const LMArgs &A;
    cudaStream_t s;
    template <int WK, int PREC, int VER>
    void run() {
        launch_sweep<WK, PREC, VER, BT>(g, lvl, ws, A, s);
    }
};

template <int BT>
struct LightF {
    int shape, cls;
    const LMArgs &A;
    uint32_t off, size;
    cudaStream_t s;
    template <int WK, int PREC, int VER>
    void run() {
        launch_light<WK, PREC, VER, BT>(shape, cls, A, off, size, s);
    }
};

// A full sweep.
template <int BT>
void dispatch_sweep(const GraphView &g, const MoveLevel &lvl, MoveWorkspace &ws, const SweepParams &p,
                    const LMArgs &A, cudaStream_t s) {
    SweepF<BT> f{g, lvl, ws, A, s};
    dispatch_kind(g, p, f);
}

// One light class alone on stream s (the autotuner's timing runs).
template <int BT>
void dispatch_light(const GraphView &g, const SweepParams &p, const LMArgs &A, int shape, int cls, uint32_t off,
                    uint32_t size, cudaStream_t s) {
    LightF<BT> f{shape, cls, A, off, size, s};
    dispatch_kind(g, p, f);
}

// Candidate shapes of light class cls (degrees <= 2^cls): shapes whose table
// holds the class, from the thinnest that fits to a few wider ones.
inline std::vector<int> tune_candidates(int cls) {
    const uint32_t maxdeg = 1u << cls;
    std::vector<int> out;
    if (cls <= 5) {
        const int t0 = cls <= 1 ? SH_T2 : SH_T2 + (cls - 1);
        out.push_back(t0);
        if (t0 < SH_T32) out.push_back(t0 + 1);
        out.push_back(SH_H32);
        if (cls == 5) out.push_back(SH_W);
        return out;
    }
    if (shape_capacity(SH_W) >= maxdeg) out.push_back(SH_W);
    for (int sh = SH_H32; sh <= SH_H512; sh++) {
        if (shape_capacity(sh) < maxdeg) continue;
        // wider groups than twice the degree leave most threads idle
        const uint32_t gt = 32u << (sh - SH_H32);
        if (gt > 2 * maxdeg && sh > SH_H32) continue;
        out.push_back(sh);
        if (out.size() == 4) break;
    }
    return out;
}

// Fill lvl.shape from the table; time the candidates of classes missing from
// it (MG_TUNE_ON).  A timing run is a normal launch of that class: it writes
// the same new assignment the sweep will write; its sums go to ws.tune_acc.
template <int BT>
void tune_light(const GraphView &g, MoveLevel &lvl, MoveWorkspace &ws, const SweepParams &p, LMArgs A,
                cudaStream_t s, bool timing = true) {
    for (int c = 0; c < kLightClasses; c++) lvl.shape[c] = (uint8_t)default_shape(c);
    TuneTable &T = ws.tune;
    if (T.mode == MG_TUNE_OFF) return;
    A.acc = ws.tune_acc.ensure(1);
    const int wk = sweep_wk(g, p);
    cudaEvent_t e0 = ws.ev_tune[0], e1 = ws.ev_tune[1];
    for (int c = 0; c < kLightClasses; c++) {
        const uint32_t size = lvl.bins.size[c];
        if (size < kTuneMinVertices) continue;
        const uint32_t key = TuneTable::key(wk, p.precision, p.version, BT, c, size);
        auto it = T.entries.find(key);
        if (it != T.entries.end()) {
            lvl.shape[c] = it->second.shape;
            continue;
        }
        if (T.mode != MG_TUNE_ON || !timing) continue;
        float best = 1e30f;
        int best_sh = default_shape(c);
        for (int sh : tune_candidates(c)) {
            float ms = 0;
            for (int rep = 0; rep < 2; rep++) {  // the first run also loads the kernel
                MG_CUDA(cudaEventRecord(e0, s));
                dispatch_light<BT>(g, p, A, sh, c, lvl.bins.offset[c], size, s);
                MG_CUDA(cudaEventRecord(e1, s));
                MG_CUDA(cudaEventSynchronize(e1));
                MG_CUDA(cudaEventElapsedTime(&ms, e0, e1));
            }
            if (T.log) fprintf(stderr, "tune: wk %d prec %d ver %d batched %d class %d size %u shape %s %.1f us\n", wk,
                               p.precision, p.version, BT, c, size, shape_name(sh), ms * 1000.0);
            if (ms < best) {
                best = ms;
                best_sh = sh;
            }
        }
        T.entries[key] = TuneEntry{(uint8_t)best_sh, best * 1000.0f};
        T.tuned++;
        lvl.shape[c] = (uint8_t)best_sh;
    }
}

}  // namespace lmk
}  // namespace mg
