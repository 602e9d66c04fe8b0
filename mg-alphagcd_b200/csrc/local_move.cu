// local_move.cu -- one Louvain local-move sweep on sm_100a.
//
// Semantics (identical arithmetic to the reference kernels
// calculate_eicj_and_move_vertex_sh_tile / _sh_bk / _gl_bk,
// src/louvain/louvain.cu:404-1030, and the version-1 variants in
// src/louvain/louvain_gl.cu:504,578):
//   for vertex i with src = P[i], a = sigma[src] - k_i:
//     every edge (i,j,w), c = P[j]:  c != src -> k_ic += w ;  c == src, j != i -> e += w
//     gain_c = (k_ic - (e - k_i*(a - sigma[c])/(2m))) / m      (m = mass/2)
//     best starts at (0, src); a candidate wins on a larger gain, or on an
//     equal gain with a smaller id (up sweep) / larger id (down sweep);
//     version 2 clamps the result to min/max(dst, src); version 1 only lets
//     communities below (up) / above (down) src compete.
// The comparison is a total order, so the winner does not depend on the order
// in which candidates are visited.
//
// Kernel shapes (bins from the reference's 10-bin scheme, src/bin/BIN.cu:72-92):
//   bins 0-4 (deg <= 2..32): T-lane tiles, one edge per lane; neighbours in the
//     same community are merged with __match_any_sync, sums over the matching
//     lanes, a T-wide shuffle argmax.  No hash table at all.
//   bins 5-8 (deg <= 128..4094): one warp / CTA per vertex with a shared-memory
//     open-addressing table of >= 2*deg slots (load <= 1/2), self-cleaning.
//   bin 9 (deg > 4094): load-balanced over many CTAs per vertex; global
//     tables of 2*deg slots (resident in L2 while a vertex is being worked on),
//     insert items (vertex, 4096-edge chunk), evaluate items (vertex, slot
//     chunk) and a per-vertex reduction of the chunk winners.
// Each sweep also accumulates sum_in(P) = sum of weights of edges inside a
// community of P (self-loops included), the first term of the modularity of P
// (src/louvain/louvain.cu:105-238), so a separate modularity pass over the
// edges is not needed.
#include <cooperative_groups.h>

#include <algorithm>
#include <vector>

#include "engine.cuh"

namespace mg {

namespace {

struct LMArgs {
    const uint32_t *__restrict__ off;
    const uint32_t *__restrict__ col;
    const void *__restrict__ w;
    const uint32_t *__restrict__ P;
    uint32_t *__restrict__ N;
    const double *__restrict__ k;
    const double *__restrict__ sigma;
    const uint32_t *__restrict__ perm;
    double m;            // mass / 2
    double two_m;        // mass
    double r_m, r_two_m; // RN(1/m), RN(1/(2m))
    float m_f, two_m_f, r_m_f, r_two_m_f;
    long long mass_i;    // mass (integral graphs)
    int up;
    int integral;
    SweepAcc *acc;
};

template <int WK>
__device__ __forceinline__ double wload(const void *w, uint32_t e) {
    if constexpr (WK == WK_UNIT) return 1.0;
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
                                             const LMArgs &A) {
        double t = __dmul_rn(ki, __dsub_rn(a, sc));
        t = div_by(t, A.two_m, A.r_two_m);
        t = __dsub_rn(e, t);
        return div_by(__dsub_rn(kic, t), A.m, A.r_m);
    }
};
template <>
struct Prec<MG_PREC_FP32> {
    using G = float;
    __device__ static __forceinline__ G gain(double kic, double e, double ki, double a, double sc,
                                             const LMArgs &A) {
        float t = __fmul_rn((float)ki, __fsub_rn((float)a, (float)sc));
        t = div_by(t, A.two_m_f, A.r_two_m_f);
        t = __fsub_rn((float)e, t);
        return div_by(__fsub_rn((float)kic, t), A.m_f, A.r_m_f);
    }
};
template <>
struct Prec<MG_PREC_INT64> {
    using G = long long;
    // 2m*m*gain = 2m*(k_ic - e) + k_i*(a - s_c), exact for integral weights
    __device__ static __forceinline__ G gain(double kic, double e, double ki, double a, double sc,
                                             const LMArgs &A) {
        return A.mass_i * ((long long)kic - (long long)e) + (long long)ki * ((long long)a - (long long)sc);
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
template <int T, int WK, int PREC, int VER>
__global__ void __launch_bounds__(256) lm_tile_kernel(LMArgs A, uint32_t bin_off, uint32_t bin_size) {
    using G = typename Prec<PREC>::G;
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
        const bool active = idx < bin_size;
        uint32_t i = 0, src = 0, lo = 0, hi = 0;
        double ki = 0, a = 0;
        if (active) {
            i = A.perm[bin_off + idx];
            lo = A.off[i];
            hi = A.off[i + 1];
            src = A.P[i];
        }
        const uint32_t e = lo + gl;
        const bool has = active && e < hi;
        uint32_t j = kEmpty, c = kEmpty;
        double w = 0;
        if (has) {
            j = __ldcs(A.col + e);
            w = wload<WK>(A.w, e);
            c = A.P[j];
        }
        if (active) {
            ki = A.k[i];
            a = A.sigma[src] - ki;
        }
        const bool self = has && j == i;
        const bool inner = has && !self && c == src;
        const bool cand = has && c != src && is_candidate<VER>(c, src, A.up);
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
            G g = Prec<PREC>::gain(kic, e_src, ki, a, A.sigma[c], A);
            if (better(g, c, best, dst, A.up)) {
                best = g;
                dst = c;
            }
            dcnt++;
        }
#pragma unroll
        for (int o = T / 2; o > 0; o >>= 1) {
            G g2 = shfl_xor_g(best, o);
            uint32_t c2 = __shfl_xor_sync(0xffffffffu, dst, o);
            if (better(g2, c2, best, dst, A.up)) {
                best = g2;
                dst = c2;
            }
        }
        if (active && gl == 0) {
            A.N[i] = final_choice<VER>(dst, src, A.up);
            sin += e_src + selfw;
        }
    }
    flush_acc(A.acc, A.integral, sin, dcnt);
}

// ============================================================================
// bins 5-8: GT threads per vertex, SLOTS-entry shared table
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

// Two sums over a group of GT threads with one pair of barriers; results
// valid in every thread.  red: 2 * 32 doubles.
template <int GT>
__device__ __forceinline__ void group_sum2(double &a, double &b, double *red) {
    a = warp_sum(a);
    b = warp_sum(b);
    if constexpr (GT > 32) {
        const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
        if (lane == 0) {
            red[warp] = a;
            red[32 + warp] = b;
        }
        __syncthreads();
        double ta = 0, tb = 0;
#pragma unroll
        for (int w2 = 0; w2 < GT / 32; w2++) {
            ta += red[w2];
            tb += red[32 + w2];
        }
        __syncthreads();
        a = ta;
        b = tb;
    }
}

// Sum over a group of GT threads; result valid in every thread.
template <int GT>
__device__ __forceinline__ double group_sum(double v, double *red) {
    v = warp_sum(v);
    if constexpr (GT == 32) {
        return v;
    } else {
        const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
        if (lane == 0) red[warp] = v;
        __syncthreads();
        double t = 0;
#pragma unroll
        for (int w2 = 0; w2 < GT / 32; w2++) t += red[w2];
        __syncthreads();
        return t;
    }
}

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
        const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
        if (lane == 0) {
            rg[warp] = best;
            rc[warp] = dst;
        }
        __syncthreads();
#pragma unroll
        for (int w2 = 0; w2 < GT / 32; w2++) {
            if (better(rg[w2], rc[w2], best, dst, up)) {
                best = rg[w2];
                dst = rc[w2];
            }
        }
        __syncthreads();
    }
}

template <int X>
struct Log2 {
    static constexpr int value = 1 + Log2<X / 2>::value;
};
template <>
struct Log2<1> {
    static constexpr int value = 0;
};

template <int SLOTS>
__device__ __forceinline__ uint32_t table_find_or_insert(uint32_t *keys, uint32_t c, int bits) {
    const uint32_t mask = (1u << bits) - 1u;
    uint32_t h = hash_slot(c, bits);
    for (int p = 0; p < SLOTS; p++) {
        uint32_t cur = ((volatile uint32_t *)keys)[h];
        if (cur == c) return h;
        if (cur == kEmpty) {
            uint32_t prev = atomicCAS(keys + h, kEmpty, c);
            if (prev == kEmpty || prev == c) return h;
        }
        h = (h + 1) & mask;
    }
    return kEmpty;  // unreachable: tables hold >= 2*deg slots
}

// table bits for a vertex of degree d: 2*d slots rounded up to a power of
// two, at least 32, at most the group's table
template <int SLOTS>
__device__ __forceinline__ int table_bits(uint32_t d) {
    const int want = d <= 16 ? 5 : 33 - __clz(2 * d - 1);
    return want < Log2<SLOTS>::value ? want : Log2<SLOTS>::value;
}

// weight of edge e as the table's value type: exact 32-bit integer for
// integral graphs (no float->int conversion instruction: the f64 value plus
// 2^52 carries the integer in its low mantissa word), double otherwise
template <int WK>
__device__ __forceinline__ typename ValT<WK>::type wget(const void *w, uint32_t e) {
    if constexpr (WK == WK_UNIT) return 1u;
    else if constexpr (WK == WK_F64I)
        return (uint32_t)__double2loint(__dadd_rn(__ldcs((const double *)w + e), 4503599627370496.0));
    else if constexpr (WK == WK_F32I) return __float2uint_rn(__ldcs((const float *)w + e));
    else return wload<WK>(w, e);
}

template <class V>
__device__ __forceinline__ double v2d(V v) {
    if constexpr (std::is_same<V, uint32_t>::value) return u2d(v);
    else return v;
}

// Shared-memory hash table per group of GT threads.  Newly inserted slots are
// appended to a per-table list, so the evaluation runs densely over the
// distinct candidates only (and resets exactly those slots).
template <int GT, int SLOTS, int WK, int PREC, int VER, int BLOCK>
__global__ void __launch_bounds__(BLOCK, 1024 / BLOCK) lm_hash_kernel(LMArgs A, uint32_t bin_off, uint32_t bin_size) {
    using G = typename Prec<PREC>::G;
    using V = typename ValT<WK>::type;
    constexpr int GPB = BLOCK / GT;
    constexpr int BATCH = 4;
    constexpr int EB = 4;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    uint32_t *keys_all = (uint32_t *)smem_raw;
    V *vals_all = (V *)(smem_raw + sizeof(uint32_t) * SLOTS * GPB);
    uint16_t *used_all = (uint16_t *)(smem_raw + (sizeof(uint32_t) + sizeof(V)) * SLOTS * GPB);
    __shared__ V acc_e[GPB], acc_s[GPB];
    __shared__ uint32_t cnt[GPB];
    __shared__ G red_g[32];
    __shared__ uint32_t red_c[32];
    const int g = threadIdx.x / GT, t = threadIdx.x % GT;
    uint32_t *keys = keys_all + g * SLOTS;
    V *vals = vals_all + g * SLOTS;
    uint16_t *used = used_all + g * (SLOTS / 2);
    for (int s2 = threadIdx.x; s2 < SLOTS * GPB; s2 += BLOCK) {
        keys_all[s2] = kEmpty;
        vals_all[s2] = V(0);
    }
    if (threadIdx.x < GPB) {
        acc_e[threadIdx.x] = V(0);
        acc_s[threadIdx.x] = V(0);
        cnt[threadIdx.x] = 0;
    }
    __syncthreads();
    double sin = 0;
    unsigned dcnt = 0;
    for (uint32_t idx = blockIdx.x * GPB + g; idx - g < bin_size; idx += gridDim.x * GPB) {
        // the loop condition is uniform inside a group (GT == 32) or block (GT > 32)
        const bool active = idx < bin_size;
        uint32_t i = 0, src = 0, lo = 0, hi = 0;
        double ki = 0, a = 0;
        if (active) {
            i = A.perm[bin_off + idx];
            lo = A.off[i];
            hi = A.off[i + 1];
            src = A.P[i];
            ki = A.k[i];
            a = A.sigma[src] - ki;  // issued early, consumed after the edge pass
        }
        const int tb = table_bits<SLOTS>(hi - lo);
        V e_part = V(0), s_part = V(0);
        for (uint32_t base = lo + t; base < hi; base += GT * BATCH) {
            uint32_t jj[BATCH], cc[BATCH];
            V ww[BATCH];
#pragma unroll
            for (int b = 0; b < BATCH; b++) {
                uint32_t e = base + b * GT;
                jj[b] = e < hi ? __ldcs(A.col + e) : kEmpty;
                ww[b] = e < hi ? wget<WK>(A.w, e) : V(0);
            }
#pragma unroll
            for (int b = 0; b < BATCH; b++) cc[b] = jj[b] != kEmpty ? A.P[jj[b]] : kEmpty;
#pragma unroll
            for (int b = 0; b < BATCH; b++) {
                if (jj[b] == kEmpty) continue;
                const uint32_t c = cc[b];
                if (c != src) {
                    if (is_candidate<VER>(c, src, A.up)) {
                        const uint32_t mask = (1u << tb) - 1u;
                        uint32_t h = hash_slot(c, tb);
                        for (int p = 0; p < SLOTS; p++) {
                            uint32_t cur = ((volatile uint32_t *)keys)[h];
                            if (cur == c) break;
                            if (cur == kEmpty) {
                                uint32_t prev = atomicCAS(keys + h, kEmpty, c);
                                if (prev == kEmpty) {
                                    used[atomicAdd(cnt + g, 1u)] = (uint16_t)h;
                                    break;
                                }
                                if (prev == c) break;
                            }
                            h = (h + 1) & mask;
                        }
                        atomicAdd(vals + h, ww[b]);
                    }
                } else if (jj[b] != i) {
                    e_part += ww[b];
                } else {
                    s_part += ww[b];
                }
            }
        }
        // group totals of e and self weight, folded into the barrier that
        // publishes the table
        e_part = warp_sum(e_part);
        s_part = warp_sum(s_part);
        if ((threadIdx.x & 31) == 0) {
            if (e_part != V(0)) atomicAdd(acc_e + g, e_part);
            if (s_part != V(0)) atomicAdd(acc_s + g, s_part);
        }
        group_sync<GT>();
        const double e_src = v2d(acc_e[g]), selfw = v2d(acc_s[g]);
        const uint32_t nd = cnt[g];
        G best = G(0);
        uint32_t dst = src;
        for (uint32_t u0 = t; u0 < nd; u0 += GT * EB) {
            uint32_t kk[EB];
            double sc[EB], kv[EB];
#pragma unroll
            for (int b = 0; b < EB; b++) {
                const uint32_t u = u0 + b * GT;
                kk[b] = kEmpty;
                if (u < nd) {
                    const uint32_t h = used[u];
                    kk[b] = keys[h];
                    kv[b] = v2d(vals[h]);
                    keys[h] = kEmpty;
                    vals[h] = V(0);
                }
            }
#pragma unroll
            for (int b = 0; b < EB; b++)
                if (kk[b] != kEmpty) sc[b] = A.sigma[kk[b]];
#pragma unroll
            for (int b = 0; b < EB; b++) {
                if (kk[b] != kEmpty) {
                    G gn = Prec<PREC>::gain(kv[b], e_src, ki, a, sc[b], A);
                    if (better(gn, kk[b], best, dst, A.up)) {
                        best = gn;
                        dst = kk[b];
                    }
                }
            }
        }
        group_argmax<GT, G>(best, dst, A.up, red_g, red_c);
        if (t == 0) {
            if (active) {
                A.N[i] = final_choice<VER>(dst, src, A.up);
                sin += e_src + selfw;
                dcnt += nd;
            }
            cnt[g] = 0;
            acc_e[g] = V(0);
            acc_s[g] = V(0);
        }
        group_sync<GT>();
    }
    flush_acc(A.acc, A.integral, sin, dcnt);
}

// ============================================================================
// bin 9, tiers 0-4: one vertex per thread-block cluster of CS CTAs, the
// cluster's distributed shared memory holding one hash table of CS *
// kClusterSlots slots.  A neighbour community hashes to (owner CTA, slot);
// inserts into other CTAs' segments go through DSMEM atomics; each CTA then
// evaluates the candidates of its own segment, and rank 0 reduces the CS
// winners.  Two cluster barriers per vertex (accumulators double-buffered).
// Unit weights use packed 64-bit slots {key:32 | count:32}.
// ============================================================================
namespace cg = cooperative_groups;
constexpr int kClusterThreads = 1024;  // one CTA per SM with a 16K-slot segment
constexpr uint64_t kEmpty64 = 0xFFFFFFFF00000000ull;

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

template <int CS, int WK, int PREC, int VER>
__global__ void __launch_bounds__(kClusterThreads, 1) lm_cluster_kernel(LMArgs A, const uint32_t *verts,
                                                                        uint32_t count) {
    using G = typename Prec<PREC>::G;
    constexpr int S = kClusterSlots;
    constexpr int BATCH = 4;
    constexpr int EB = 4;  // slots per thread per evaluation batch
    extern __shared__ __align__(16) unsigned char smem_raw[];
    uint64_t *packed = (uint64_t *)smem_raw;                 // integral weights
    uint32_t *keys = (uint32_t *)smem_raw;                   // real weights
    double *vals = (double *)(smem_raw + sizeof(uint32_t) * S);
    // slots of this CTA's segment that received a new key, in insertion order
    uint16_t *used = (uint16_t *)(smem_raw + (kIntg<WK> ? sizeof(uint64_t) : sizeof(uint32_t) + sizeof(double)) * S);
    __shared__ uint32_t ucnt;
    __shared__ double acc_e[2], acc_s[2];
    __shared__ G best_g[2][CS];
    __shared__ uint32_t best_c[2][CS];
    __shared__ G red_g[32];
    __shared__ uint32_t red_c[32];
    unsigned rank = 0;
    if constexpr (CS > 1) rank = cg::this_cluster().block_rank();
    for (int s = threadIdx.x; s < S; s += kClusterThreads) {
        if constexpr (kIntg<WK>) packed[s] = kEmpty64;
        else {
            keys[s] = kEmpty;
            vals[s] = 0.0;
        }
    }
    if (threadIdx.x < 2) {
        acc_e[threadIdx.x] = 0;
        acc_s[threadIdx.x] = 0;
    }
    if (threadIdx.x == 0) ucnt = 0;
    cluster_barrier<CS>();
    const uint32_t cluster_id = blockIdx.x / CS, nclusters = gridDim.x / CS;
    const uint32_t tc = rank * kClusterThreads + threadIdx.x;
    constexpr uint32_t stride = CS * kClusterThreads;
    double sin = 0;
    unsigned dcnt = 0;
    int par = 0;
    for (uint32_t vi = cluster_id; vi < count; vi += nclusters, par ^= 1) {
        const uint32_t i = verts[vi];
        const uint32_t lo = A.off[i], hi = A.off[i + 1], src = A.P[i];
        const double ki = A.k[i];
        const double a = A.sigma[src] - ki;
        double e_part = 0, s_part = 0;
        for (uint32_t base = lo + tc; base < hi; base += stride * BATCH) {
            uint32_t jj[BATCH], cc[BATCH];
            double ww[BATCH];
#pragma unroll
            for (int b = 0; b < BATCH; b++) {
                uint32_t e = base + b * stride;
                jj[b] = e < hi ? __ldcs(A.col + e) : kEmpty;
                ww[b] = e < hi ? wload<WK>(A.w, e) : 0.0;
            }
#pragma unroll
            for (int b = 0; b < BATCH; b++) cc[b] = jj[b] != kEmpty ? A.P[jj[b]] : kEmpty;
#pragma unroll
            for (int b = 0; b < BATCH; b++) {
                if (jj[b] == kEmpty) continue;
                const uint32_t c = cc[b];
                if (c != src) {
                    if (!is_candidate<VER>(c, src, A.up)) continue;
                    const uint32_t h = hash_range(c, (uint32_t)CS * S);
                    const unsigned owner = h / S;
                    uint32_t s = h & (S - 1);
                    if constexpr (kIntg<WK>) {
                        const unsigned long long wi = (uint32_t)ww[b];
                        uint64_t *seg = rank_ptr<CS>(packed, owner);
                        bool placed = false;
                        for (int p = 0; p < S; p++) {
                            uint64_t cur = ((volatile uint64_t *)seg)[s];
                            uint32_t k = (uint32_t)(cur >> 32);
                            if (k == c) {
                                atomicAdd((unsigned long long *)(seg + s), wi);
                                placed = true;
                                break;
                            }
                            if (k == kEmpty) {
                                uint64_t prev = atomicCAS((unsigned long long *)(seg + s), kEmpty64,
                                                          ((uint64_t)c << 32) | wi);
                                if (prev == kEmpty64) {
                                    rank_ptr<CS>(used, owner)[atomicAdd(rank_ptr<CS>(&ucnt, owner), 1u)] =
                                        (uint16_t)s;
                                    placed = true;
                                    break;
                                }
                                if ((uint32_t)(prev >> 32) == c) {
                                    atomicAdd((unsigned long long *)(seg + s), wi);
                                    placed = true;
                                    break;
                                }
                            }
                            s = (s + 1) & (S - 1);
                        }
                        if (!placed) atomicAdd(&A.acc->overflow, 1ull);
                    } else {
                        uint32_t *ks = rank_ptr<CS>(keys, owner);
                        double *vs = rank_ptr<CS>(vals, owner);
                        bool placed = false;
                        for (int p = 0; p < S; p++) {
                            uint32_t cur = ((volatile uint32_t *)ks)[s];
                            if (cur == c) {
                                placed = true;
                                break;
                            }
                            if (cur == kEmpty) {
                                uint32_t prev = atomicCAS(ks + s, kEmpty, c);
                                if (prev == kEmpty) {
                                    rank_ptr<CS>(used, owner)[atomicAdd(rank_ptr<CS>(&ucnt, owner), 1u)] =
                                        (uint16_t)s;
                                    placed = true;
                                    break;
                                }
                                if (prev == c) {
                                    placed = true;
                                    break;
                                }
                            }
                            s = (s + 1) & (S - 1);
                        }
                        if (placed) atomicAdd(vs + s, ww[b]);
                        else atomicAdd(&A.acc->overflow, 1ull);
                    }
                } else if (jj[b] != i) {
                    e_part += ww[b];
                } else {
                    s_part += ww[b];
                }
            }
        }
        e_part = warp_sum(e_part);
        s_part = warp_sum(s_part);
        if ((threadIdx.x & 31) == 0) {
            if (e_part != 0) atomicAdd(rank_ptr<CS>(&acc_e[par], 0), e_part);
            if (s_part != 0) atomicAdd(rank_ptr<CS>(&acc_s[par], 0), s_part);
        }
        cluster_barrier<CS>();  // all inserts and partial sums are in
        const double e_src = *rank_ptr<CS>(&acc_e[par], 0);
        G best = G(0);
        uint32_t dst = src;
        const uint32_t nd = ucnt;
        for (uint32_t u0 = threadIdx.x; u0 < nd; u0 += kClusterThreads * EB) {
            uint32_t kk[EB];
            double kv[EB], sc[EB];
#pragma unroll
            for (int b = 0; b < EB; b++) {
                const uint32_t u = u0 + b * kClusterThreads;
                kk[b] = kEmpty;
                if (u < nd) {
                    const uint32_t s = used[u];
                    if constexpr (kIntg<WK>) {
                        uint64_t v = packed[s];
                        kk[b] = (uint32_t)(v >> 32);
                        kv[b] = u2d((uint32_t)v);
                        packed[s] = kEmpty64;
                    } else {
                        kk[b] = keys[s];
                        kv[b] = vals[s];
                        keys[s] = kEmpty;
                        vals[s] = 0.0;
                    }
                }
            }
#pragma unroll
            for (int b = 0; b < EB; b++)
                if (kk[b] != kEmpty) sc[b] = A.sigma[kk[b]];
#pragma unroll
            for (int b = 0; b < EB; b++) {
                if (kk[b] != kEmpty) {
                    G gn = Prec<PREC>::gain(kv[b], e_src, ki, a, sc[b], A);
                    if (better(gn, kk[b], best, dst, A.up)) {
                        best = gn;
                        dst = kk[b];
                    }
                }
            }
        }
        group_argmax<kClusterThreads, G>(best, dst, A.up, red_g, red_c);
        if (threadIdx.x == 0) {
            dcnt += nd;
            ucnt = 0;  // every thread of this CTA has read it (barriers in group_argmax)
            rank_ptr<CS>(&best_g[par][0], 0)[rank] = best;
            rank_ptr<CS>(&best_c[par][0], 0)[rank] = dst;
        }
        cluster_barrier<CS>();  // winners of every CTA are with rank 0
        if (rank == 0 && threadIdx.x == 0) {
            G bg = G(0);
            uint32_t bc = src;
            for (int r = 0; r < CS; r++)
                if (better(best_g[par][r], best_c[par][r], bg, bc, A.up)) {
                    bg = best_g[par][r];
                    bc = best_c[par][r];
                }
            A.N[i] = final_choice<VER>(bc, src, A.up);
            sin += e_src + acc_s[par];
            acc_e[par] = 0;
            acc_s[par] = 0;
        }
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

__global__ void heavy_degree_kernel(const uint32_t *off, const uint32_t *hv, uint32_t H, uint32_t *deg) {
    uint32_t h = blockIdx.x * blockDim.x + threadIdx.x;
    if (h < H) deg[h] = off[hv[h] + 1] - off[hv[h]];
}

__global__ void heavy_layout_kernel(const uint32_t *off, const uint32_t *hv, uint32_t H, uint32_t *tsize,
                                    uint32_t *ins_cnt, uint32_t *eval_cnt, uint64_t *tsz64) {
    uint32_t h = blockIdx.x * blockDim.x + threadIdx.x;
    if (h >= H) return;
    uint32_t v = hv[h];
    uint32_t d = off[v + 1] - off[v];
    uint32_t ts = (uint32_t)((2ull * d + 63) & ~63ull);
    tsize[h] = ts;
    tsz64[h] = ts;
    ins_cnt[h] = (d + kHeavyChunkE - 1) / kHeavyChunkE;
    eval_cnt[h] = (ts + kHeavyChunkS - 1) / kHeavyChunkS;
}

template <int WK, int VER>
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
    const uint32_t chunk = q - ins_off[h];
    const uint32_t vlo = A.off[v], vhi = A.off[v + 1];
    const uint32_t lo = vlo + chunk * kHeavyChunkE;
    const uint32_t hi = min(vhi, lo + kHeavyChunkE);
    const uint32_t src = A.P[v];
    const uint32_t ts = tsize[h];
    uint32_t *keys = tkeys + toff[h];
    double *vals = tvals + toff[h];
    double e_part = 0, s_part = 0;
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
        for (int b = 0; b < BATCH; b++) cc[b] = jj[b] != kEmpty ? A.P[jj[b]] : kEmpty;
#pragma unroll
        for (int b = 0; b < BATCH; b++) {
            if (jj[b] == kEmpty) continue;
            const uint32_t c = cc[b];
            if (c != src) {
                if (is_candidate<VER>(c, src, A.up)) {
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
                    atomicAdd(vals + s, ww[b]);
                }
            } else if (jj[b] != v) {
                e_part += ww[b];
            } else {
                s_part += ww[b];
            }
        }
    }
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
template <int PREC>
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
    const uint32_t part = q - eval_off[h];
    const uint32_t ts = tsize[h];
    const uint32_t lo = part * kHeavyChunkS, hi = min(ts, lo + kHeavyChunkS);
    uint32_t *keys = tkeys + toff[h];
    double *vals = tvals + toff[h];
    const uint32_t src = A.P[v];
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
            G gn = Prec<PREC>::gain(kv, e_src, ki, a, A.sigma[c], A);
            if (better(gn, c, best, dst, A.up)) {
                best = gn;
                dst = c;
            }
            dcnt++;
        }
    }
    group_argmax<kHeavyThreads, G>(best, dst, A.up, rg, rc);
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

template <int PREC, int VER>
__global__ void heavy_final_kernel(LMArgs A, const uint32_t *hv, uint32_t H, const uint32_t *eval_off,
                                   double *hacc, const unsigned long long *item_best) {
    using G = typename Prec<PREC>::G;
    const uint32_t h = blockIdx.x * blockDim.x + threadIdx.x;
    double sin = 0;
    if (h < H) {
        const uint32_t v = hv[h];
        const uint32_t src = A.P[v];
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
            if (better(g, c, best, dst, A.up)) {
                best = g;
                dst = c;
            }
        }
        A.N[v] = final_choice<VER>(dst, src, A.up);
        sin = hacc[2 * h] + hacc[2 * h + 1];
        hacc[2 * h] = 0;
        hacc[2 * h + 1] = 0;
    }
    flush_acc(A.acc, A.integral, sin, 0);
}

// ============================================================================
// sigma / modularity helpers
// ============================================================================
__global__ void sigma_update_kernel(const uint32_t *P, const uint32_t *N, const double *k, double *sigma, uint32_t n,
                                    SweepAcc *acc) {
    unsigned moved = 0;
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
        uint32_t a = P[v], b = N[v];
        if (a != b) {
            double kv = k[v];
            atomicAdd(sigma + a, -kv);
            atomicAdd(sigma + b, kv);
            moved++;
        }
    }
    unsigned long long m = warp_sum((unsigned long long)moved);
    if ((threadIdx.x & 31) == 0 && m) atomicAdd(&acc->moved, m);
}

__global__ void sigma_sumsq_kernel(const double *sigma, uint32_t n, int integral, SweepAcc *acc) {
    unsigned long long su = 0;
    double sf = 0;
    for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) {
        double s = sigma[c];
        if (integral) {
            unsigned long long u = (unsigned long long)s;
            su += u * u;
        } else {
            sf += s * s;
        }
    }
    su = warp_sum(su);
    sf = warp_sum(sf);
    if ((threadIdx.x & 31) == 0) {
        if (integral) {
            if (su) atomicAdd(&acc->s2_u, su);
        } else if (sf != 0) {
            atomicAdd(&acc->s2_f, sf);
        }
    }
}

template <int WK>
__global__ void level_init_kernel(const uint32_t *off, const void *w, uint32_t n, double *k, double *sigma,
                                  uint32_t *C) {
    // one warp per vertex
    const uint32_t lane = threadIdx.x & 31;
    for (uint32_t v = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; v < n; v += (gridDim.x * blockDim.x) >> 5) {
        uint32_t lo = off[v], hi = off[v + 1];
        double s;
        if constexpr (WK == WK_UNIT) {
            s = (double)(hi - lo);
        } else {
            s = 0;
            for (uint32_t e = lo + lane; e < hi; e += 32) s += wload<WK>(w, e);
            s = warp_sum(s);
        }
        if (lane == 0) {
            k[v] = s;
            sigma[v] = s;
            C[v] = v;
        }
    }
}

template <int CS, int WK, int PREC, int VER>
size_t cluster_smem() {
    return (size_t)kClusterSlots * ((kIntg<WK> ? sizeof(uint64_t) : sizeof(uint32_t) + sizeof(double)) + sizeof(uint16_t));
}

template <int CS, int WK, int PREC, int VER>
cudaLaunchConfig_t cluster_config(size_t smem, unsigned grid, cudaStream_t s, cudaLaunchAttribute *attr) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid, 1, 1);
    cfg.blockDim = dim3(kClusterThreads, 1, 1);
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

// Maximum co-resident clusters of a cluster kernel (0 when the shape cannot run).
template <int CS, int WK, int PREC, int VER>
int cluster_capacity() {
    static int cap = -1;
    if (cap >= 0) return cap;
    auto kern = lm_cluster_kernel<CS, WK, PREC, VER>;
    const size_t smem = cluster_smem<CS, WK, PREC, VER>();
    MG_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    if (CS > 8) MG_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
    cudaLaunchAttribute attr[1];
    cudaLaunchConfig_t cfg = cluster_config<CS, WK, PREC, VER>(smem, CS * 148, nullptr, attr);
    int n = 0;
    if (cudaOccupancyMaxActiveClusters(&n, (void *)kern, &cfg) != cudaSuccess) {
        cudaGetLastError();
        n = 0;
    }
    cap = n;
    return cap;
}

template <int CS, int WK, int PREC, int VER>
void launch_cluster(const LMArgs &A, const uint32_t *verts, uint32_t count, cudaStream_t s) {
    auto kern = lm_cluster_kernel<CS, WK, PREC, VER>;
    const size_t smem = cluster_smem<CS, WK, PREC, VER>();
    int cap = cluster_capacity<CS, WK, PREC, VER>();
    MG_CHECK(cap > 0, MG_ERR_UNSUPPORTED, "cluster shape cannot be scheduled on this device");
    unsigned clusters = (unsigned)std::min<uint64_t>(count, (uint64_t)cap);
    cudaLaunchAttribute attr[1];
    cudaLaunchConfig_t cfg = cluster_config<CS, WK, PREC, VER>(smem, clusters * CS, s, attr);
    MG_CUDA(cudaLaunchKernelEx(&cfg, kern, A, verts, count));
    MG_LAUNCH_CHECK();
}

// Largest cluster size (8 or 16) the device schedules for the heavy tiers.
int probe_max_cluster() {
    return cluster_capacity<16, WK_F64, MG_PREC_FP64, 2>() > 0 && cluster_capacity<16, WK_UNIT, MG_PREC_FP64, 2>() > 0
               ? 16
               : 8;
}

template <int WK, int PREC, int VER>
void launch_sweep(const GraphView &g, const MoveLevel &lvl, MoveWorkspace &ws, const LMArgs &A, cudaStream_t s) {
    const Bins &B = lvl.bins;
    // fork: heavy path on its own stream, the tile and hash bins on others
    MG_CUDA(cudaEventRecord(ws.ev_fork, s));
    for (int q = 0; q < 3; q++) MG_CUDA(cudaStreamWaitEvent(ws.streams[q], ws.ev_fork, 0));
    cudaStream_t sh = ws.streams[0], sm = ws.streams[1], st = ws.streams[2];
    // heavy tiers, largest clusters first
    if (lvl.tier_off[5] > lvl.tier_off[4])
        launch_cluster<16, WK, PREC, VER>(A, ws.h_tier.get() + lvl.tier_off[4], lvl.tier_off[5] - lvl.tier_off[4], sh);
    if (lvl.tier_off[4] > lvl.tier_off[3])
        launch_cluster<8, WK, PREC, VER>(A, ws.h_tier.get() + lvl.tier_off[3], lvl.tier_off[4] - lvl.tier_off[3], sh);
    if (lvl.tier_off[3] > lvl.tier_off[2])
        launch_cluster<4, WK, PREC, VER>(A, ws.h_tier.get() + lvl.tier_off[2], lvl.tier_off[3] - lvl.tier_off[2], sh);
    if (lvl.tier_off[2] > lvl.tier_off[1])
        launch_cluster<2, WK, PREC, VER>(A, ws.h_tier.get() + lvl.tier_off[1], lvl.tier_off[2] - lvl.tier_off[1], sh);
    if (lvl.tier_off[1] > lvl.tier_off[0])
        launch_cluster<1, WK, PREC, VER>(A, ws.h_tier.get() + lvl.tier_off[0], lvl.tier_off[1] - lvl.tier_off[0], sm);
    if (lvl.giants > 0) {
        const uint32_t H = lvl.giants;
        const uint32_t *hv = ws.h_tier.get() + lvl.tier_off[kTiers - 1];
        heavy_insert_kernel<WK, VER><<<lvl.ins_items, kHeavyThreads, 0, sh>>>(
            A, hv, H, ws.h_ins.get(), ws.h_toff.get(), ws.h_tsize.get(), ws.h_keys.get(), ws.h_vals.get(),
            ws.h_acc.get());
        MG_LAUNCH_CHECK();
        heavy_eval_kernel<PREC><<<lvl.eval_items, kHeavyThreads, 0, sh>>>(
            A, hv, H, ws.h_eval.get(), ws.h_toff.get(), ws.h_tsize.get(), ws.h_keys.get(), ws.h_vals.get(),
            ws.h_acc.get(), ws.h_best.get());
        MG_LAUNCH_CHECK();
        heavy_final_kernel<PREC, VER><<<(unsigned)ceil_div(H, 256), 256, 0, sh>>>(A, hv, H, ws.h_eval.get(),
                                                                                  ws.h_acc.get(), ws.h_best.get());
        MG_LAUNCH_CHECK();
    }
    using V = typename ValT<WK>::type;
    auto hash_launch = [&](auto kern, int slots, int gpb, int block, int bin, cudaStream_t str) {
        if (B.size[bin] == 0) return;
        size_t smem = (size_t)slots * gpb * (sizeof(uint32_t) + sizeof(V) + sizeof(uint16_t) / 2);
        MG_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        unsigned grid = (unsigned)std::min<uint64_t>(ceil_div(B.size[bin], gpb), 148ull * 64);
        kern<<<grid, block, smem, str>>>(A, B.offset[bin], B.size[bin]);
        MG_LAUNCH_CHECK();
    };
    hash_launch(lm_hash_kernel<512, 8192, WK, PREC, VER, 512>, 8192, 1, 512, 8, sm);
    hash_launch(lm_hash_kernel<256, 4096, WK, PREC, VER, 256>, 4096, 1, 256, 7, sm);
    hash_launch(lm_hash_kernel<128, 1024, WK, PREC, VER, 128>, 1024, 1, 128, 6, sm);
    hash_launch(lm_hash_kernel<32, 256, WK, PREC, VER, 256>, 256, 8, 256, 5, st);
    auto tile_launch = [&](auto kern, int T, int bin, cudaStream_t str) {
        if (B.size[bin] == 0) return;
        uint64_t groups_per_block = 256 / T;
        unsigned grid = (unsigned)std::min<uint64_t>(ceil_div(B.size[bin], groups_per_block), 148ull * 32);
        kern<<<grid, 256, 0, str>>>(A, B.offset[bin], B.size[bin]);
        MG_LAUNCH_CHECK();
    };
    tile_launch(lm_tile_kernel<32, WK, PREC, VER>, 32, 4, st);
    tile_launch(lm_tile_kernel<16, WK, PREC, VER>, 16, 3, st);
    tile_launch(lm_tile_kernel<8, WK, PREC, VER>, 8, 2, st);
    tile_launch(lm_tile_kernel<4, WK, PREC, VER>, 4, 1, st);
    tile_launch(lm_tile_kernel<2, WK, PREC, VER>, 2, 0, st);
    for (int q = 0; q < 3; q++) {
        MG_CUDA(cudaEventRecord(ws.ev_join[q], ws.streams[q]));
        MG_CUDA(cudaStreamWaitEvent(s, ws.ev_join[q], 0));
    }
}

}  // namespace

MoveWorkspace::~MoveWorkspace() {
    for (auto &s : streams)
        if (s) cudaStreamDestroy(s);
    if (ev_fork) cudaEventDestroy(ev_fork);
    for (auto &e : ev_join)
        if (e) cudaEventDestroy(e);
}

void MoveWorkspace::init_streams() {
    if (streams[0]) return;
    for (auto &s : streams) MG_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    MG_CUDA(cudaEventCreateWithFlags(&ev_fork, cudaEventDisableTiming));
    for (auto &e : ev_join) MG_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
}

void move_prepare_level(const GraphView &g, MoveLevel &lvl, MoveWorkspace &ws, cudaStream_t s) {
    ws.init_streams();
    ws.acc.ensure(1);
    uint32_t *perm = ws.perm.ensure(g.n + 1);
    compute_bins(0, g.n, g.off, perm, lvl.bins, s, ws.prim);
    lvl.heavy = lvl.bins.size[9];
    lvl.ins_items = lvl.eval_items = 0;
    lvl.table_slots = 0;
    lvl.giants = 0;
    for (int t = 0; t <= kTiers; t++) lvl.tier_off[t] = 0;
    if (lvl.heavy == 0) return;
    if (ws.max_cluster == 0) ws.max_cluster = probe_max_cluster();
    // tiers by degree: tier t (cluster of 2^t CTAs) takes deg <= 2^t * S / 2
    {
        const uint32_t Hall = lvl.heavy;
        const uint32_t *hall = perm + lvl.bins.offset[9];
        uint32_t *deg = ws.h_deg.ensure(Hall + 1);
        heavy_degree_kernel<<<(unsigned)ceil_div(Hall, 256), 256, 0, s>>>(g.off, hall, Hall, deg);
        MG_LAUNCH_CHECK();
        std::vector<uint32_t> hv_h(Hall), dg_h(Hall);
        MG_CUDA(cudaMemcpyAsync(hv_h.data(), hall, sizeof(uint32_t) * Hall, cudaMemcpyDeviceToHost, s));
        MG_CUDA(cudaMemcpyAsync(dg_h.data(), deg, sizeof(uint32_t) * Hall, cudaMemcpyDeviceToHost, s));
        MG_CUDA(cudaStreamSynchronize(s));
        std::vector<uint32_t> lists[kTiers];
        const int top = ws.max_cluster >= 16 ? 4 : 3;
        for (uint32_t h = 0; h < Hall; h++) {
            int t = kTiers - 1;
            for (int c = 0; c <= top; c++)
                if ((uint64_t)dg_h[h] <= (uint64_t)(kClusterSlots / 2) << c) {
                    t = c;
                    break;
                }
            lists[t].push_back(hv_h[h]);
        }
        std::vector<uint32_t> tiered;
        tiered.reserve(Hall);
        for (int t = 0; t < kTiers; t++) {
            lvl.tier_off[t] = (uint32_t)tiered.size();
            tiered.insert(tiered.end(), lists[t].begin(), lists[t].end());
        }
        lvl.tier_off[kTiers] = (uint32_t)tiered.size();
        MG_CUDA(cudaMemcpyAsync(ws.h_tier.ensure(Hall + 1), tiered.data(), sizeof(uint32_t) * Hall,
                                cudaMemcpyHostToDevice, s));
        lvl.giants = lvl.tier_off[kTiers] - lvl.tier_off[kTiers - 1];
        MG_CUDA(cudaStreamSynchronize(s));
    }
    if (lvl.giants == 0) return;
    const uint32_t H = lvl.giants;
    const uint32_t *hv = ws.h_tier.get() + lvl.tier_off[kTiers - 1];
    uint32_t *tsize = ws.h_tsize.ensure(H + 1);
    uint32_t *ins = ws.h_ins.ensure(H + 1);
    uint32_t *ev = ws.h_eval.ensure(H + 1);
    uint64_t *toff = ws.h_toff.ensure(H + 1);
    uint64_t *tmp = ws.tmp64.ensure(H + 1);
    heavy_layout_kernel<<<(unsigned)ceil_div(H, 256), 256, 0, s>>>(g.off, hv, H, tsize, ins, ev, tmp);
    MG_LAUNCH_CHECK();
    exclusive_scan<uint32_t>(ins, ins, H, ins + H, s, ws.prim);
    exclusive_scan<uint32_t>(ev, ev, H, ev + H, s, ws.prim);
    exclusive_scan<uint64_t>(tmp, toff, H, toff + H, s, ws.prim);
    uint32_t ni = 0, ne = 0;
    uint64_t slots = 0;
    MG_CUDA(cudaMemcpyAsync(&ni, ins + H, sizeof ni, cudaMemcpyDeviceToHost, s));
    MG_CUDA(cudaMemcpyAsync(&ne, ev + H, sizeof ne, cudaMemcpyDeviceToHost, s));
    MG_CUDA(cudaMemcpyAsync(&slots, toff + H, sizeof slots, cudaMemcpyDeviceToHost, s));
    MG_CUDA(cudaStreamSynchronize(s));
    lvl.ins_items = ni;
    lvl.eval_items = ne;
    lvl.table_slots = slots;
    uint32_t *keys = ws.h_keys.ensure(slots);
    double *vals = ws.h_vals.ensure(slots);
    MG_CUDA(cudaMemsetAsync(keys, 0xFF, slots * sizeof(uint32_t), s));
    MG_CUDA(cudaMemsetAsync(vals, 0, slots * sizeof(double), s));
    double *hacc = ws.h_acc.ensure(2ull * H);
    MG_CUDA(cudaMemsetAsync(hacc, 0, 2ull * H * sizeof(double), s));
    ws.h_best.ensure(2ull * ne + 2);
}

void sweep_reset_acc(MoveWorkspace &ws, cudaStream_t s) {
    MG_CUDA(cudaMemsetAsync(ws.acc.ensure(1), 0, sizeof(SweepAcc), s));
}

void move_sweep(const GraphView &g, const MoveLevel &lvl, MoveWorkspace &ws, const SweepParams &p,
                const uint32_t *P, uint32_t *N, const double *k, const double *sigma, cudaStream_t s) {
    LMArgs A;
    A.off = g.off;
    A.col = g.col;
    A.w = g.w;
    A.P = P;
    A.N = N;
    A.k = k;
    A.sigma = sigma;
    A.perm = ws.perm.get();
    A.m = p.mass / 2.0;
    A.two_m = 2.0 * A.m;
    A.r_m = 1.0 / A.m;
    A.r_two_m = 1.0 / A.two_m;
    A.m_f = (float)(p.mass / 2.0);
    A.two_m_f = 2.0f * A.m_f;
    A.r_m_f = 1.0f / A.m_f;
    A.r_two_m_f = 1.0f / A.two_m_f;
    A.mass_i = (long long)p.mass;
    A.up = p.up;
    A.integral = p.integral;
    A.acc = ws.acc.ensure(1);
    MG_CHECK(p.version == 1 || p.version == 2, MG_ERR_INVALID, "version must be 0, 1 or 2");
    if (p.precision == MG_PREC_INT64)
        MG_CHECK(p.integral && p.mass < 2147483648.0, MG_ERR_UNSUPPORTED,
                 "int64 precision needs integral weights with total below 2^31");
    // integral graphs accumulate in integer table slots
    const int wk = p.integral ? (g.wk == WK_F32 ? (int)WK_F32I : g.wk == WK_F64 ? (int)WK_F64I : g.wk) : g.wk;
#define MG_SWEEP_CASE(WKV, PRECV)                                                                  \
    if (wk == WKV && p.precision == PRECV) {                                                       \
        if (p.version == 1) launch_sweep<WKV, PRECV, 1>(g, lvl, ws, A, s);                         \
        else launch_sweep<WKV, PRECV, 2>(g, lvl, ws, A, s);                                        \
        return;                                                                                    \
    }
    MG_SWEEP_CASE(WK_UNIT, MG_PREC_FP64)
    MG_SWEEP_CASE(WK_F32I, MG_PREC_FP64)
    MG_SWEEP_CASE(WK_F64I, MG_PREC_FP64)
    MG_SWEEP_CASE(WK_F32, MG_PREC_FP64)
    MG_SWEEP_CASE(WK_F64, MG_PREC_FP64)
    MG_SWEEP_CASE(WK_UNIT, MG_PREC_INT64)
    MG_SWEEP_CASE(WK_F32I, MG_PREC_INT64)
    MG_SWEEP_CASE(WK_F64I, MG_PREC_INT64)
    MG_SWEEP_CASE(WK_UNIT, MG_PREC_FP32)
    MG_SWEEP_CASE(WK_F32I, MG_PREC_FP32)
    MG_SWEEP_CASE(WK_F64I, MG_PREC_FP32)
    MG_SWEEP_CASE(WK_F32, MG_PREC_FP32)
    MG_SWEEP_CASE(WK_F64, MG_PREC_FP32)
#undef MG_SWEEP_CASE
    throw Error(MG_ERR_INVALID, "unknown weight kind or precision");
}

void sigma_sumsq(const double *sigma, uint32_t n, int integral, MoveWorkspace &ws, cudaStream_t s) {
    if (n == 0) return;
    unsigned grid = (unsigned)std::min<uint64_t>(ceil_div(n, 256), 148ull * 8);
    sigma_sumsq_kernel<<<grid, 256, 0, s>>>(sigma, n, integral, ws.acc.ensure(1));
    MG_LAUNCH_CHECK();
}

void sigma_update(const uint32_t *P, const uint32_t *N, const double *k, double *sigma, uint32_t n,
                  MoveWorkspace &ws, cudaStream_t s) {
    if (n == 0) return;
    unsigned grid = (unsigned)std::min<uint64_t>(ceil_div(n, 256), 148ull * 8);
    sigma_update_kernel<<<grid, 256, 0, s>>>(P, N, k, sigma, n, ws.acc.ensure(1));
    MG_LAUNCH_CHECK();
}

void level_init(const GraphView &g, double *k, double *sigma, uint32_t *C, cudaStream_t s) {
    if (g.n == 0) return;
    unsigned grid = (unsigned)std::min<uint64_t>(ceil_div(g.n, 8), 148ull * 16);
    if (g.wk == WK_UNIT) level_init_kernel<WK_UNIT><<<grid, 256, 0, s>>>(g.off, g.w, g.n, k, sigma, C);
    else if (g.wk == WK_F32) level_init_kernel<WK_F32><<<grid, 256, 0, s>>>(g.off, g.w, g.n, k, sigma, C);
    else level_init_kernel<WK_F64><<<grid, 256, 0, s>>>(g.off, g.w, g.n, k, sigma, C);
    MG_LAUNCH_CHECK();
}

double modularity_from_acc(const SweepAcc &a, double mass, int integral) {
    if (integral) return (double)a.sin_u / mass - (double)a.s2_u / (mass * mass);
    return a.sin_f / mass - a.s2_f / (mass * mass);
}

}  // namespace mg
