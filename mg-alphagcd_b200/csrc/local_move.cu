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
#include "lm_kernels.cuh"

namespace mg {

namespace {

using namespace lmk;

// row range of every class-list entry (class order)
__global__ void row_ranges_kernel(const uint32_t *off, const uint32_t *perm, uint32_t n, uint2 *rows) {
    for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
        const uint32_t i = perm[q];
        rows[q] = make_uint2(off[i], off[i + 1]);
    }
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

// Largest cluster size (8 or 16) the device schedules for the heavy tiers.
// (the largest tier: 16 CTAs for real weights, 8 dense CTAs for integral ones)
int probe_max_cluster() {
    return cluster_capacity<tier_ctas<WK_F64>(4), WK_F64, MG_PREC_FP64, 2, 0>() > 0 &&
                   cluster_capacity<tier_ctas<WK_UNIT>(4), WK_UNIT, MG_PREC_FP64, 2, 0, kDenseTier<WK_UNIT>(4)>() > 0
               ? 16
               : 8;
}

}  // namespace

const char *shape_name(int sh) {
    static const char *names[SH_COUNT] = {"t2", "t4", "t8", "t16", "t32", "h32", "h64", "h128", "h256", "h512", "w"};
    return sh >= 0 && sh < SH_COUNT ? names[sh] : "?";
}

// The shapes before any tuning: T-lane tiles up to degree 32, a warp per
// vertex up to 128, then 128 / 256 / 512 threads per vertex.
int default_shape(int cls) {
    static const uint8_t d[kLightClasses] = {SH_T2,  SH_T2,   SH_T4,   SH_T8,   SH_T16,  SH_T32, SH_H32,
                                             SH_H32, SH_H128, SH_H128, SH_H256, SH_H256, SH_H512};
    return cls >= 0 && cls < kLightClasses ? d[cls] : SH_H512;
}

MoveWorkspace::~MoveWorkspace() {
    for (auto &s : streams)
        if (s) cudaStreamDestroy(s);
    if (ev_fork) cudaEventDestroy(ev_fork);
    for (auto &e : ev_join)
        if (e) cudaEventDestroy(e);
    for (auto &e : ev_tune)
        if (e) cudaEventDestroy(e);
}

void MoveWorkspace::init_streams() {
    if (streams[0]) return;
    for (auto &s : streams) MG_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    MG_CUDA(cudaEventCreateWithFlags(&ev_fork, cudaEventDisableTiming));
    for (auto &e : ev_join) MG_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    for (auto &e : ev_tune) MG_CUDA(cudaEventCreate(&e));
}

void move_prepare_level(const GraphView &g, MoveLevel &lvl, MoveWorkspace &ws, cudaStream_t s) {
    ws.init_streams();
    ws.acc.ensure(1);
    uint32_t *perm = ws.perm.ensure(g.n + 1);
    compute_bins(kSweepScheme, g.n, g.off, perm, lvl.bins, s, ws.prim);
    uint2 *rows = ws.rows.ensure(g.n + 1);
    if (g.n) {
        row_ranges_kernel<<<(unsigned)std::min<uint64_t>(ceil_div(g.n, 256), 148 * 16), 256, 0, s>>>(g.off, perm, g.n,
                                                                                                     rows);
        MG_LAUNCH_CHECK();
    }
    for (int c = 0; c < kLightClasses; c++) lvl.shape[c] = (uint8_t)default_shape(c);
    const uint32_t h0 = lvl.bins.offset[kFirstHeavyClass];
    lvl.heavy = g.n - h0;
    lvl.heavy_list = perm + h0;
    lvl.ins_items = lvl.eval_items = 0;
    lvl.table_slots = 0;
    lvl.giants = 0;
    for (int t = 0; t <= kTiers; t++) lvl.tier_off[t] = 0;
    if (lvl.heavy == 0) return;
    if (ws.max_cluster == 0) ws.max_cluster = probe_max_cluster();
    // classes 13..17 are the cluster tiers (tier t: tier_ctas(t) CTAs holding
    // degrees up to 2^(13+t) at load <= 1/2, or <= 2/3 with dense segments),
    // class 18 the giants; on a
    // device without 12- and 16-CTA clusters class 17 joins the giants, and so
    // do the classes from ws.giant_class on
    int first_giant = std::min(ws.giant_class - kFirstHeavyClass, kTiers - 1);
    if (ws.max_cluster < 16) first_giant = std::min(first_giant, kTiers - 2);
    for (int t = 0; t < kTiers; t++)
        lvl.tier_off[t] = lvl.bins.offset[kFirstHeavyClass + std::min(t, first_giant)] - h0;
    lvl.tier_off[kTiers] = lvl.heavy;
    lvl.giants = lvl.tier_off[kTiers] - lvl.tier_off[kTiers - 1];
    if (lvl.giants == 0) return;
    const uint32_t H = lvl.giants;
    const uint32_t *hv = lvl.heavy_list + lvl.tier_off[kTiers - 1];
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

GainK gain_constants(double mass) {
    GainK K;
    K.m = mass / 2.0;
    K.two_m = 2.0 * K.m;
    K.r_m = 1.0 / K.m;
    K.r_two_m = 1.0 / K.two_m;
    K.m_f = (float)(mass / 2.0);
    K.two_m_f = 2.0f * K.m_f;
    K.r_m_f = 1.0f / K.m_f;
    K.r_two_m_f = 1.0f / K.two_m_f;
    K.mass_i = (long long)mass;
    return K;
}

namespace {
LMArgs single_args(const GraphView &g, MoveWorkspace &ws, const SweepParams &p, const uint32_t *P, uint32_t *N,
                   const double *k, const double *sigma) {
    LMArgs A = {};
    A.off = g.off;
    A.col = g.col;
    A.w = g.w;
    A.P = P;
    A.N = N;
    A.k = k;
    A.sigma = sigma;
    A.perm = ws.perm.get();
    A.rows = ws.rows.get();
    A.K = gain_constants(p.mass);
    A.up = p.up;
    A.integral = p.integral;
    A.agg = p.agg;
    A.split = p.split;
    A.first = p.first;
    A.acc = ws.acc.ensure(1);
    if (p.precision == MG_PREC_INT64)
        MG_CHECK(p.integral && p.mass < 2147483648.0, MG_ERR_UNSUPPORTED,
                 "int64 precision needs integral weights with total below 2^31");
    return A;
}
}  // namespace

void move_sweep(const GraphView &g, const MoveLevel &lvl, MoveWorkspace &ws, const SweepParams &p,
                const uint32_t *P, uint32_t *N, const double *k, const double *sigma, cudaStream_t s) {
    const LMArgs A = single_args(g, ws, p, P, N, k, sigma);
    dispatch_sweep<0>(g, lvl, ws, p, A, s);
}

void move_tune(const GraphView &g, MoveLevel &lvl, MoveWorkspace &ws, const SweepParams &p, const uint32_t *P,
               uint32_t *N, const double *k, const double *sigma, cudaStream_t s, bool timing) {
    tune_light<0>(g, lvl, ws, p, single_args(g, ws, p, P, N, k, sigma), s, timing);
}

void sigma_sumsq(const double *sigma, uint32_t n, int integral, MoveWorkspace &ws, cudaStream_t s) {
    if (n == 0) return;
    unsigned grid = (unsigned)std::min<uint64_t>(ceil_div(n, 256), 148ull * 8);
    SweepAcc *acc = ws.acc.ensure(1);  // (allocations stay out of launch argument lists)
    sigma_sumsq_kernel<<<grid, 256, 0, s>>>(sigma, n, integral, acc);
    MG_LAUNCH_CHECK();
}

void sigma_update(const uint32_t *P, const uint32_t *N, const double *k, double *sigma, uint32_t n,
                  MoveWorkspace &ws, cudaStream_t s) {
    if (n == 0) return;
    unsigned grid = (unsigned)std::min<uint64_t>(ceil_div(n, 256), 148ull * 8);
    SweepAcc *acc = ws.acc.ensure(1);
    sigma_update_kernel<<<grid, 256, 0, s>>>(P, N, k, sigma, n, acc);
    MG_LAUNCH_CHECK();
}

void level_init(const GraphView &g, double *k, double *sigma, uint32_t *C, cudaStream_t s) {
    if (g.n == 0) return;
    unsigned grid = (unsigned)std::min<uint64_t>(ceil_div(g.n, 8), 148ull * 16);
    if (g.wk == WK_UNIT) level_init_kernel<WK_UNIT><<<grid, 256, 0, s>>>(g.off, g.w, g.n, k, sigma, C);
    else if (g.wk == WK_F32) level_init_kernel<WK_F32><<<grid, 256, 0, s>>>(g.off, g.w, g.n, k, sigma, C);
    else if (g.wk == WK_U32) level_init_kernel<WK_U32><<<grid, 256, 0, s>>>(g.off, g.w, g.n, k, sigma, C);
    else level_init_kernel<WK_F64><<<grid, 256, 0, s>>>(g.off, g.w, g.n, k, sigma, C);
    MG_LAUNCH_CHECK();
}

double modularity_from_acc(const SweepAcc &a, double mass, int integral) {
    if (integral) return (double)a.sin_u / mass - (double)a.s2_u / (mass * mass);
    return a.sin_f / mass - a.s2_f / (mass * mass);
}

}  // namespace mg
