// batch.cu -- the batched form: many graphs run as one disjoint union.
//
// Every graph follows louvain::run's control flow (src/louvain/louvain.cu:
// 1401-1715) on its own -- own mass, gain constants, modularity, accept /
// reject decisions, phase exit -- while one set of kernel launches per sweep
// covers all graphs:
//   * sweeps: the local-move kernels with per-vertex graph lookups
//     (local_move_batch.cu); each graph's control word says which of the three
//     assignment buffers the sweep reads and writes, and graphs that are done
//     with the phase are skipped;
//   * after a sweep, per-graph sums of sum_in and sigma^2 (vertex ranges of a
//     graph are contiguous) give each graph's Q; one thread per graph then
//     takes the accept / reject decision of the single-graph loop with the same
//     double operations, rotates the graph's buffers and flags the sigma
//     update; a vertex-parallel kernel applies the updates;
//   * at the end of a phase the final assignments of all graphs are relabelled
//     densely in one pass (order preserving, so each graph's communities stay a
//     contiguous, ordered id range) and the union is coarsened in one pass,
//     which coarsens every graph exactly as alone.
// Graphs whose run has ended stay in the union as inactive vertices (their
// coarsest level, with the identity assignment).
//
// Graphs converge after different numbers of sweeps, so a phase runs until its
// slowest graph is done.  The sweeps therefore walk compacted lists of the
// vertices of active graphs -- the degree-class list (classes 0-12, in class order)
// and the vertex list (id order) for the per-graph sums and sigma updates --
// with the graph of every entry stored beside it.  The lists are rebuilt at the
// start of a phase and whenever the vertices of active graphs fall to half of
// the listed ones, so the cost of a sweep follows the work left.
//
// With MG_BATCH_GRAPHS the iterations of a phase run as one CUDA graph: a
// conditional while node whose body is the sweep, the per-graph sums, the
// decisions and the sigma update; the decision kernel ends the loop when no
// graph is active or the launch's sweep budget is used up, and the host
// relaunches while graphs remain active.
#include <cmath>
#include <memory>

#include "handles.cuh"

namespace mg {

BatchWork::~BatchWork() {
    if (h_ctrl) cudaFreeHost(h_ctrl);
}

namespace {

constexpr int kSumVPT = 8;  // vertices per lane in the per-graph sums
constexpr long long kGraphBudget = 64;  // sweeps per CUDA-graph launch

unsigned grid_n(uint64_t n, unsigned per = 256, uint64_t cap = 148ull * 16) {
    uint64_t b = ceil_div(n, per);
    if (b < 1) b = 1;
    return (unsigned)(b < cap ? b : cap);
}

// gid[v] = last g with goff[g] <= v
__global__ void gid_fill_kernel(const uint32_t *goff, uint32_t G, uint32_t n, uint32_t *gid) {
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
        uint32_t lo = 0, hi = G;
        while (hi - lo > 1) {
            uint32_t mid = (lo + hi) >> 1;
            if (goff[mid] <= v) lo = mid;
            else hi = mid;
        }
        gid[v] = lo;
    }
}

__global__ void gnnz_kernel(const uint32_t *off, const uint32_t *goff, uint32_t G, uint32_t *gnnz) {
    uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g < G) gnnz[g] = off[goff[g + 1]] - off[goff[g]];
}

// start of a phase: graphs still running sweep first from buffer 0 (the
// identity) into buffer 1; the others are inactive with base buffer 0
__global__ void phase_init_kernel(const uint8_t *alive, uint32_t G, uint32_t *gword, GSum *sums, uint32_t *loops,
                                  BatchCtrl *ctrl) {
    uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g < G) {
        gword[g] = alive[g] ? gw_make(true, 0, 1, 0, true, false, 0, 0) : 0u;
        sums[g] = GSum{0, 0, 0, 0};
        loops[g] = 0;
    }
    if (g == 0) {
        ctrl->up = 1;
        ctrl->active = 0;
    }
}

// Per-graph sums over the vertices of active graphs: sum_in contributions of
// the sweep and sigma^2 (community ids are vertex ids of the same graph).
// One warp per chunk of 32 * kSumVPT consecutive vertices: a chunk inside one
// graph is reduced in the warp and added with one atomic per sum; chunks that
// straddle graphs add per vertex.
// The list is in id order, so the graphs of its entries do not decrease.
template <int INTEGRAL>
__global__ void gsum_kernel(const uint32_t *list, const uint32_t *lgid, uint32_t L, const uint32_t *gword,
                            const double *sinv, const double *sigma, GSum *sums, BatchCtrl *ctrl) {
    if (blockIdx.x == 0 && threadIdx.x == 0) {  // recounted by the decisions
        ctrl->active = 0;
        ctrl->active_vertices = 0;
    }
    const uint32_t lane = threadIdx.x & 31;
    constexpr uint32_t CH = 32 * kSumVPT;
    const uint64_t nchunks = ((uint64_t)L + CH - 1) / CH;
    for (uint64_t ch = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5; ch < nchunks;
         ch += ((uint64_t)gridDim.x * blockDim.x) >> 5) {
        const uint32_t i0 = (uint32_t)(ch * CH);
        const uint32_t i1 = (uint32_t)min((uint64_t)i0 + CH, (uint64_t)L);
        const uint32_t g0 = lgid[i0], g1 = lgid[i1 - 1];
        if (g0 == g1) {
            if (!(gword[g0] & kGwActive)) continue;
            unsigned long long su = 0, s2u = 0;
            double sf = 0, s2f = 0;
#pragma unroll
            for (int t = 0; t < kSumVPT; t++) {
                const uint32_t i = i0 + lane + 32 * t;
                if (i < i1) {
                    const uint32_t v = list[i];
                    const double x = sinv[v], sg = sigma[v];
                    if (INTEGRAL) {
                        const unsigned long long q = (unsigned long long)sg;
                        su += (unsigned long long)x;
                        s2u += q * q;
                    } else {
                        sf += x;
                        s2f += sg * sg;
                    }
                }
            }
            if (INTEGRAL) {
                su = warp_sum(su);
                s2u = warp_sum(s2u);
                if (lane == 0) {
                    if (su) atomicAdd(&sums[g0].sin_u, su);
                    if (s2u) atomicAdd(&sums[g0].s2_u, s2u);
                }
            } else {
                sf = warp_sum(sf);
                s2f = warp_sum(s2f);
                if (lane == 0) {
                    if (sf != 0) atomicAdd(&sums[g0].sin_f, sf);
                    if (s2f != 0) atomicAdd(&sums[g0].s2_f, s2f);
                }
            }
        } else {
            for (uint32_t i = i0 + lane; i < i1; i += 32) {
                const uint32_t g = lgid[i];
                if (!(gword[g] & kGwActive)) continue;
                const uint32_t v = list[i];
                const double x = sinv[v], sg = sigma[v];
                if (INTEGRAL) {
                    const unsigned long long q = (unsigned long long)sg;
                    if (x != 0) atomicAdd(&sums[g].sin_u, (unsigned long long)x);
                    if (q) atomicAdd(&sums[g].s2_u, q * q);
                } else {
                    if (x != 0) atomicAdd(&sums[g].sin_f, x);
                    if (sg != 0) atomicAdd(&sums[g].s2_f, sg * sg);
                }
            }
        }
    }
}

// Q = sum_in / mass - sum sigma^2 / mass^2, the host's operations of the
// single-graph loop, each rounded as written
__device__ __forceinline__ double batch_q(const GSum &S, double mass, int integral) {
    const double a = integral ? __ull2double_rn(S.sin_u) : S.sin_f;
    const double b = integral ? __ull2double_rn(S.s2_u) : S.s2_f;
    return __dsub_rn(__ddiv_rn(a, mass), __ddiv_rn(b, __dmul_rn(mass, mass)));
}

// One thread per graph: the accept / reject step of the single-graph loop
// (louvain.cu above), its buffer rotation and the sigma update flag.
__global__ void decide_kernel(uint32_t G, GSum *sums, const double *mass, double thr, int integral, uint32_t *gword,
                              double *curQ, uint32_t *loops, unsigned long long *iters, const uint32_t *gnnz,
                              const uint32_t *goff, BatchCtrl *ctrl, int set_cond, cudaGraphConditionalHandle cond) {
    const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
    int act = 0;
    unsigned long long edges = 0, verts = 0;
    if (g < G) {
        const uint32_t w = gword[g];
        if (w & kGwActive) {
            const GSum S = sums[g];
            sums[g] = GSum{0, 0, 0, 0};
            const double Q = batch_q(S, mass[g], integral);
            edges = gnnz[g];
            const uint32_t p = gw_p(w), nx = gw_n(w);
            const uint32_t after = 3u - p - nx;
            if (w & kGwFirst) {
                // first sweep: Q of the identity; always continue from the proposal
                curQ[g] = Q;
                gword[g] = gw_make(true, nx, after, p, false, true, p, nx);
                act = 1;
            } else {
                loops[g]++;
                if (__dsub_rn(Q, curQ[g]) > thr) {
                    curQ[g] = Q;
                    gword[g] = gw_make(true, nx, after, p, false, true, p, nx);
                    act = 1;
                } else {
                    iters[g] += loops[g];
                    gword[g] = gw_make(false, p, nx, gw_base(w), false, false, 0, 0);
                }
            }
        }
    }
    if (act) verts = goff[g + 1] - goff[g];
    const int a = __syncthreads_count(act);
    edges = warp_sum(edges);
    verts = warp_sum(verts);
    __shared__ unsigned long long es[32], vs[32];
    if ((threadIdx.x & 31) == 0) {
        es[threadIdx.x >> 5] = edges;
        vs[threadIdx.x >> 5] = verts;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long t = 0, tv = 0;
        for (unsigned i = 0; i < (blockDim.x >> 5); i++) {
            t += es[i];
            tv += vs[i];
        }
        if (a) atomicAdd(&ctrl->active, a);
        if (t) atomicAdd(&ctrl->edges, t);
        if (tv) atomicAdd(&ctrl->active_vertices, tv);
    }
    // the last block to finish flips the direction and, in a CUDA-graph loop,
    // decides whether the body runs again: not when no graph is active, the
    // launch's budget is used up or the lists should be compacted
    __shared__ bool last;
    __threadfence();
    if (threadIdx.x == 0) {
        unsigned int done = atomicAdd((unsigned int *)&ctrl->pad[0], 1u);
        last = done == gridDim.x - 1;
    }
    __syncthreads();
    if (last && threadIdx.x == 0) {
        __threadfence();
        ctrl->pad[0] = 0;
        ctrl->up ^= 1;
        ctrl->sweeps++;
        const int active = *(volatile int *)&ctrl->active;
        const unsigned long long av = *(volatile unsigned long long *)&ctrl->active_vertices;
        const long long left = --ctrl->budget;
        if (set_cond)
            cudaGraphSetConditional(cond, (active > 0 && left > 0 && 2 * av > ctrl->listed) ? 1u : 0u);
    }
}

// sigma += k moved, for graphs whose decision accepted the sweep
__global__ void sigma_update_batch_kernel(const uint32_t *list, const uint32_t *lgid, uint32_t L,
                                          const uint32_t *gword, const uint32_t *C0, const uint32_t *C1,
                                          const uint32_t *C2, const double *k, double *sigma, SweepAcc *acc) {
    unsigned moved = 0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < L; i += gridDim.x * blockDim.x) {
        const uint32_t w = gword[lgid[i]];
        if (!(w & kGwUpdate)) continue;
        const uint32_t v = list[i];
        const uint32_t f = gw_from(w), t = gw_to(w);
        const uint32_t a = (f == 0 ? C0 : f == 1 ? C1 : C2)[v];
        const uint32_t b = (t == 0 ? C0 : t == 1 ? C1 : C2)[v];
        if (a != b) {
            const double kv = k[v];
            atomicAdd(sigma + a, -kv);
            atomicAdd(sigma + b, kv);
            moved++;
        }
    }
    unsigned long long m = warp_sum((unsigned long long)moved);
    if ((threadIdx.x & 31) == 0 && m) atomicAdd(&acc->moved, m);
}

// final assignment of the phase: each graph's base buffer
__global__ void gather_final_kernel(uint32_t n, const uint32_t *gid, const uint32_t *gword, const uint32_t *C0,
                                    const uint32_t *C1, const uint32_t *C2, uint32_t *Cf) {
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
        const uint32_t b = gw_base(gword[gid[v]]);
        Cf[v] = (b == 0 ? C0 : b == 1 ? C1 : C2)[v];
    }
}

// graph offsets of the next level: the dense id of each graph's first vertex
__global__ void goff_remap_kernel(const uint32_t *goff, uint32_t G, const uint32_t *newid, uint32_t *goff_new) {
    uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g <= G) goff_new[g] = newid[goff[g]];
}

// graph-local community of every input vertex
__global__ void local_assign_kernel(uint32_t n0, const uint32_t *voff, uint32_t G, const uint32_t *goff_final,
                                    uint32_t *assign) {
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n0; v += gridDim.x * blockDim.x) {
        uint32_t lo = 0, hi = G;
        while (hi - lo > 1) {
            uint32_t mid = (lo + hi) >> 1;
            if (voff[mid] <= v) lo = mid;
            else hi = mid;
        }
        assign[v] -= goff_final[lo];
    }
}

// Compaction of a list to the entries of active graphs.  list == nullptr is the
// identity list [0, L); lgid == nullptr takes the graph of an entry from gid.
__global__ void list_flags_kernel(const uint32_t *list, const uint32_t *lgid, const uint32_t *gid, uint32_t L,
                                  const uint32_t *gword, uint32_t *flags) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < L; i += gridDim.x * blockDim.x) {
        const uint32_t v = list ? list[i] : i;
        const uint32_t g = lgid ? lgid[i] : gid[v];
        flags[i] = gword[g] & kGwActive;
    }
}

__global__ void list_scatter_kernel(const uint32_t *list, const uint32_t *lgid, const uint32_t *gid, uint32_t L,
                                    const uint32_t *flags, const uint32_t *pos, uint32_t *out, uint32_t *out_gid) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < L; i += gridDim.x * blockDim.x) {
        if (!flags[i]) continue;
        const uint32_t v = list ? list[i] : i;
        out[pos[i]] = v;
        out_gid[pos[i]] = lgid ? lgid[i] : gid[v];
    }
}

struct Idx12 {
    uint32_t v[kLightClasses + 1];
};
__global__ void gather_idx_kernel(const uint32_t *pos, Idx12 idx, int cnt, uint32_t *out) {
    if ((int)threadIdx.x < cnt) out[threadIdx.x] = pos[idx.v[threadIdx.x]];
}

// Keeps the entries of active graphs, in order.  The positions of the entries
// at the indices bounds[0..nb) map to out_bounds (bin offsets); the new length
// is out_bounds[nb].
void compact_list(const uint32_t *list, const uint32_t *lgid, const uint32_t *gid, uint32_t L, const uint32_t *gword,
                  uint32_t *out, uint32_t *out_gid, BatchWork &W, PrimWorkspace &pw, cudaStream_t s,
                  const uint32_t *bounds, int nb, uint32_t *out_bounds) {
    uint32_t *flags = W.flags.get(), *pos = W.pos.get();
    Idx12 idx = {};
    for (int b = 0; b < nb; b++) idx.v[b] = bounds[b];
    idx.v[nb] = L;
    if (L > 0) {
        list_flags_kernel<<<grid_n(L), 256, 0, s>>>(list, lgid, gid, L, gword, flags);
        MG_LAUNCH_CHECK();
        exclusive_scan<uint32_t>(flags, pos, L, pos + L, s, pw);
        list_scatter_kernel<<<grid_n(L), 256, 0, s>>>(list, lgid, gid, L, flags, pos, out, out_gid);
        MG_LAUNCH_CHECK();
        gather_idx_kernel<<<1, 32, 0, s>>>(pos, idx, nb + 1, flags);
        MG_LAUNCH_CHECK();
        MG_CUDA(cudaMemcpyAsync(out_bounds, flags, sizeof(uint32_t) * (nb + 1), cudaMemcpyDeviceToHost, s));
        MG_CUDA(cudaStreamSynchronize(s));
    } else {
        for (int b = 0; b <= nb; b++) out_bounds[b] = 0;
    }
}

// The active lists of a phase.
struct Lists {
    int cur = 0;          // buffers in use
    MoveLevel lvl;        // the level with the bins of the compacted list
    uint32_t vlen = 0;    // entries of the vertex list
};

// Rebuild both lists from the current ones (or, at the start of a phase,
// from the level's bins and the identity).
void rebuild_lists(mg_ctx *ctx, BatchWork &W, const MoveLevel &full, Lists &Ls, bool from_level, uint32_t n,
                   cudaStream_t s) {
    const int nxt = from_level ? Ls.cur : Ls.cur ^ 1;
    const uint32_t *gid = W.gid.get(), *gword = W.gword.get();
    PrimWorkspace &pw = ctx->cws.prim;
    // light classes (0-12); the heavy classes keep the level's own lists
    const Bins &src = from_level ? full.bins : Ls.lvl.bins;
    uint32_t bounds[kLightClasses + 1], nb[kLightClasses + 1];
    for (int b = 0; b < kLightClasses; b++) bounds[b] = src.offset[b];
    const uint32_t L = src.offset[kLightClasses];
    compact_list(from_level ? ctx->mws.perm.get() : W.lperm[Ls.cur].get(), from_level ? nullptr : W.lpgid[Ls.cur].get(),
                 gid, L, gword, W.lperm[nxt].get(), W.lpgid[nxt].get(), W, pw, s, bounds, kLightClasses, nb);
    uint8_t shapes[kLightClasses];
    for (int b = 0; b < kLightClasses; b++) shapes[b] = Ls.lvl.shape[b];
    Ls.lvl = full;
    for (int b = 0; b < kLightClasses; b++) {
        Ls.lvl.bins.offset[b] = nb[b];
        Ls.lvl.bins.size[b] = nb[b + 1] - nb[b];
        if (!from_level) Ls.lvl.shape[b] = shapes[b];  // a phase keeps the shapes tuned at its start
    }
    Ls.lvl.bins.offset[kLightClasses] = nb[kLightClasses];
    // vertices in id order
    uint32_t vb[1];
    compact_list(from_level ? nullptr : W.lvert[Ls.cur].get(), from_level ? nullptr : W.lvgid[Ls.cur].get(), gid,
                 from_level ? n : Ls.vlen, gword, W.lvert[nxt].get(), W.lvgid[nxt].get(), W, pw, s, nullptr, 0, vb);
    Ls.vlen = vb[0];
    Ls.cur = nxt;
}

struct Body {
    const GraphView *g;
    const MoveLevel *lvl;  // bins of the compacted list
    SweepParams sp;
    BatchSweep bs;
    const uint32_t *vlist, *vgid;  // vertex list
    uint32_t vlen;
    const uint32_t *goff;  // first vertex of each graph in the level
    uint32_t G;
    double thr;
    const double *k;
    double *sigma;
};

// one iteration: sweep, per-graph sums, decisions, sigma updates
void run_body(mg_ctx *ctx, mg_batch *b, const Body &B, cudaStream_t s, int set_cond, cudaGraphConditionalHandle h) {
    BatchWork &W = b->work;
    move_sweep_batch(*B.g, *B.lvl, ctx->mws, B.sp, B.bs, B.k, B.sigma, s);
    const unsigned gs = grid_n(ceil_div(B.vlen, kSumVPT), 256, 148ull * 32);
    if (B.sp.integral)
        gsum_kernel<1><<<gs, 256, 0, s>>>(B.vlist, B.vgid, B.vlen, W.gword.get(), W.sinv.get(), B.sigma,
                                          W.sums.get(), W.ctrl.get());
    else
        gsum_kernel<0><<<gs, 256, 0, s>>>(B.vlist, B.vgid, B.vlen, W.gword.get(), W.sinv.get(), B.sigma,
                                          W.sums.get(), W.ctrl.get());
    MG_LAUNCH_CHECK();
    decide_kernel<<<(unsigned)ceil_div(B.G, 256), 256, 0, s>>>(
        B.G, W.sums.get(), W.gmass.get(), B.thr, B.sp.integral, W.gword.get(), W.curQ.get(), W.loops.get(),
        W.iters.get(), W.gnnz.get(), B.goff, W.ctrl.get(), set_cond, h);
    MG_LAUNCH_CHECK();
    sigma_update_batch_kernel<<<grid_n(B.vlen), 256, 0, s>>>(B.vlist, B.vgid, B.vlen, W.gword.get(), B.bs.C[0],
                                                             B.bs.C[1], B.bs.C[2], B.k, B.sigma,
                                                             ctx->mws.acc.get());
    MG_LAUNCH_CHECK();
}

// Iterations of one phase as a CUDA graph with a conditional while loop.
struct PhaseGraph {
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    unsigned long long body_launches = 0;
    ~PhaseGraph() {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
    }
};

void build_phase_graph(mg_ctx *ctx, mg_batch *b, const Body &B, cudaStream_t s, PhaseGraph &pg) {
    MG_CUDA(cudaGraphCreate(&pg.graph, 0));
    cudaGraphConditionalHandle h;
    MG_CUDA(cudaGraphConditionalHandleCreate(&h, pg.graph, 1u, cudaGraphCondAssignDefault));
    cudaGraphNodeParams cp = {};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = h;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaGraphNode_t node;
    MG_CUDA(cudaGraphAddNode(&node, pg.graph, nullptr, 0, &cp));
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    const unsigned long long l0 = g_kernel_launches;
    MG_CUDA(cudaStreamBeginCaptureToGraph(s, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
    try {
        run_body(ctx, b, B, s, 1, h);
    } catch (...) {
        cudaGraph_t dummy;
        cudaStreamEndCapture(s, &dummy);
        throw;
    }
    MG_CUDA(cudaStreamEndCapture(s, &body));
    pg.body_launches = g_kernel_launches - l0;
    g_kernel_launches = l0;  // counted per execution below
    MG_CUDA(cudaGraphInstantiate(&pg.exec, pg.graph, 0));
}

}  // namespace

void batch_run(mg_batch *b, const mg_run_opts &o, int flags, mg_batch_result &res, const GraphDoneFn *done) {
    mg_ctx *ctx = b->ctx;
    ctx_prepare(ctx);
    cudaStream_t s = ctx->stream;
    BatchWork &W = b->work;
    const uint32_t G = b->graphs;
    const uint32_t n0 = b->u.n;
    const int version = o.version == 1 ? 1 : 2;
    const double thr = o.threshold;
    res = mg_batch_result();
    res.graphs = G;
    res.voff = b->voff;
    res.per.assign(G, mg_batch_graph_summary{});
    res.assignment.assign(n0, 0);
    mg_summary &S = res.sum;
    // graphs without edges keep the identity (as mg_louvain_run does)
    std::vector<uint8_t> alive(G, 0);
    int integral = 1;
    for (uint32_t g = 0; g < G; g++) {
        const uint32_t ng = b->voff[g + 1] - b->voff[g];
        const uint64_t eg = b->eoff[g + 1] - b->eoff[g];
        res.per[g].n = ng;
        res.per[g].nnz = eg;
        res.per[g].communities = ng;
        alive[g] = ng > 0 && eg > 0 && b->mass[g] > 0;
        if (alive[g]) integral &= b->integral[g];
        if (alive[g] && o.precision == MG_PREC_INT64)
            MG_CHECK(b->integral[g] && b->mass[g] < 2147483648.0, MG_ERR_UNSUPPORTED,
                     "int64 precision needs integral weights with total below 2^31");
    }
    // device state
    uint32_t *C[3] = {ctx->C[0].ensure(n0 + 1), ctx->C[1].ensure(n0 + 1), ctx->C[2].ensure(n0 + 1)};
    uint32_t *Cd = ctx->Cd.ensure(n0 + 1);
    uint32_t *assign = ctx->assign.ensure(n0 + 1);
    double *k = ctx->k.ensure(n0 + 1);
    double *sigma = ctx->sigma.ensure(n0 + 1);
    uint32_t *gid = W.gid.ensure(n0 + 1);
    uint32_t *Cf = W.Cf.ensure(n0 + 1);
    for (int i = 0; i < 2; i++) {
        W.lperm[i].ensure(n0 + 1);
        W.lpgid[i].ensure(n0 + 1);
        W.lvert[i].ensure(n0 + 1);
        W.lvgid[i].ensure(n0 + 1);
    }
    W.flags.ensure(n0 + 1);
    W.pos.ensure(n0 + 1);
    W.sinv.ensure(n0 + 1);
    uint32_t *goff = W.goff.ensure(G + 1);
    uint32_t *goff_new = W.goff_new.ensure(G + 1);
    uint32_t *goff0 = W.goff0.ensure(G + 1);
    W.gword.ensure(G);
    W.gnnz.ensure(G);
    W.loops.ensure(G);
    W.curQ.ensure(G);
    W.sums.ensure(G);
    double *gmass = W.gmass.ensure(G);
    GainK *gk = W.gk.ensure(G);
    unsigned long long *iters = W.iters.ensure(G);
    BatchCtrl *ctrl = W.ctrl.ensure(1);
    if (!W.h_ctrl) MG_CUDA(cudaMallocHost(&W.h_ctrl, sizeof(BatchCtrl)));
    uint8_t *alive_d = W.alive.ensure(G);
    {
        std::vector<GainK> hk(G);
        for (uint32_t g = 0; g < G; g++) hk[g] = gain_constants(alive[g] ? b->mass[g] : 1.0);
        MG_CUDA(cudaMemcpyAsync(gk, hk.data(), sizeof(GainK) * G, cudaMemcpyHostToDevice, s));
        MG_CUDA(cudaMemcpyAsync(gmass, b->mass.data(), sizeof(double) * G, cudaMemcpyHostToDevice, s));
        MG_CUDA(cudaMemcpyAsync(goff, b->voff.data(), sizeof(uint32_t) * (G + 1), cudaMemcpyHostToDevice, s));
        MG_CUDA(cudaMemcpyAsync(goff0, b->voff.data(), sizeof(uint32_t) * (G + 1), cudaMemcpyHostToDevice, s));
        MG_CUDA(cudaMemsetAsync(iters, 0, sizeof(unsigned long long) * G, s));
        MG_CUDA(cudaMemsetAsync(ctrl, 0, sizeof(BatchCtrl), s));
    }
    if (n0 > 0) fill_identity(assign, n0, s);
    std::vector<uint32_t> hgoff(b->voff.begin(), b->voff.end()), hgoff_new(G + 1);
    std::vector<double> hq(G), Qh(G, 0.0), Qold(G, -1.0);
    std::vector<int> phases(G, 0);
    // results handed out early (done callback): graphs without edges now,
    // the others when their run ends
    std::vector<unsigned long long> hit(G);
    std::vector<uint32_t> tmp_assign;
    if (done) {
        for (uint32_t g = 0; g < G; g++) {
            if (alive[g]) continue;
            tmp_assign.resize(res.per[g].n);
            for (uint32_t v = 0; v < res.per[g].n; v++) tmp_assign[v] = v;
            (*done)(g, res.per[g], tmp_assign.data());
        }
    }

    const unsigned long long launches0 = g_kernel_launches;
    W.h_ctrl->sweeps = 0;
    MG_CUDA(cudaEventRecord(ctx->ev[2], s));
    GraphView cur = b->u.view();
    int lvl_out = 0;
    int phase = 0;
    MoveLevel mlv;
    SweepParams sp;
    sp.version = version;
    sp.precision = o.precision;
    sp.integral = integral;
    const bool use_graph = (flags & MG_BATCH_GRAPHS) != 0;
    int any_alive = 0;
    for (uint32_t g = 0; g < G; g++) any_alive |= alive[g];

    while (phase < o.max_phases && any_alive) {
        const uint32_t n = cur.n;
        for (uint32_t g = 0; g < G; g++)
            if (alive[g]) {
                res.per[g].levels++;
                Qold[g] = Qh[g];
            }
        S.levels++;
        MG_CUDA(cudaEventRecord(ctx->ev[0], s));
        // level setup: graph of every vertex, entries per graph, k, sigma, C0
        gid_fill_kernel<<<grid_n(n), 256, 0, s>>>(goff, G, n, gid);
        MG_LAUNCH_CHECK();
        gnnz_kernel<<<(unsigned)ceil_div(G, 256), 256, 0, s>>>(cur.off, goff, G, W.gnnz.get());
        MG_LAUNCH_CHECK();
        MG_CUDA(cudaMemcpyAsync(alive_d, alive.data(), G, cudaMemcpyHostToDevice, s));
        phase_init_kernel<<<(unsigned)ceil_div(G, 256), 256, 0, s>>>(alive_d, G, W.gword.get(), W.sums.get(),
                                                                     W.loops.get(), ctrl);
        MG_LAUNCH_CHECK();
        level_init(cur, k, sigma, C[0], s);
        move_prepare_level(cur, mlv, ctx->mws, s);
        sweep_reset_acc(ctx->mws, s);
        // active lists of the phase
        Lists Ls;
        rebuild_lists(ctx, W, mlv, Ls, true, n, s);
        Body B;
        B.g = &cur;
        B.sp = sp;
        B.bs.gid = gid;
        B.bs.gword = W.gword.get();
        B.bs.gk = gk;
        B.bs.C[0] = C[0];
        B.bs.C[1] = C[1];
        B.bs.C[2] = C[2];
        B.bs.sinv = W.sinv.get();
        B.bs.up = &ctrl->up;
        B.goff = goff;
        B.G = G;
        B.thr = thr;
        B.k = k;
        B.sigma = sigma;
        auto use_lists = [&]() {
            B.lvl = &Ls.lvl;
            B.bs.perm = W.lperm[Ls.cur].get();
            B.bs.pgid = W.lpgid[Ls.cur].get();
            B.vlist = W.lvert[Ls.cur].get();
            B.vgid = W.lvgid[Ls.cur].get();
            B.vlen = Ls.vlen;
            W.h_ctrl->listed = Ls.vlen;
            MG_CUDA(cudaMemcpyAsync(&ctrl->listed, &W.h_ctrl->listed, sizeof(unsigned long long),
                                    cudaMemcpyHostToDevice, s));
        };
        use_lists();
        // shapes of the light classes (autotuner): the timing runs write what
        // the first sweep of the phase writes
        move_tune_batch(cur, Ls.lvl, ctx->mws, sp, B.bs, k, sigma, s);
        // iterate until every graph has rejected a sweep.  The first sweep
        // after the lists change runs as plain launches (it also sets up the
        // launch shapes); the rest, with MG_BATCH_GRAPHS, as CUDA-graph loops.
        std::unique_ptr<PhaseGraph> pg;
        unsigned long long graph_sweeps0 = 0;
        auto retire_graph = [&]() {
            if (pg) g_kernel_launches += pg->body_launches * (W.h_ctrl->sweeps - graph_sweeps0);
            pg.reset();
        };
        bool plain = true;
        B.sp.agg = 0;  // the phase's first sweep: every community is one vertex
        B.sp.split = sweep_split(ctx->mws, 0);
        while (true) {
            if (use_graph && !plain) {
                if (!pg) {
                    pg.reset(new PhaseGraph());
                    build_phase_graph(ctx, b, B, s, *pg);
                    graph_sweeps0 = W.h_ctrl->sweeps;
                }
                W.h_ctrl->budget = kGraphBudget;
                MG_CUDA(cudaMemcpyAsync(&ctrl->budget, &W.h_ctrl->budget, sizeof(long long), cudaMemcpyHostToDevice,
                                        s));
                MG_CUDA(cudaGraphLaunch(pg->exec, s));
            } else {
                run_body(ctx, b, B, s, 0, cudaGraphConditionalHandle());
            }
            plain = false;
            B.sp.agg = 1;  // later sweeps: communities repeat among neighbours
            B.sp.split = sweep_split(ctx->mws, 1);
            MG_CUDA(cudaMemcpyAsync(W.h_ctrl, ctrl, sizeof(BatchCtrl), cudaMemcpyDeviceToHost, s));
            MG_CUDA(cudaStreamSynchronize(s));
            if (W.h_ctrl->active == 0) break;
            if (2 * W.h_ctrl->active_vertices <= W.h_ctrl->listed) {
                retire_graph();
                rebuild_lists(ctx, W, mlv, Ls, false, n, s);
                use_lists();
                plain = true;
            }
        }
        retire_graph();
        SweepAcc hacc;
        MG_CUDA(cudaMemcpyAsync(&hacc, ctx->mws.acc.get(), sizeof(SweepAcc), cudaMemcpyDeviceToHost, s));
        MG_CUDA(cudaMemcpyAsync(hq.data(), W.curQ.get(), sizeof(double) * G, cudaMemcpyDeviceToHost, s));
        MG_CUDA(cudaEventRecord(ctx->ev[1], s));
        MG_CUDA(cudaStreamSynchronize(s));
        MG_CHECK(hacc.overflow == 0, MG_ERR_UNSUPPORTED, "local move: a cluster hash segment overflowed");
        float ms = 0;
        MG_CUDA(cudaEventElapsedTime(&ms, ctx->ev[0], ctx->ev[1]));
        S.seconds_local_move += ms * 1e-3;
        if (phase == 0) S.phase0_seconds = ms * 1e-3;
        S.distinct_pairs += hacc.distinct;
        // final assignments -> dense relabel over the union -> compose
        MG_CUDA(cudaEventRecord(ctx->ev[0], s));
        gather_final_kernel<<<grid_n(n), 256, 0, s>>>(n, gid, W.gword.get(), C[0], C[1], C[2], Cf);
        MG_LAUNCH_CHECK();
        const uint32_t nn = relabel_dense(Cf, n, Cd, ctx->cws, s);
        goff_remap_kernel<<<(unsigned)ceil_div(G + 1, 256), 256, 0, s>>>(goff, G, ctx->cws.newid.get(), goff_new);
        MG_LAUNCH_CHECK();
        gather_compose(assign, Cd, n0, s);
        MG_CUDA(cudaMemcpyAsync(hgoff_new.data(), goff_new, sizeof(uint32_t) * (G + 1), cudaMemcpyDeviceToHost, s));
        MG_CUDA(cudaStreamSynchronize(s));
        any_alive = 0;
        std::vector<uint32_t> fin;
        for (uint32_t g = 0; g < G; g++) {
            if (!alive[g]) continue;
            Qh[g] = hq[g];
            res.per[g].communities = hgoff_new[g + 1] - hgoff_new[g];
            if (Qh[g] - Qold[g] <= thr) {
                alive[g] = 0;
                phases[g] = phase;
                fin.push_back(g);
            } else {
                any_alive = 1;
            }
        }
        if (done && !fin.empty()) {
            // the composed assignment of a finished graph is final; its local
            // ids are offsets from the graph's first community
            MG_CUDA(cudaMemcpyAsync(hit.data(), iters, sizeof(unsigned long long) * G, cudaMemcpyDeviceToHost, s));
            for (uint32_t g : fin)
                if (res.per[g].n)
                    MG_CUDA(cudaMemcpyAsync(res.assignment.data() + b->voff[g], assign + b->voff[g],
                                            sizeof(uint32_t) * res.per[g].n, cudaMemcpyDeviceToHost, s));
            MG_CUDA(cudaStreamSynchronize(s));
            for (uint32_t g : fin) {
                uint32_t *a = res.assignment.data() + b->voff[g];
                for (uint32_t v = 0; v < res.per[g].n; v++) a[v] -= hgoff_new[g];
                mg_batch_graph_summary P = res.per[g];
                P.modularity = Qh[g];
                P.phases = phases[g];
                P.iterations = hit[g];
                (*done)(g, P, a);
            }
        }
        if (!any_alive) {
            MG_CUDA(cudaEventRecord(ctx->ev[1], s));
            MG_CUDA(cudaEventSynchronize(ctx->ev[1]));
            MG_CUDA(cudaEventElapsedTime(&ms, ctx->ev[0], ctx->ev[1]));
            S.seconds_coarsen += ms * 1e-3;
            std::swap(goff, goff_new);  // the assignment is in the relabelled ids
            break;
        }
        coarsen_level(cur, Cd, nn, integral, ctx->lv[lvl_out], ctx->cws, s, nullptr,
                      ctx->mws.coarsen_combine == MG_COMBINE_ON);
        MG_CUDA(cudaEventRecord(ctx->ev[1], s));
        MG_CUDA(cudaEventSynchronize(ctx->ev[1]));
        MG_CUDA(cudaEventElapsedTime(&ms, ctx->ev[0], ctx->ev[1]));
        S.seconds_coarsen += ms * 1e-3;
        cur = ctx->lv[lvl_out].view();
        lvl_out ^= 1;
        std::swap(goff, goff_new);
        hgoff.swap(hgoff_new);
        phase++;
    }
    for (uint32_t g = 0; g < G; g++)
        if (alive[g]) phases[g] = phase;  // stopped by max_phases
    // graph-local assignment
    if (n0 > 0) {
        local_assign_kernel<<<grid_n(n0), 256, 0, s>>>(n0, goff0, G, goff, assign);
        MG_LAUNCH_CHECK();
    }
    MG_CUDA(cudaEventRecord(ctx->ev[3], s));
    MG_CUDA(cudaMemcpyAsync(hit.data(), iters, sizeof(unsigned long long) * G, cudaMemcpyDeviceToHost, s));
    MG_CUDA(cudaMemcpyAsync(W.h_ctrl, ctrl, sizeof(BatchCtrl), cudaMemcpyDeviceToHost, s));
    if (n0 > 0)
        MG_CUDA(cudaMemcpyAsync(res.assignment.data(), assign, sizeof(uint32_t) * n0, cudaMemcpyDeviceToHost, s));
    MG_CUDA(cudaStreamSynchronize(s));
    float ms = 0;
    MG_CUDA(cudaEventElapsedTime(&ms, ctx->ev[2], ctx->ev[3]));
    S.seconds_total = ms * 1e-3;
    S.sweeps = W.h_ctrl->sweeps;
    S.edges_swept = W.h_ctrl->edges;
    S.kernel_launches = g_kernel_launches - launches0;
    for (uint32_t g = 0; g < G; g++) {
        mg_batch_graph_summary &P = res.per[g];
        P.modularity = Qh[g];
        P.phases = phases[g];
        P.iterations = hit[g];
        S.iterations += (int)hit[g];
    }
    if (done)  // graphs stopped by max_phases
        for (uint32_t g = 0; g < G; g++)
            if (alive[g]) (*done)(g, res.per[g], res.assignment.data() + b->voff[g]);
}

}  // namespace mg
