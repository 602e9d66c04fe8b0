// louvain.cu -- the phase / iteration loop.
//
// Control flow of louvain::run (src/louvain/louvain.cu:1401-1715):
//   Q_host = 0, Q_old = -1
//   while phase < max_phases and Q_host - Q_old > threshold:
//     Q_old = Q_host; C = identity; k = row sums; sigma = k; Q = Q(C)
//     cur = Q - 1; up = true
//     while Q - cur > threshold:
//       cur = Q; C_new = move(C, up); up = !up; sigma += delta(C -> C_new)
//       Q = Q(C_new); accept C_new if Q - cur > threshold, else Q = cur
//     Q_host = Q; stop if Q_host - Q_old <= threshold; else coarsen by C
//
// Here each sweep over the edges does double duty: while it proposes C_next
// from the pending assignment P it also sums the internal weight of P, so
// Q(P) comes out of the same pass (plus a pass over sigma).  The decision on
// P is taken after that sweep: accepted -> P becomes the base, C_next the new
// pending assignment; rejected -> the base is final and C_next is dropped.
// The reference needs a move pass and a separate modularity pass per
// iteration; this loop runs one edge pass per iteration plus one at the end.
#include <chrono>
#include <cstdio>

#include "handles.cuh"

namespace mg {

namespace {

struct Timer {
    cudaEvent_t a, b;
    cudaStream_t s;
    Timer(cudaEvent_t a_, cudaEvent_t b_, cudaStream_t s_) : a(a_), b(b_), s(s_) { MG_CUDA(cudaEventRecord(a, s)); }
    double stop_sync() {
        MG_CUDA(cudaEventRecord(b, s));
        MG_CUDA(cudaEventSynchronize(b));
        float ms = 0;
        MG_CUDA(cudaEventElapsedTime(&ms, a, b));
        return ms * 1e-3;
    }
};

// Device time of the sweep's kernels (events ev[4] -> ev[5], already
// complete) and its algorithmic bytes: 12 per edge (column, weight, community
// of the neighbour), 24 per vertex (offset, community, k_i, sigma of the own
// community, new community), 8 per distinct candidate (sigma of the candidate).
void account_sweep(mg_ctx *ctx, const GraphView &g, const SweepAcc &acc, mg_summary &S) {
    MG_CHECK(acc.overflow == 0, MG_ERR_UNSUPPORTED, "local move: a cluster hash segment overflowed");
    float ms = 0;
    MG_CUDA(cudaEventElapsedTime(&ms, ctx->ev[4], ctx->ev[5]));
    S.seconds_sweep_kernels += ms * 1e-3;
    S.sweep_bytes += 12.0 * (double)g.nnz + 24.0 * (double)g.n + 8.0 * (double)acc.distinct;
}

void print_phase_header(int phase) {
    printf("----------------------------------------\n");
    printf("Phase %d\n", phase);
    printf("| %-10s | %-10s | %-10s | %-10s | %-10s |\n", "Loop", "Q", "dQ", "time(s)", "time(ms)");
    printf("|------------|------------|------------|------------|------------|\n");
}

}  // namespace

// Host copy of the graph a level works on (opt-in: keep_levels >= 2).
void keep_level_csr(const GraphView &cur, mg_result &res, cudaStream_t s) {
    res.level_csr.emplace_back();
    mg_result::LevelCsr &L = res.level_csr.back();
    L.off.resize((size_t)cur.n + 1);
    L.col.resize(cur.nnz);
    L.w.assign(cur.nnz, 1.0);
    MG_CUDA(cudaMemcpyAsync(L.off.data(), cur.off, sizeof(uint32_t) * ((size_t)cur.n + 1), cudaMemcpyDeviceToHost, s));
    if (cur.nnz) MG_CUDA(cudaMemcpyAsync(L.col.data(), cur.col, sizeof(uint32_t) * cur.nnz, cudaMemcpyDeviceToHost, s));
    if (cur.nnz && cur.wk == WK_F64) {
        MG_CUDA(cudaMemcpyAsync(L.w.data(), cur.w, sizeof(double) * cur.nnz, cudaMemcpyDeviceToHost, s));
    } else if (cur.nnz && cur.wk == WK_F32) {
        std::vector<float> w32(cur.nnz);
        MG_CUDA(cudaMemcpyAsync(w32.data(), cur.w, sizeof(float) * cur.nnz, cudaMemcpyDeviceToHost, s));
        MG_CUDA(cudaStreamSynchronize(s));
        for (uint64_t e = 0; e < cur.nnz; e++) L.w[e] = w32[e];
    } else if (cur.nnz && cur.wk == WK_U32) {
        std::vector<uint32_t> wi(cur.nnz);
        MG_CUDA(cudaMemcpyAsync(wi.data(), cur.w, sizeof(uint32_t) * cur.nnz, cudaMemcpyDeviceToHost, s));
        MG_CUDA(cudaStreamSynchronize(s));
        for (uint64_t e = 0; e < cur.nnz; e++) L.w[e] = wi[e];
    }
}

void louvain_run(mg_ctx *ctx, const mg_graph *g, const mg_run_opts &o, mg_result &res) {
    ctx_prepare(ctx);
    cudaStream_t s = ctx->stream;
    const uint32_t n0 = g->n;
    const double mass = g->mass;
    const int integral = g->integral;
    const int version = o.version == 1 ? 1 : 2;  // version 0 behaves as 2 on one GPU
    const double thr = o.threshold;
    const bool verbose = o.verbose || ctx->verbose;
    res = mg_result();
    res.n0 = n0;
    res.assignment.assign(n0, 0);
    mg_summary &S = res.sum;
    if (n0 == 0 || g->nnz == 0 || mass <= 0) {
        for (uint32_t v = 0; v < n0; v++) res.assignment[v] = v;
        S.communities = n0;
        return;
    }
    uint32_t *C[3] = {ctx->C[0].ensure(n0 + 1), ctx->C[1].ensure(n0 + 1), ctx->C[2].ensure(n0 + 1)};
    uint32_t *Cd = ctx->Cd.ensure(n0 + 1);
    uint32_t *assign = ctx->assign.ensure(n0 + 1);
    double *k = ctx->k.ensure(n0 + 1);
    double *sigma = ctx->sigma.ensure(n0 + 1);
    SweepAcc &hacc = *ctx->h_acc;
    fill_identity(assign, n0, s);

    const unsigned long long launches0 = g_kernel_launches;
    MG_CUDA(cudaEventRecord(ctx->ev[2], s));
    GraphView cur = g->view();
    int lvl_out = 0;
    double Qh = 0, Qold = -1;
    int phase = 0;
    MoveLevel mlv;
    SweepParams sp;
    sp.version = version;
    sp.precision = o.precision;
    sp.mass = mass;
    sp.integral = integral;
    uint32_t communities = n0;

    while (phase < o.max_phases && (Qh - Qold) > thr) {
        Qold = Qh;
        const uint32_t n = cur.n;
        res.level_sizes.push_back(n);
        S.levels++;
        if (o.keep_levels >= 2) keep_level_csr(cur, res, s);
        if (verbose) print_phase_header(phase);
        double phase_lm = 0;
        Timer tp(ctx->ev[0], ctx->ev[1], s);
        level_init(cur, k, sigma, C[0], s);
        move_prepare_level(cur, mlv, ctx->mws, s);
        int base = 0, pend = 1;
        // first sweep: P = identity (base), proposes C[1]; yields Q0
        sp.up = 1;
        sp.agg = 0;
        sp.split = sweep_split(ctx->mws, 0);
        sp.first = ctx->mws.first_sweep_kernels && cur.sorted_rows;
        // shapes of the light classes from the tuning table; classes missing
        // from it are timed on the level's second sweep, which is more like
        // the rest of the level than the first (every community one vertex)
        move_tune(cur, mlv, ctx->mws, sp, C[base], C[pend], k, sigma, s, false);
        sweep_reset_acc(ctx->mws, s);
        sigma_sumsq(sigma, n, integral, ctx->mws, s);
        MG_CUDA(cudaEventRecord(ctx->ev[4], s));
        move_sweep(cur, mlv, ctx->mws, sp, C[base], C[pend], k, sigma, s);
        MG_CUDA(cudaEventRecord(ctx->ev[5], s));
        MG_CUDA(cudaMemcpyAsync(&hacc, ctx->mws.acc.get(), sizeof(SweepAcc), cudaMemcpyDeviceToHost, s));
        double lm = tp.stop_sync();
        phase_lm += lm;
        account_sweep(ctx, cur, hacc, S);
        S.sweeps++;
        S.edges_swept += cur.nnz;
        S.distinct_pairs += hacc.distinct;
        if (phase == 0) {
            S.phase0_edges_swept += cur.nnz;
        }
        double curQ = modularity_from_acc(hacc, mass, integral);
        res.trace.insert(res.trace.end(), {(double)phase, 0.0, curQ, 0.0});
        if (verbose) printf("| %-10d | %-10f | %-10f | %-10f | %-10f |\n", 0, curQ, 0., 0., 0.);
        sigma_update(C[base], C[pend], k, sigma, n, ctx->mws, s);
        int loop = 0;
        while (true) {
            sp.up = !sp.up;
            // combine equal communities in the warp once they repeat: fewer
            // than half of the last sweep's edges were distinct candidates
            sp.first = 0;
            sp.agg = 2 * hacc.distinct < cur.nnz;
            sp.split = sweep_split(ctx->mws, sp.agg);
            const int next = 3 - base - pend;
            // autotuner: its timing runs write the proposal this sweep writes
            if (loop == 0) move_tune(cur, mlv, ctx->mws, sp, C[pend], C[next], k, sigma, s, true);
            Timer ti(ctx->ev[0], ctx->ev[1], s);
            sweep_reset_acc(ctx->mws, s);
            sigma_sumsq(sigma, n, integral, ctx->mws, s);
            MG_CUDA(cudaEventRecord(ctx->ev[4], s));
            move_sweep(cur, mlv, ctx->mws, sp, C[pend], C[next], k, sigma, s);
            MG_CUDA(cudaEventRecord(ctx->ev[5], s));
            MG_CUDA(cudaMemcpyAsync(&hacc, ctx->mws.acc.get(), sizeof(SweepAcc), cudaMemcpyDeviceToHost, s));
            double dt = ti.stop_sync();
            phase_lm += dt;
            account_sweep(ctx, cur, hacc, S);
            S.sweeps++;
            S.edges_swept += cur.nnz;
            S.distinct_pairs += hacc.distinct;
            if (phase == 0) S.phase0_edges_swept += cur.nnz;
            loop++;
            const double Qp = modularity_from_acc(hacc, mass, integral);
            if ((Qp - curQ) > thr) {
                res.trace.insert(res.trace.end(), {(double)phase, (double)loop, Qp, Qp - curQ});
                if (verbose) printf("| %-10d | %-10f | %-10f | %-10f | %-10f |\n", loop, Qp, Qp - curQ, dt, dt * 1e3);
                curQ = Qp;
                sigma_update(C[pend], C[next], k, sigma, n, ctx->mws, s);
                base = pend;
                pend = next;
            } else {
                res.trace.insert(res.trace.end(), {(double)phase, (double)loop, curQ, 0.0});
                if (verbose) printf("| %-10d | %-10f | %-10f | %-10f | %-10f |\n", loop, curQ, 0., dt, dt * 1e3);
                break;
            }
        }
        S.iterations += loop;  // the reference's loop count (moves evaluated)
        S.seconds_local_move += phase_lm;
        if (phase == 0) S.phase0_seconds = phase_lm;
        if (verbose) {
            printf("Main loop total execution time: %f s, %f ms\n", phase_lm, phase_lm * 1e3);
            printf("The average execution time per loop: %f s, %f ms\n", phase_lm / (loop + 1),
                   phase_lm * 1e3 / (loop + 1));
        }
        Qh = curQ;
        // dense relabel of the final assignment of this phase, composed into
        // the assignment of the input vertices
        Timer tc(ctx->ev[0], ctx->ev[1], s);
        const uint32_t nn = relabel_dense(C[base], n, Cd, ctx->cws, s);
        gather_compose(assign, Cd, n0, s);
        if (o.keep_levels) {
            res.level_maps.emplace_back(n);
            MG_CUDA(cudaMemcpyAsync(res.level_maps.back().data(), Cd, sizeof(uint32_t) * n, cudaMemcpyDeviceToHost, s));
        }
        communities = nn;
        if ((Qh - Qold) <= thr) {
            S.seconds_coarsen += tc.stop_sync();
            break;
        }
        coarsen_level(cur, Cd, nn, integral, ctx->lv[lvl_out], ctx->cws, s, nullptr,
                      coarsen_combine(ctx->mws, hacc.distinct, cur.nnz));
        double ct = tc.stop_sync();
        S.seconds_coarsen += ct;
        if (verbose) printf("Coarsen graph execution time: %f s, %f ms\n", ct, ct * 1e3);
        cur = ctx->lv[lvl_out].view();
        lvl_out ^= 1;
        phase++;
    }
    MG_CUDA(cudaEventRecord(ctx->ev[3], s));
    MG_CUDA(cudaMemcpyAsync(res.assignment.data(), assign, sizeof(uint32_t) * n0, cudaMemcpyDeviceToHost, s));
    MG_CUDA(cudaStreamSynchronize(s));
    float ms = 0;
    MG_CUDA(cudaEventElapsedTime(&ms, ctx->ev[2], ctx->ev[3]));
    S.kernel_launches = g_kernel_launches - launches0;
    S.seconds_total = ms * 1e-3;
    S.modularity = Qh;
    S.phases = phase;
    S.communities = communities;
    if (verbose) {
        printf("----------------------------------------\n");
        printf("Total time for clustering   : %f s\n", S.seconds_local_move);
        printf("Total time for coarsen graph: %f s\n", S.seconds_coarsen);
        printf("TOTAL TIME                  : %f s\n", S.seconds_total);
    }
}

}  // namespace mg
