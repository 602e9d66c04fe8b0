// local_move_batch.cu -- the local-move sweep over a batch of graphs packed as
// one disjoint union.  Same kernels as the single-graph sweep, instantiated
// with per-vertex graph lookups: the graph's control word picks the
// assignment buffers it reads and writes (graphs sit at different points of
// their accept / reject sequence), its gain constants come from its own mass,
// vertices of inactive graphs are skipped, and sum_in is written per vertex so
// that it can be summed per graph.
#include "lm_kernels.cuh"

namespace mg {

using namespace lmk;

namespace {
LMArgs batch_args(const GraphView &g, MoveWorkspace &ws, const SweepParams &p, const BatchSweep &b, const double *k,
                  const double *sigma) {
    LMArgs A = {};
    A.off = g.off;
    A.col = g.col;
    A.w = g.w;
    A.k = k;
    A.sigma = sigma;
    A.perm = b.perm;
    A.pgid = b.pgid;
    A.integral = p.integral;
    A.agg = p.agg;
    A.split = p.split;
    A.acc = ws.acc.ensure(1);
    A.gid = b.gid;
    A.gword = b.gword;
    A.gk = b.gk;
    A.Cb0 = b.C[0];
    A.Cb1 = b.C[1];
    A.Cb2 = b.C[2];
    A.sinv = b.sinv;
    A.up_dev = b.up;
    return A;
}
}  // namespace

void move_sweep_batch(const GraphView &g, const MoveLevel &lvl, MoveWorkspace &ws, const SweepParams &p,
                      const BatchSweep &b, const double *k, const double *sigma, cudaStream_t s) {
    const LMArgs A = batch_args(g, ws, p, b, k, sigma);
    dispatch_sweep<1>(g, lvl, ws, p, A, s);
}

void move_tune_batch(const GraphView &g, MoveLevel &lvl, MoveWorkspace &ws, const SweepParams &p,
                     const BatchSweep &b, const double *k, const double *sigma, cudaStream_t s) {
    tune_light<1>(g, lvl, ws, p, batch_args(g, ws, p, b, k, sigma), s);
}

}  // namespace mg
