"""GPU parity tests of the batched form: every graph of a batch must give the
result the oracle (and the single-graph engine) gives for it alone.

Bar: bit-exact modularity, assignment, phases, levels, iterations and
community count on integral graphs, for both launch modes (plain stream
launches and the CUDA-graph loop); real weights within 1e-9 of the
single-graph engine's modularity.
"""
import numpy as np
import pytest

from conftest import path, ring_of_cliques, star, two_cliques

pytestmark = pytest.mark.gpu


def _mixed_graphs(O):
    """Uneven sizes, hand-checkable shapes, an edgeless graph and a heavy one."""
    gs = [O.csr_from_pairs(*two_cliques()), O.csr_from_pairs(*ring_of_cliques()), O.csr_from_pairs(*star(40)),
          O.csr_from_pairs(*path(50))]
    gs.append(O.csr_from_pairs(7, np.zeros(0, np.int64), np.zeros(0, np.int64)))  # no edges
    gs.append(O.gen_sbm(4096, 16, 16.0, 0.8, seed=4))
    gs.append(O.gen_rmat(13, seed=2))  # heavy-tailed: hash and cluster bins
    gs.append(O.gen_sbm(1500, 4, 8.0, 0.7, seed=8))
    gs.append(O.gen_sbm(20000, 128, 24.0, 0.9, seed=9))
    return gs


def _pack(ctx, gs, weights=False):
    return ctx.batch_from_csr([(g.n, g.offsets, g.cols, g.weights if weights else None) for g in gs])


def _check_graph(res, g, ref, exact=True):
    per = res["graphs"]
    assert per["n"][g] == len(ref["assignment"])
    if exact:
        assert per["modularity"][g] == ref["modularity"], g
        assert (res["assignments"][g] == ref["assignment"]).all(), g
    else:
        assert abs(per["modularity"][g] - ref["modularity"]) < 1e-9, g
    assert per["communities"][g] == ref["communities"], g
    assert per["phases"][g] == ref["phases"], g
    assert per["levels"][g] == ref["levels"], g
    assert per["iterations"][g] == ref["iterations"], g


@pytest.mark.parametrize("graphs", [False, True])
def test_batch_matches_oracle(O, ctx, graphs):
    gs = _mixed_graphs(O)
    b = _pack(ctx, gs)
    res = b.run(graphs=graphs)
    for i, g in enumerate(gs):
        if g.nnz == 0:  # no modularity is defined; the engine keeps singletons (as mg_louvain_run)
            _check_graph(res, i, ctx.graph_from_csr(g.n, g.offsets, g.cols).louvain())
            continue
        _check_graph(res, i, O.louvain(g))
    assert res["graphs"]["communities"][4] == 7 and res["graphs"]["phases"][4] == 0


@pytest.mark.parametrize("version", [1, 2])
def test_batch_matches_single_engine(O, ctx, version):
    gs = _mixed_graphs(O)
    b = _pack(ctx, gs)
    res = b.run(version=version)
    for i, g in enumerate(gs):
        single = ctx.graph_from_csr(g.n, g.offsets, g.cols, g.weights).louvain(version=version)
        _check_graph(res, i, single)


def test_batch_generated_sbm_equals_single(O, ctx, mg):
    params = mg.draw_sbm_params(24, n_range=(500, 30000), blocks_range=(4, 256), deg_range=(8.0, 32.0),
                                intra_range=(0.7, 0.9), seed=11)
    b = ctx.batch_generate_sbm(params)
    info = b.info()
    assert info["graphs"] == 24 and info["n"] == sum(p["n"] for p in params)
    res = b.run()
    for i, p in enumerate(params[:8]):
        og = O.gen_sbm(p["n"], p["blocks"], p["mean_degree"], p["intra_frac"], seed=p["seed"])
        gi = b.graph_info(i)
        assert gi["n"] == og.n and gi["nnz"] == og.nnz and gi["mass"] == og.nnz
        _check_graph(res, i, O.louvain(og))
    for i, p in enumerate(params[8:], start=8):
        single = ctx.generate_sbm(p["n"], p["blocks"], p["mean_degree"], p["intra_frac"], p["seed"]).louvain()
        _check_graph(res, i, single)


def test_batch_integer_weights_and_precisions(O, ctx):
    gs = []
    for seed, n in ((1, 3000), (2, 800), (3, 9000)):
        g = O.gen_sbm(n, 8, 12.0, 0.8, seed=seed)
        # symmetric integer weights 1..4
        src = np.repeat(np.arange(g.n), np.diff(g.offsets).astype(np.int64))
        key = np.minimum(src, g.cols) * g.n + np.maximum(src, g.cols)
        w = (key * 2654435761 % 4 + 1).astype(np.float64)
        gs.append(type(g)(g.n, g.offsets, g.cols, w))
    b = _pack(ctx, gs, weights=True)
    for prec in ("fp64", "int64", "fp32"):
        res = b.run(precision=prec)
        for i, g in enumerate(gs):
            single = ctx.graph_from_csr(g.n, g.offsets, g.cols, g.weights).louvain(precision=prec)
            _check_graph(res, i, single)
            if prec == "fp64":
                _check_graph(res, i, O.louvain(g))


def test_batch_real_weights(O, ctx):
    gs = [O.gen_chunglu(4096, max_degree=500.0, seed=s) for s in (3, 4)]
    b = _pack(ctx, gs, weights=True)
    res = b.run()
    for i, g in enumerate(gs):
        ref = O.louvain(g)
        assert abs(res["graphs"]["modularity"][i] - ref["modularity"]) < 1e-3
        assert abs(O.modularity(g, res["assignments"][i]) - res["graphs"]["modularity"][i]) < 1e-9


def test_batch_max_phases_and_rerun(O, ctx):
    gs = [O.gen_sbm(5000, 16, 16.0, 0.8, seed=s) for s in (21, 22, 23)]
    b = _pack(ctx, gs)
    for mp in (1, 2):
        res = b.run(max_phases=mp)
        for i, g in enumerate(gs):
            _check_graph(res, i, O.louvain(g, max_phases=mp))
    # a batch is resident: running it again gives the same result
    r1, r2 = b.run(), b.run(graphs=False)
    assert (r1["graphs"]["modularity"] == r2["graphs"]["modularity"]).all()
    for a1, a2 in zip(r1["assignments"], r2["assignments"]):
        assert (a1 == a2).all()


def test_batch_rejects_bad_input(ctx, mg):
    with pytest.raises(mg.MGError):
        ctx.batch_from_csr([(3, np.array([0, 1, 2, 2], np.uint64), np.array([1, 5], np.uint32), None)])
