"""GPU parity tests: the CUDA engine (through the C ABI) against the oracle.

Bar: bit-exact for bins, assignments, integral-weight coarsening and the
modularity trace of integral graphs (both sides compute Q from exact integer
sums); real weights within the tolerances written in each test.
"""
import os

import numpy as np
import pytest

from conftest import boundary_degree_graph, path, ring_of_cliques, star, two_cliques

pytestmark = pytest.mark.gpu


def _up(ctx, g, weights_f32=False):
    w = g.weights
    if w is not None and weights_f32:
        w = w.astype(np.float32)
    return ctx.graph_from_csr(g.n, g.offsets, g.cols, w)


def _graphs(O):
    out = []
    for spec in (two_cliques(), ring_of_cliques(), star(40), path(50), boundary_degree_graph()):
        out.append(("small", O.csr_from_pairs(*spec)))
    out.append(("sbm4k", O.gen_sbm(4096, 16, 16.0, 0.8, seed=4)))
    out.append(("rmat14", O.gen_rmat(14, seed=2)))
    return out


def _states(O, g, k, mass):
    """(C, sigma) pairs: phase start, a mid-run state, a random assignment."""
    n = g.n
    res = []
    C0 = np.arange(n, dtype=np.uint32)
    res.append((C0, k.copy()))
    C = C0.copy()
    sig = k.copy()
    for it in range(3):
        Cn, _ = O.local_move(g, C, sig, k, mass, 2, it % 2 == 0)
        sig = np.zeros(n)
        np.add.at(sig, Cn, k)
        C = Cn
    res.append((C, sig))
    rng = np.random.default_rng(11)
    Cr = rng.integers(0, max(1, n // 8), n).astype(np.uint32)
    sr = np.zeros(n)
    np.add.at(sr, Cr, k)
    res.append((Cr, sr))
    return res


def test_bins_match(O, ctx):
    for name, g in _graphs(O):
        dg = _up(ctx, g)
        for scheme in (0, 1, 2):
            a = dg.bins(scheme)
            b = O.bins(scheme, g.offsets)
            assert (a["sizes"] == b["sizes"]).all(), (name, scheme)
            assert (a["offsets"] == b["offsets"]).all(), (name, scheme)
            assert a["max_degree"] == b["max_degree"], (name, scheme)
            assert (a["perm"] == b["perm"]).all(), (name, scheme)
            c = ctx.bins_offsets(scheme, g.offsets)
            assert (c["perm"] == b["perm"]).all() and (c["sizes"] == b["sizes"]).all()


@pytest.mark.parametrize("version", [1, 2])
def test_local_move_bit_exact(O, ctx, version):
    for name, g in _graphs(O):
        dg = _up(ctx, g)
        k = O.vertex_weights(g)
        mass = O.mass(g)
        for si, (C, sig) in enumerate(_states(O, g, k, mass)):
            for up in (True, False):
                a, da = dg.local_move(C, sig, k, version, up)
                b, db = O.local_move(g, C, sig, k, mass, version, up)
                bad = np.nonzero(a != b)[0]
                assert len(bad) == 0, (name, si, up, bad[:10], a[bad[:10]], b[bad[:10]])
                assert da == db, (name, si, up)


def test_local_move_integer_weights_bit_exact(O, ctx):
    rng = np.random.default_rng(5)
    base = O.gen_rmat(13, seed=3)
    row = np.repeat(np.arange(base.n), np.diff(base.offsets).astype(np.int64))
    m = row < base.cols
    w = rng.integers(1, 9, m.sum()).astype(np.float64)
    g = O.csr_from_pairs(base.n, row[m], base.cols[m], w)
    dg = _up(ctx, g)
    k = O.vertex_weights(g)
    mass = O.mass(g)
    for C, sig in _states(O, g, k, mass):
        for up in (True, False):
            for prec in ("fp64", "int64"):
                a, _ = dg.local_move(C, sig, k, 2, up, prec)
                b, _ = O.local_move(g, C, sig, k, mass, 2, up)
                if prec == "fp64":
                    assert (a == b).all()
                else:  # exact arithmetic may only differ on rounding ties
                    assert (a != b).mean() < 1e-3


def test_local_move_real_weights(O, ctx):
    g = O.gen_chunglu(1 << 14, max_degree=3000.0, seed=3)
    dg = _up(ctx, g, weights_f32=True)
    k = O.vertex_weights(g)
    mass = O.mass(g)
    for C, sig in _states(O, g, k, mass)[:2]:
        a, _ = dg.local_move(C, sig, k, 2, True)
        b, _ = O.local_move(g, C, sig, k, mass, 2, True)
        # summation order of k_ic differs (the reference's is unspecified too):
        # only near-ties may flip
        assert (a != b).mean() < 1e-3


def test_modularity_exact(O, ctx):
    for name, g in _graphs(O):
        dg = _up(ctx, g)
        k = O.vertex_weights(g)
        for C, _ in _states(O, g, k, O.mass(g)):
            assert dg.modularity(C) == O.modularity(g, C), name


def test_coarsen_bit_exact(O, ctx):
    for name, g in _graphs(O):
        dg = _up(ctx, g)
        k = O.vertex_weights(g)
        for C, _ in _states(O, g, k, O.mass(g)):
            cd_a, g2 = dg.coarsen(C)
            cd_b, h2, _ = O.coarsen(g, C)
            assert (cd_a == cd_b).all(), name
            off, cols, w = g2.csr()
            assert (off == h2.offsets).all(), name
            assert (cols == h2.cols).all(), name
            assert (w == h2.weights).all(), name


def test_coarsen_real_weights(O, ctx):
    g = O.gen_chunglu(1 << 13, max_degree=1000.0, seed=4)
    dg = _up(ctx, g)
    rng = np.random.default_rng(2)
    C = rng.integers(0, 500, g.n).astype(np.uint32)
    _, g2 = dg.coarsen(C)
    _, h2, _ = O.coarsen(g, C)
    off, cols, w = g2.csr()
    assert (off == h2.offsets).all() and (cols == h2.cols).all()
    np.testing.assert_allclose(w, h2.weights, rtol=1e-12)


def _compare_runs(a, b, exact=True):
    assert a["levels"] == b["levels"]
    assert (a["level_sizes"] == b["level_sizes"]).all()
    assert a["iterations"] == b["iterations"]
    if exact:
        assert (a["trace"] == b["trace"]).all()
        assert a["modularity"] == b["modularity"]
        assert (a["assignment"] == b["assignment"]).all()


@pytest.mark.parametrize("version", [0, 1, 2])
def test_louvain_bit_exact(O, ctx, version):
    for name, g in _graphs(O) + [("sbm64k", O.gen_sbm(65536, 64, 16.0, 0.8, seed=1))]:
        dg = _up(ctx, g)
        a = dg.louvain(version=version)
        b = O.louvain(g, version=2 if version == 0 else version)
        _compare_runs(a, b)
        assert a["communities"] == b["communities"]
        assert O.modularity(g, a["assignment"]) == a["modularity"]


def test_louvain_max_phases_and_threshold(O, ctx):
    g = O.gen_sbm(8192, 32, 16.0, 0.8, seed=9)
    dg = _up(ctx, g)
    for mp in (1, 2):
        _compare_runs(dg.louvain(max_phases=mp), O.louvain(g, max_phases=mp))
    _compare_runs(dg.louvain(threshold=1e-3), O.louvain(g, threshold=1e-3))


def test_louvain_precisions(O, ctx):
    g = O.gen_rmat(14, seed=5)
    dg = _up(ctx, g)
    ref = O.louvain(g)
    q64 = dg.louvain(precision="int64")["modularity"]
    q32 = dg.louvain(precision="fp32")["modularity"]
    # the precision contract: |Q - Q_oracle| <= 1e-3 for every mode
    assert abs(q64 - ref["modularity"]) <= 1e-3
    assert abs(q32 - ref["modularity"]) <= 1e-3


def test_louvain_real_weights(O, ctx):
    g = O.gen_chunglu(1 << 15, max_degree=5000.0, seed=3)
    dg = _up(ctx, g, weights_f32=True)
    a = dg.louvain()
    b = O.louvain(g)
    assert abs(a["modularity"] - b["modularity"]) < 1e-3
    # FP64 modularity recomputed from the returned assignment
    assert abs(O.modularity(g, a["assignment"]) - a["modularity"]) < 1e-9


def test_generators_match_oracle(O, ctx):
    for scale in (10, 14):
        dg = ctx.generate_rmat(scale, seed=2)
        g = O.gen_rmat(scale, seed=2)
        off, cols, _ = dg.csr()
        assert (off == g.offsets).all() and (cols == g.cols).all()
    dg = ctx.generate_sbm(65536, 64, 16.0, 0.8, seed=1)
    g = O.gen_sbm(65536, 64, 16.0, 0.8, seed=1)
    off, cols, _ = dg.csr()
    assert (off == g.offsets).all() and (cols == g.cols).all()


def test_chunglu_generator_matches_oracle(O, ctx):
    """Same topology as the oracle's Chung-Lu generator; lognormal weights equal
    up to the device's and host's libm (float-rounded values, relative 1e-6)."""
    for lognormal in (False, True):
        dg = ctx.generate_chunglu(20000, 2.1, 20.0, 2000.0, lognormal=lognormal, seed=3)
        g = O.gen_chunglu(20000, 2.1, 20.0, 2000.0, lognormal=lognormal, seed=3)
        off, cols, w = dg.csr()
        assert (off == g.offsets).all() and (cols == g.cols).all()
        info = dg.info()
        if lognormal:
            assert np.allclose(w, g.weights, rtol=1e-6, atol=0)
            assert not info["integral"]
        else:
            assert (w == 1.0).all() and info["integral"] and info["mass"] == g.nnz


def test_mtx_loader_matches_oracle(O, ctx, tmp_path):
    g = O.gen_sbm(3000, 10, 8.0, 0.8, seed=6)
    row = np.repeat(np.arange(g.n), np.diff(g.offsets).astype(np.int64))
    m = row > g.cols
    sym = tmp_path / "s.mtx"
    with open(sym, "w") as f:
        f.write("%%MatrixMarket matrix coordinate pattern symmetric\n%% test\n")
        f.write(f"{g.n} {g.n} {m.sum()}\n")
        for r, c in zip(row[m], g.cols[m]):
            f.write(f"{r + 1} {c + 1}\n")
    a = ctx.graph_from_mtx(str(sym))
    b = O.load_mtx(str(sym))
    off, cols, w = a.csr()
    assert (off == b.offsets).all() and (cols == b.cols).all() and (w == 1).all()
    rng = np.random.default_rng(1)
    gen = tmp_path / "g.mtx"
    with open(gen, "w") as f:
        f.write("%%MatrixMarket matrix coordinate real general\n")
        f.write(f"{g.n} {g.n} {len(row)}\n")
        for r, c in zip(row, g.cols):
            f.write(f"{r + 1} {c + 1} {rng.integers(1, 100) / 4}\n")
    a = ctx.graph_from_mtx(str(gen))
    b = O.load_mtx(str(gen))
    off, cols, w = a.csr()
    assert (off == b.offsets).all() and (cols == b.cols).all() and (w == b.weights).all()
    assert a.louvain()["modularity"] == O.louvain(b)["modularity"]
    # through the binary CSR cache (written, then mapped): the same graph
    for flags in ({"cache_read": True, "cache_write": True}, {"cache_read": True}):
        c = ctx.graph_from_mtx(str(gen), **flags)
        off2, cols2, w2 = c.csr()
        assert (off2 == off).all() and (cols2 == cols).all() and (w2 == w).all()
    assert os.path.exists(str(gen) + ".mgcsr")


def test_empty_and_edge_cases(O, ctx):
    # no edges: every vertex its own community, Q = 0
    dg = ctx.graph_from_csr(5, np.zeros(6, np.uint64), np.zeros(0, np.uint32))
    r = dg.louvain()
    assert r["modularity"] == 0 and (r["assignment"] == np.arange(5)).all()
    # a single edge
    g = O.csr_from_pairs(2, [0], [1])
    _compare_runs(_up(ctx, g).louvain(), O.louvain(g))
    # bad input is rejected with a status, not a crash
    import importlib
    mg = importlib.import_module("mg-alphagcd_b200")
    with pytest.raises(mg.MGError):
        ctx.graph_from_csr(3, np.array([0, 1, 2, 3], np.uint64), np.array([0, 5, 1], np.uint32))
    with pytest.raises(mg.MGError):
        _up(ctx, g).coarsen(np.array([0, 7], np.uint32))


def _permute_rows(g, rng, duplicate=0.0):
    """Same graph with every row's entries shuffled, optionally with some
    (symmetric) entries listed twice."""
    off = g.offsets.astype(np.int64)
    src = np.repeat(np.arange(g.n), np.diff(off))
    u, v = src, g.cols.astype(np.int64)
    keep = u < v
    u, v = u[keep], v[keep]
    if duplicate:
        d = rng.random(len(u)) < duplicate
        u, v = np.concatenate([u, u[d]]), np.concatenate([v, v[d]])
    a, b = np.concatenate([u, v]), np.concatenate([v, u])
    order = np.lexsort((rng.random(len(a)), a))
    a, b = a[order], b[order]
    offs = np.zeros(g.n + 1, np.uint64)
    np.add.at(offs, a + 1, 1)
    return type(g)(g.n, np.cumsum(offs).astype(np.uint64), b.astype(np.uint32), None)


@pytest.mark.parametrize("duplicate", [0.0, 0.05])
def test_unsorted_and_repeated_columns(O, ctx, duplicate):
    """Rows that are not sorted (shuffled) or list an edge twice (parallel
    edges, summed into k_ic like any repeated community): results stay exact."""
    rng = np.random.default_rng(17)
    for base in (O.gen_rmat(13, seed=4), O.gen_sbm(6000, 32, 14.0, 0.8, seed=5)):
        g = _permute_rows(base, rng, duplicate)
        a = _up(ctx, g).louvain()
        b = O.louvain(g)
        _compare_runs(a, b)


def test_dendrogram_levels_compose_to_assignment(O, ctx):
    """keep_levels: one dense community map per level; composing them gives
    the final assignment, which equals the oracle's."""
    for g in (O.gen_sbm(65536, 64, 16.0, 0.8, seed=1), O.gen_rmat(14, seed=2)):
        dg = _up(ctx, g)
        a = dg.louvain(keep_levels=True)
        maps = a["level_maps"]
        assert len(maps) == a["levels"] == len(a["level_sizes"])
        comp = np.arange(g.n, dtype=np.int64)
        for lvl, m in enumerate(maps):
            assert len(m) == a["level_sizes"][lvl]
            nxt = a["level_sizes"][lvl + 1] if lvl + 1 < len(maps) else a["communities"]
            assert m.max() + 1 == nxt and len(np.unique(m)) == nxt  # dense relabel
            comp = m[comp]
        assert (comp == a["assignment"]).all()
        assert (a["assignment"] == O.louvain(g)["assignment"]).all()
        assert "level_maps" not in dg.louvain()


def test_level_graphs_equal_oracle_coarsening(O, ctx):
    """keep_levels = 2: the graph of every level; level 0 is the input, level
    l + 1 is the oracle's coarsening of level l by level l's map (bit-exact)."""
    g = O.gen_rmat(14, seed=2)
    dg = _up(ctx, g)
    a = dg.louvain(keep_levels=2)
    graphs, maps = a["level_csr"], a["level_maps"]
    assert len(graphs) == len(maps) == a["levels"]
    off, cols, w = graphs[0]
    assert (off == g.offsets).all() and (cols == g.cols).all() and (w == 1).all()
    cur = g
    for lvl in range(len(graphs) - 1):
        _, h, _ = O.coarsen(cur, maps[lvl])
        off, cols, w = graphs[lvl + 1]
        assert len(off) - 1 == a["level_sizes"][lvl + 1]
        assert (off == h.offsets).all() and (cols == h.cols).all() and (w == h.weights).all(), lvl
        cur = h
    assert "level_csr" not in dg.louvain(keep_levels=1)


@pytest.mark.parametrize("combine", [1, 2])  # COMBINE_OFF, COMBINE_ON
def test_coarsen_combine_modes_bit_exact(O, mg, ctx, combine):
    """Coarsening with and without warp combining of equal keys gives the
    oracle's next-level graph (integral weights exactly, real weights to
    1e-12 relative), also for a phase's final assignment, where communities
    repeat inside rows and combining merges most entries."""
    ctx.sweep_options(coarsen_combine=combine)
    try:
        rng = np.random.default_rng(3)
        base = O.gen_rmat(13, seed=3)
        row = np.repeat(np.arange(base.n), np.diff(base.offsets).astype(np.int64))
        m = row < base.cols
        wint = O.csr_from_pairs(base.n, row[m], base.cols[m], rng.integers(1, 9, m.sum()).astype(np.float64))
        for name, g in _graphs(O) + [("rmat13w", wint)]:
            dg = _up(ctx, g)
            k = O.vertex_weights(g)
            states = [C for C, _ in _states(O, g, k, O.mass(g))]
            states.append(O.louvain(g, max_phases=1)["assignment"].astype(np.uint32))
            for C in states:
                cd_a, g2 = dg.coarsen(C)
                cd_b, h2, _ = O.coarsen(g, C)
                assert (cd_a == cd_b).all(), name
                off, cols, w = g2.csr()
                assert (off == h2.offsets).all() and (cols == h2.cols).all(), name
                assert (w == h2.weight_array()).all(), name
        g = O.gen_chunglu(1 << 13, max_degree=1000.0, seed=4)
        dg = _up(ctx, g)
        for C in (np.random.default_rng(2).integers(0, 500, g.n).astype(np.uint32),
                  O.louvain(g, max_phases=1)["assignment"].astype(np.uint32)):
            _, g2 = dg.coarsen(C)
            _, h2, _ = O.coarsen(g, C)
            off, cols, w = g2.csr()
            assert (off == h2.offsets).all() and (cols == h2.cols).all()
            np.testing.assert_allclose(w, h2.weights, rtol=1e-12)
    finally:
        ctx.sweep_options()


@pytest.mark.parametrize("combine", [1, 2])
def test_louvain_combine_modes(O, ctx, combine):
    ctx.sweep_options(coarsen_combine=combine)
    try:
        for name, g in [("sbm64k", O.gen_sbm(65536, 64, 16.0, 0.8, seed=1)), ("rmat14", O.gen_rmat(14, seed=2))]:
            _compare_runs(_up(ctx, g).louvain(), O.louvain(g))
    finally:
        ctx.sweep_options()


def test_first_sweep_kernels_equal_table_kernels(O, ctx):
    """A level's first sweep (every community one vertex) runs table-free
    kernels by default; forcing the table kernels gives the same runs, and
    both equal the oracle (integral weights bit for bit, real weights: the
    same assignment is not required, Q within 1e-3)."""
    graphs = [("rmat14", O.gen_rmat(14, seed=2)), ("sbm64k", O.gen_sbm(65536, 64, 16.0, 0.8, seed=1))]
    try:
        for name, g in graphs:
            dg = _up(ctx, g)
            ref = O.louvain(g)
            for table_first in (False, True):
                ctx.sweep_options(table_first_sweep=table_first)
                for version in (1, 2):
                    _compare_runs(dg.louvain(version=version), O.louvain(g, version=version) if version == 1 else ref)
        g = O.gen_chunglu(1 << 15, max_degree=5000.0, seed=3)
        dg = _up(ctx, g, weights_f32=True)
        ref = O.louvain(g)
        for table_first in (False, True):
            ctx.sweep_options(table_first_sweep=table_first)
            assert abs(dg.louvain()["modularity"] - ref["modularity"]) <= 1e-3
    finally:
        ctx.sweep_options()


@pytest.mark.parametrize("streams", [1, 3, 7])
def test_light_streams_do_not_change_results(O, ctx, streams):
    """The light classes on 1, 3 or 7 streams beside the heavy stream: the
    oracle's run bit for bit."""
    ctx.sweep_options(light_streams=streams)
    try:
        g = O.gen_rmat(14, seed=2)
        _compare_runs(_up(ctx, g).louvain(), O.louvain(g))
    finally:
        ctx.sweep_options()
