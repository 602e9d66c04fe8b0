"""Coarsening of symmetric integral graphs from the transposed side.

A symmetric integral graph (every entry (u, v, w) matched by an entry
(v, u, w)) is expanded in community order from the transposed side, so the
coarsening sorts only the high half of every key; any other graph takes the
full sort.  Both must give the oracle's next-level graph bit for bit
(oracle/oracle.c, the restatement of coarsen_graph_mg::coarsen_graph,
src/coarsen_graph/coarsen_graph_mg.cu:2054-2240).  The symmetry of an upload
is decided by two 64-bit multiset fingerprints of the entries and of their
transposes: symmetric uploads must pass, and one-sided changes must not.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _csr(O, n, row, col, w=None):
    """CSR of the entries as given (no symmetrisation), rows sorted by column."""
    row = np.asarray(row, np.int64)
    col = np.asarray(col, np.int64)
    order = np.lexsort((col, row))
    row, col = row[order], col[order]
    off = np.zeros(n + 1, np.uint64)
    np.add.at(off, row + 1, 1)
    off = np.cumsum(off).astype(np.uint64)
    ww = None if w is None else np.asarray(w, np.float64)[order]
    return O.CSR(n, off, col.astype(np.uint32), ww)


def _entries(g):
    row = np.repeat(np.arange(g.n), np.diff(g.offsets).astype(np.int64))
    return row, g.cols.astype(np.int64), g.weight_array().copy()


def _states(O, g):
    n = g.n
    rng = np.random.default_rng(5)
    yield np.arange(n, dtype=np.uint32)
    yield rng.integers(0, max(1, n // 16), n).astype(np.uint32)
    yield (np.arange(n) // 7).astype(np.uint32)


def _check_coarsen(O, dg, g):
    for C in _states(O, g):
        cd_a, g2 = dg.coarsen(C)
        cd_b, h2, _ = O.coarsen(g, C)
        assert (cd_a == cd_b).all()
        off, cols, w = g2.csr()
        assert (off == h2.offsets).all() and (cols == h2.cols).all()
        assert (w == h2.weight_array()).all()


def test_symmetry_of_generated_uploaded_and_coarsened_graphs(O, ctx):
    assert ctx.generate_rmat(12, seed=3).properties() == {"sorted_rows": True, "symmetric": True}
    assert ctx.generate_sbm(5000, 8, seed=2).properties()["symmetric"]
    g = O.gen_rmat(12, seed=3)
    assert ctx.graph_from_csr(g.n, g.offsets, g.cols, None).properties() == {"sorted_rows": True,
                                                                             "symmetric": True}
    # integral weights, equal in both directions
    row, col, _ = _entries(g)
    lo = row < col
    rng = np.random.default_rng(1)
    wt = O.csr_from_pairs(g.n, row[lo], col[lo], rng.integers(1, 9, lo.sum()).astype(np.float64))
    dw = ctx.graph_from_csr(wt.n, wt.offsets, wt.cols, wt.weights)
    assert dw.properties()["symmetric"]
    # its coarsened graph keeps the property
    assert dw.coarsen(np.arange(wt.n, dtype=np.uint32) // 3)[1].properties()["symmetric"]
    # one weight changed on one side only
    r2, c2, w2 = _entries(wt)
    w2[7] += 1
    bad = _csr(O, wt.n, r2, c2, w2)
    assert not ctx.graph_from_csr(bad.n, bad.offsets, bad.cols, bad.weights).properties()["symmetric"]
    # weights swapped between two entries of one row (same multiset of weights per row)
    w3 = wt.weight_array().copy()
    k = next(i for i in range(wt.n) if wt.offsets[i + 1] - wt.offsets[i] >= 2 and
             wt.weights[wt.offsets[i]] != wt.weights[wt.offsets[i] + 1])
    a = int(wt.offsets[k])
    w3[a], w3[a + 1] = w3[a + 1], w3[a]
    sw = O.CSR(wt.n, wt.offsets, wt.cols, w3)
    assert not ctx.graph_from_csr(sw.n, sw.offsets, sw.cols, sw.weights).properties()["symmetric"]
    # one extra entry in one direction
    ex = _csr(O, g.n, np.append(row, 0), np.append(col, g.n - 1))
    assert ex.cols[ex.offsets[1] - 1] == g.n - 1
    assert not ctx.graph_from_csr(ex.n, ex.offsets, ex.cols, None).properties()["symmetric"]
    # a repeated entry in both directions: symmetric as a multiset, rows not strictly increasing
    rep = _csr(O, g.n, np.append(row, [0, int(col[0])]), np.append(col, [int(col[0]), 0]))
    assert ctx.graph_from_csr(rep.n, rep.offsets, rep.cols, None).properties() == {"sorted_rows": False,
                                                                                   "symmetric": True}
    # real weights: never marked (the coarsening keeps the full sort)
    rw = O.CSR(wt.n, wt.offsets, wt.cols, wt.weights + 0.5)
    assert not ctx.graph_from_csr(rw.n, rw.offsets, rw.cols, rw.weights).properties()["symmetric"]


@pytest.mark.parametrize("weighted", [False, True])
def test_coarsen_of_directed_graphs_bit_exact(O, ctx, weighted):
    """Directed graphs (each edge stored once, or with unequal weights in the
    two directions) take the full sort and still give the oracle's graph."""
    rng = np.random.default_rng(4)
    base = O.gen_rmat(13, seed=5)
    row, col, _ = _entries(base)
    keep = rng.random(len(row)) < 0.7
    w = rng.integers(1, 20, keep.sum()).astype(np.float64) if weighted else None
    g = _csr(O, base.n, row[keep], col[keep], w)
    dg = ctx.graph_from_csr(g.n, g.offsets, g.cols, g.weights)
    assert not dg.properties()["symmetric"]
    _check_coarsen(O, dg, g)


@pytest.mark.parametrize("combine", [1, 2])  # COMBINE_OFF, COMBINE_ON
def test_coarsen_of_symmetric_uploads_bit_exact(O, ctx, combine):
    """Symmetric uploads (unit and integral weights, a repeated entry pair,
    isolated vertices): through the transposed expansion without warp
    combining, through the full sort of the combined keys with it."""
    ctx.sweep_options(coarsen_combine=combine)
    try:
        g = O.gen_rmat(14, seed=7)
        row, col, _ = _entries(g)
        lo = row < col
        rng = np.random.default_rng(8)
        wt = O.csr_from_pairs(g.n, row[lo], col[lo], rng.integers(1, 1000, lo.sum()).astype(np.float64))
        rep = _csr(O, g.n, np.append(row, [3, int(col[0])]), np.append(col, [int(col[0]), 3]))
        for h in (g, wt, rep):
            dh = ctx.graph_from_csr(h.n, h.offsets, h.cols, h.weights)
            assert dh.properties()["symmetric"]
            _check_coarsen(O, dh, h)
            C = O.louvain(h, max_phases=1)["assignment"].astype(np.uint32)
            cd_a, g2 = dh.coarsen(C)
            cd_b, h2, _ = O.coarsen(h, C)
            off, cols, w = g2.csr()
            assert (off == h2.offsets).all() and (cols == h2.cols).all() and (w == h2.weight_array()).all()
    finally:
        ctx.sweep_options()
