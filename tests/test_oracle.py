"""CPU tests of the oracle (the checker the GPU parity tests rely on)."""
import numpy as np
import pytest

import pyref
from conftest import boundary_degree_graph, path, ring_of_cliques, star, two_cliques


def _csr(O, spec, w=None):
    n, u, v = spec
    return O.csr_from_pairs(n, u, v, w)


SMALL = [two_cliques(), ring_of_cliques(), star(), path(), two_cliques(7)]


def test_bins_thresholds(O):
    n, u, v = boundary_degree_graph()
    g = O.csr_from_pairs(n, u, v)
    deg = np.diff(g.offsets)
    th = {0: [2, 4, 8, 16, 32, 128, 512, 2048, 4094], 1: [32, 64, 128, 256, 512, 1024, 2048, 4096, 8192, 12288],
          2: [32, 64, 128, 256, 512, 1024, 2048, 4095]}
    for scheme, t in th.items():
        b = O.bins(scheme, g.offsets)
        expect = np.searchsorted(np.array(t), deg, side="left")
        sizes = np.bincount(expect, minlength=len(t) + 1)
        assert (b["sizes"] == sizes).all(), scheme
        assert b["max_degree"] == deg.max()
        assert (b["offsets"] == np.concatenate([[0], np.cumsum(sizes)[:-1]])).all()
        # perm: bin by bin, ascending id inside a bin
        order = np.lexsort((np.arange(n), expect))
        assert (b["perm"] == order).all()


@pytest.mark.parametrize("spec", SMALL)
@pytest.mark.parametrize("version", [1, 2])
@pytest.mark.parametrize("up", [True, False])
def test_local_move_matches_python(O, spec, version, up):
    g = _csr(O, spec)
    k = O.vertex_weights(g)
    mass = O.mass(g)
    rng = np.random.default_rng(7)
    for trial in range(3):
        C = np.arange(g.n, dtype=np.uint32) if trial == 0 else rng.integers(0, g.n, g.n).astype(np.uint32)
        sig = np.zeros(g.n)
        np.add.at(sig, C, k)
        a, _ = O.local_move(g, C, sig, k, mass, version, up)
        b = pyref.local_move(g.n, g.offsets, g.cols, None, C, sig, k, mass, version, up)
        assert (a == b).all()


def test_local_move_weighted_matches_python(O):
    n, u, v = ring_of_cliques(5, 5)
    rng = np.random.default_rng(3)
    w = rng.integers(1, 5, len(u)).astype(np.float64)
    g = O.csr_from_pairs(n, u, v, w)
    k = O.vertex_weights(g)
    mass = O.mass(g)
    for up in (True, False):
        C = rng.integers(0, n, n).astype(np.uint32)
        sig = np.zeros(n)
        np.add.at(sig, C, k)
        a, _ = O.local_move(g, C, sig, k, mass, 2, up)
        b = pyref.local_move(n, g.offsets, g.cols, g.weights, C, sig, k, mass, 2, up)
        assert (a == b).all()


def test_modularity_matches_python(O):
    n, u, v = ring_of_cliques()
    g = O.csr_from_pairs(n, u, v)
    rng = np.random.default_rng(1)
    for _ in range(3):
        C = rng.integers(0, 4, n).astype(np.uint32)
        assert O.modularity(g, C) == pytest.approx(pyref.modularity(n, g.offsets, g.cols, None, C), abs=1e-14)


def test_two_cliques_closed_form(O):
    k = 5
    g = _csr(O, two_cliques(k))
    r = O.louvain(g)
    # two communities = the two cliques; Q = sum_in/2m - sum sigma^2/(2m)^2
    a = r["assignment"]
    assert len(set(a[:k])) == 1 and len(set(a[k:])) == 1 and a[0] != a[k]
    m2 = 2 * (2 * (k * (k - 1) // 2) + 1)
    sin = 2 * 2 * (k * (k - 1) // 2)
    sig = (k * (k - 1) + 1)
    q = sin / m2 - 2 * sig * sig / m2 ** 2
    assert r["modularity"] == pytest.approx(q, abs=1e-12)


def test_ring_of_cliques_finds_cliques(O):
    n, u, v = ring_of_cliques(8, 5)
    g = O.csr_from_pairs(n, u, v)
    r = O.louvain(g)
    assert r["communities"] <= 8
    assert r["modularity"] == pytest.approx(O.modularity(g, r["assignment"]), abs=1e-12)


def test_coarsen_invariants(O):
    g = O.gen_sbm(2048, 16, 12.0, 0.8, seed=5)
    r = O.louvain(g, max_phases=1)
    rng = np.random.default_rng(0)
    for C in (r["assignment"], rng.integers(0, 300, g.n).astype(np.uint32)):
        cd, g2, up = O.coarsen(g, C)
        assert g2.weights.sum() == O.mass(g)  # mass invariant
        # rows sorted by neighbour community, no duplicates
        for rr in range(g2.n):
            row = g2.cols[g2.offsets[rr]:g2.offsets[rr + 1]]
            assert (np.diff(row.astype(np.int64)) > 0).all()
        # modularity invariant: Q(G, C) == Q(G', identity)
        q1 = O.modularity(g, C)
        q2 = O.modularity(g2, np.arange(g2.n, dtype=np.uint32))
        assert q1 == pytest.approx(q2, abs=1e-12)
        # dense, order-preserving relabel
        used = np.unique(C)
        assert (cd == np.searchsorted(used, C)).all()
        # upper degree = sum of member degrees
        deg = np.diff(g.offsets)
        expect = np.zeros(g2.n, np.int64)
        np.add.at(expect, cd, deg)
        assert (np.diff(up) == expect).all()


def test_louvain_sbm64k_quality(O):
    g = O.gen_sbm(65536, 64, 16.0, 0.8, seed=1)
    assert g.n == 65536 and 1.0e6 < g.nnz < 1.1e6
    r = O.louvain(g)
    assert r["modularity"] > 0.7
    assert r["modularity"] == pytest.approx(O.modularity(g, r["assignment"]), abs=1e-12)
    # trace rows: loop 0 opens every phase; the last row of a phase is a rejection (dQ 0)
    t = r["trace"]
    assert t[0][1] == 0 and t[0][0] == 0
    assert r["level_sizes"][0] == 65536


def test_version1_differs_and_is_valid(O):
    g = O.gen_rmat(12, seed=2)
    r1 = O.louvain(g, version=1)
    r2 = O.louvain(g, version=2)
    assert r1["modularity"] == pytest.approx(O.modularity(g, r1["assignment"]), abs=1e-12)
    assert r2["modularity"] == pytest.approx(O.modularity(g, r2["assignment"]), abs=1e-12)


def test_generators_deterministic(O):
    a = O.gen_rmat(10, seed=9)
    b = O.gen_rmat(10, seed=9)
    c = O.gen_rmat(10, seed=10)
    assert (a.offsets == b.offsets).all() and (a.cols == b.cols).all()
    assert not ((len(a.cols) == len(c.cols)) and (a.cols == c.cols).all())
    # symmetric, no self-loops, sorted rows
    for g in (a, O.gen_sbm(1000, 10, seed=3)):
        row = np.repeat(np.arange(g.n), np.diff(g.offsets).astype(np.int64))
        assert (row != g.cols).all()
        fwd = set(zip(row.tolist(), g.cols.tolist()))
        assert all((v, u) in fwd for (u, v) in fwd)


def test_chunglu_weights(O):
    g = O.gen_chunglu(1 << 14, max_degree=2000.0, seed=3)
    assert g.weights is not None and (g.weights > 0).all()
    assert (g.weights.astype(np.float32).astype(np.float64) == g.weights).all()
    assert not O.is_integral(g)
    row = np.repeat(np.arange(g.n), np.diff(g.offsets).astype(np.int64))
    # weight is a function of the unordered pair
    d = {}
    for u, v, w in zip(row.tolist(), g.cols.tolist(), g.weights.tolist()):
        key = (min(u, v), max(u, v))
        assert d.setdefault(key, w) == w


def test_loader_rules(O, tmp_path):
    sym = tmp_path / "s.mtx"
    sym.write_text("%%MatrixMarket matrix coordinate pattern symmetric\n% c\n5 5 6\n2 1\n3 1\n3 3\n4 2\n5 4\n5 1\n")
    g = O.load_mtx(str(sym))
    assert list(g.offsets) == [0, 3, 5, 7, 9, 11]
    assert list(g.cols) == [1, 2, 4, 0, 3, 0, 2, 1, 4, 3, 0]
    gen = tmp_path / "g.mtx"
    gen.write_text("%%MatrixMarket matrix coordinate real general\n5 5 7\n2 1 0.5\n1 2 0.5\n3 1 2.25\n3 3 9\n"
                   "4 2 1\n5 4 3\n5 1\n")
    g = O.load_mtx(str(gen))
    # upper triangle and diagonal dropped, weights read, both directions stored
    assert list(g.offsets) == [0, 3, 5, 6, 8, 10]
    assert g.weights.sum() == 2 * (0.5 + 2.25 + 1 + 3 + 1)
    bad = tmp_path / "bad.mtx"
    bad.write_text("%%MatrixMarket matrix coordinate pattern symmetric\n3 3 2\n2 1\n")
    with pytest.raises(ValueError):
        O.load_mtx(str(bad))


def test_constant_division_identity(O):
    """The engine divides by m and 2m with a precomputed reciprocal and one fma
    correction; this checks the identity against IEEE division on the CPU."""
    import ctypes as ct
    L = O.lib()
    L.or_check_const_division.restype = ct.c_uint64
    L.or_check_const_division.argtypes = [ct.c_uint64, ct.c_uint64, ct.c_void_p, ct.c_int]
    rng = np.random.default_rng(3)
    d = np.ascontiguousarray(np.concatenate([[1.0, 2.0, 3.0, 520770236.0, 260385118.0, 521211.0],
                                             rng.uniform(1, 4e9, 64), rng.integers(1, 2**32, 64).astype(float)]))
    assert L.or_check_const_division(4_000_000, 11, d.ctypes.data, len(d)) == 0
