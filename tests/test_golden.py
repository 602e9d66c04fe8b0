"""Golden vectors produced by the reference's own code (tests/golden/make_golden.py,
run through oracle/_ref/ref_harness).  CPU tests pin the oracle to them; GPU
tests hold the engine to them.

Integral-weight cases are compared exactly (assignments, bins, coarsened
CSR after sorting rows by neighbour id); the reference's trace is printed
with six decimals, so Q is compared to 5e-7 and iteration counts exactly.
Real-weight cases (chunglu4k) use tolerances: the reference sums with FP64
atomics in an unspecified order.
"""
import glob
import hashlib
import json
import os

import numpy as np
import pytest

from conftest import GOLDEN

CASES = sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN, "*.npz")))


def _load(name):
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    meta = json.load(open(os.path.join(GOLDEN, name + ".json")))
    return z, meta


def _graph(O, z):
    return O.CSR(len(z["load_offsets"]) - 1, z["load_offsets"].astype(np.uint64), z["load_cols"],
                 z["load_weights"])


def _sorted_rows(off, cols, w):
    row = np.repeat(np.arange(len(off) - 1), np.diff(off).astype(np.int64))
    o = np.lexsort((w, cols, row))
    return cols[o], w[o]


def test_fixtures_present():
    if not CASES:
        pytest.skip("golden vectors not generated yet (tests/golden/make_golden.py on a GPU host)")
    assert {"sbm2k", "rmat12", "bounds", "rmat11w", "chunglu4k"} <= set(CASES)


def _check_bins(res_by_scheme, z):
    for scheme in range(3):
        b = res_by_scheme(scheme)
        nb = len(z[f"bins{scheme}_sizes"])
        assert (b["sizes"][:nb] == z[f"bins{scheme}_sizes"]).all(), scheme
        assert (b["offsets"][:nb] == z[f"bins{scheme}_offsets"]).all(), scheme
        assert b["max_degree"] == int(z[f"bins{scheme}_maxdeg"][0]), scheme
        # the reference's order inside a bin is unspecified: compare as sets
        off = z[f"bins{scheme}_offsets"]
        sz = z[f"bins{scheme}_sizes"]
        for i in range(nb):
            a = np.sort(b["perm"][off[i]:off[i] + sz[i]])
            r = np.sort(z[f"bins{scheme}_perm"][off[i]:off[i] + sz[i]])
            assert (a == r).all(), (scheme, i)


def _check_moves(move, z, exact):
    for sname in ("start", "mid"):
        C, sig, k = z[f"move_{sname}_C"], z[f"move_{sname}_sigma"], z[f"move_{sname}_k"]
        for version in (1, 2):
            for up in (1, 0):
                a = move(C, sig, k, version, bool(up))
                r = z[f"move_{sname}_v{version}_up{up}"]
                if exact:
                    assert (a == r).all(), (sname, version, up, np.nonzero(a != r)[0][:10])
                else:
                    assert (a != r).mean() < 5e-3, (sname, version, up)


def _check_coarsen(coarsen, z, exact):
    for cname in ("mid", "final"):
        off, cols, w = coarsen(z[f"coarsen_{cname}_C"])
        roff = z[f"coarsen_{cname}_offsets"]
        assert (np.asarray(off, np.uint64) == roff).all(), cname
        ac, aw = _sorted_rows(np.asarray(off, np.int64), np.asarray(cols), np.asarray(w))
        rc, rw = _sorted_rows(roff.astype(np.int64), z[f"coarsen_{cname}_cols"], z[f"coarsen_{cname}_weights"])
        assert (ac == rc).all(), cname
        if exact:
            assert (aw == rw).all(), cname
        else:
            np.testing.assert_allclose(aw, rw, rtol=1e-12, atol=1e-9)


def _check_trace(run, meta, exact):
    for version in ("0", "1", "2"):
        ref = np.array(meta["trace"][version], dtype=np.float64)
        got = run(int(version))
        if exact:
            assert len(got) == len(ref), version
            assert (got[:, :2] == ref[:, :2]).all(), version
            assert np.abs(got[:, 2] - ref[:, 2]).max() <= 5e-7, version
        else:
            # real weights: final modularity within the contract's 1e-3
            assert abs(got[-1, 2] - ref[-1, 2]) < 1e-3, version


# ---- oracle (CPU) -------------------------------------------------------------------


@pytest.mark.parametrize("name", CASES)
def test_oracle_against_reference(O, name):
    z, meta = _load(name)
    g = _graph(O, z)
    exact = O.is_integral(g)
    _check_bins(lambda s: O.bins(s, g.offsets), z)
    k = O.vertex_weights(g)
    mass = O.mass(g)
    _check_moves(lambda C, sig, kk, v, up: O.local_move(g, C, sig, kk, mass, v, up)[0], z, exact)

    def co(C):
        _, h, _ = O.coarsen(g, C)
        return h.offsets, h.cols, h.weights

    _check_coarsen(co, z, exact)
    _check_trace(lambda v: O.louvain(g, version=2 if v == 0 else v)["trace"], meta, exact)


# ---- engine (GPU) -------------------------------------------------------------------


@pytest.mark.gpu
@pytest.mark.parametrize("name", CASES)
def test_engine_against_reference(O, ctx, name):
    z, meta = _load(name)
    g = _graph(O, z)
    exact = O.is_integral(g)
    dg = ctx.graph_from_csr(g.n, g.offsets, g.cols, g.weights)
    _check_bins(lambda s: dg.bins(s), z)
    _check_moves(lambda C, sig, k, v, up: dg.local_move(C, sig, k, v, up)[0], z, exact)

    def co(C):
        _, h = dg.coarsen(C)
        return h.csr()

    _check_coarsen(co, z, exact)
    _check_trace(lambda v: dg.louvain(version=v)["trace"], meta, exact)


# ---- larger graphs: the reference's printed tables only (tests/golden/traces.json) ----------

TRACES = os.path.join(GOLDEN, "traces.json")
TRACE_NAMES = sorted(json.load(open(TRACES))) if os.path.exists(TRACES) else []


def _trace_case(name):
    return json.load(open(TRACES))[name]


def _trace_graph(O, meta):
    kw = dict(meta["args"])
    return O.gen_sbm(**kw) if meta["generator"] == "sbm" else O.gen_rmat(**kw)


def _digest(off, cols):
    h = hashlib.sha256()
    h.update(np.asarray(off, np.uint64).tobytes())
    h.update(np.asarray(cols, np.uint32).tobytes())
    return h.hexdigest()


def test_trace_fixtures_present():
    if not TRACE_NAMES:
        pytest.skip("reference traces not generated yet (make_golden.py --traces on a GPU host)")
    assert {"sbm64k", "rmat16"} <= set(TRACE_NAMES)


@pytest.mark.parametrize("name", TRACE_NAMES)
def test_oracle_trace_against_reference(O, name):
    """The oracle's Louvain on the regenerated graph prints the reference's table:
    same phases and loops, Q to the printed 6 decimals (versions 0/1/2)."""
    meta = _trace_case(name)
    g = _trace_graph(O, meta)
    assert (g.n, len(g.cols)) == (meta["n"], meta["nnz"])
    assert _digest(g.offsets, g.cols) == meta["sha256"]
    _check_trace(lambda v: O.louvain(g, version=2 if v == 0 else v)["trace"], meta, True)


@pytest.mark.gpu
@pytest.mark.parametrize("name", TRACE_NAMES)
def test_engine_trace_against_reference(ctx, name):
    """The engine's generator gives the reference's input graph (same digest) and
    its Louvain run prints the reference's table (versions 0/1/2)."""
    meta = _trace_case(name)
    kw = dict(meta["args"])
    if meta["generator"] == "sbm":
        dg = ctx.generate_sbm(kw["n"], kw["blocks"], kw["mean_degree"], kw["intra_frac"], kw["seed"])
    else:
        dg = ctx.generate_rmat(kw["scale"], seed=kw["seed"])
    off, cols, _ = dg.csr()
    assert _digest(off, cols) == meta["sha256"]
    _check_trace(lambda v: dg.louvain(version=v)["trace"], meta, True)
