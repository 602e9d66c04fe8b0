"""GPU tests of the autotuner: the sweep's result must not depend on the
kernel shape picked for any degree class.  Runs with tuning on, tuning off and
a loaded table that forces unusual (but valid) shapes on every class all give
the oracle's result bit for bit (integral weights)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _run(ctx, g, **kw):
    return ctx.graph_from_csr(g.n, g.offsets, g.cols, g.weights).louvain(**kw)


def _same(a, b):
    assert a["modularity"] == b["modularity"]
    assert (a["assignment"] == b["assignment"]).all()
    assert a["iterations"] == b["iterations"] and a["levels"] == b["levels"]


WIDE = {0: "t4", 1: "t4", 2: "t8", 3: "t16", 4: "t32", 5: "h32", 6: "h64", 7: "h64", 8: "h32", 9: "h64",
        10: "h64", 11: "h128", 12: "h512"}
# the warp-batch kernel on every class it serves (5-10)
WARP = {c: "w" for c in range(5, 11)}


def _forced_table(path, bt=0, shapes=WIDE):
    """Every listed light class on the given shape, for level 0 (unit
    weights, kernel weight kind 0) and the coarsened levels (32-bit integer
    weights, kind 5)."""
    lines = []
    for wk in (0, 5):
        for c, sh in shapes.items():
            for bucket in range(12, 26):
                lines.append(f"{wk} 0 2 {bt} {c} {bucket} {sh} 1.0")
    path.write_text("\n".join(lines) + "\n")


def test_shapes_do_not_change_results(O, mg, tmp_path):
    g = O.gen_rmat(17, seed=7)  # classes 0-12 with >= 4096 vertices, heavy tiers
    ref = O.louvain(g)
    c1 = mg.Context(0)
    a = _run(c1, g)
    assert len(c1.tune_table()) > 0  # something was tuned
    _same(a, ref)
    b = _run(c1, g)  # second run: shapes from the table
    _same(b, ref)
    c1.tune_mode(mg.TUNE_OFF)
    _same(_run(c1, g), ref)
    c1.close()
    for shapes in (WIDE, WARP):
        c2 = mg.Context(0)
        p = tmp_path / "forced.txt"
        _forced_table(p, shapes=shapes)
        c2.tune_load(str(p))
        c2.tune_mode(mg.TUNE_CACHED)
        _same(_run(c2, g), ref)
        c2.close()


def test_batched_shapes_do_not_change_results(O, mg, tmp_path):
    gs = [O.gen_sbm(30000, 64, 20.0, 0.8, seed=s) for s in (1, 2)] + [O.gen_rmat(15, seed=3)]
    refs = [O.louvain(g) for g in gs]
    for shapes in (WARP, WIDE):
        c = mg.Context(0)
        p = tmp_path / "forced.txt"
        _forced_table(p, bt=1, shapes=shapes)
        c.tune_load(str(p))
        c.tune_mode(mg.TUNE_CACHED)
        res = c.batch_from_csr([(g.n, g.offsets, g.cols, None) for g in gs]).run()
        for i, r in enumerate(refs):
            assert res["graphs"]["modularity"][i] == r["modularity"]
            assert (res["assignments"][i] == r["assignment"]).all()
    c.tune_mode(mg.TUNE_ON)
    res2 = c.batch_from_csr([(g.n, g.offsets, g.cols, None) for g in gs]).run()
    assert (res2["graphs"]["modularity"] == res["graphs"]["modularity"]).all()
    c.close()
