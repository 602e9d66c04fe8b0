"""CPU checks of the C ABI: the library loads and exports every entry point
declared in include/mgagcd.h (no compute calls without a GPU)."""
import ctypes as ct
import os
import re

from conftest import ROOT


def _declared():
    src = open(os.path.join(ROOT, "include", "mgagcd.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(mg_[a-z0-9_]+)\s*\(", src)))


def test_header_declares_entry_points():
    names = _declared()
    assert "mg_louvain_run" in names and "mg_local_move" in names and "mg_coarsen" in names
    assert len(names) >= 20


def test_library_exports_every_declared_symbol(mg):
    lib = mg.lib()
    for name in _declared():
        assert hasattr(lib, name), name
    assert set(mg.EXPORTED) <= set(_declared())


def test_status_strings(mg):
    lib = mg.lib()
    for s in range(9):
        assert lib.mg_status_string(s)
    assert b"sm_100a" in lib.mg_version()


def test_null_arguments_fail_cleanly(mg):
    lib = mg.lib()
    assert lib.mg_graph_destroy(None) != 0
    assert lib.mg_result_destroy(None) != 0
    assert lib.mg_init(None, None) != 0
    assert lib.mg_last_error(None)


def test_batch_sbm_parameter_draw(mg):
    """Host-side draw of a batch's SBM parameters: deterministic, inside the ranges."""
    a = mg.draw_sbm_params(4096, seed=4)
    b = mg.draw_sbm_params(4096, seed=4)
    assert a == b
    assert a != mg.draw_sbm_params(4096, seed=5)
    n = [p["n"] for p in a]
    assert min(n) >= 1000 and max(n) <= 200000
    # log-uniform: the median sits near the geometric mean of the range
    assert 10000 < sorted(n)[len(n) // 2] < 20000
    for p in a:
        assert 4 <= p["blocks"] <= min(256, p["n"])
        assert 8.0 <= p["mean_degree"] <= 32.0 and 0.7 <= p["intra_frac"] <= 0.9
    assert len({p["seed"] for p in a}) == 4096
    lib = mg.lib()
    assert lib.mg_batch_draw_sbm_params(1, 10, 5, 4, 256, 8.0, 32.0, 0.7, 0.9, 1, None) != 0


def test_batch_null_arguments(mg):
    lib = mg.lib()
    assert lib.mg_batch_destroy(None) != 0
    assert lib.mg_batch_result_destroy(None) != 0
    assert lib.mg_batch_run(None, None, 0, None) != 0
