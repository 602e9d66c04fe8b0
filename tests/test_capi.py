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
