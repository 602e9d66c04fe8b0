"""The autotuner table: text format, load/save round trip and refusal of
malformed or impossible entries (a shape whose table cannot hold the class).
The table lives on the host, but a context needs a CUDA device, so those
checks are marked gpu; the NULL-argument checks run anywhere."""
import ctypes as ct

import pytest


def _ctx_handle(mg):
    return mg.Context(0)


@pytest.mark.gpu
def test_tune_mode_and_table_round_trip(mg, tmp_path):
    c = _ctx_handle(mg)
    assert c.tune_table() == []
    p = tmp_path / "tune.txt"
    p.write_text("0 0 2 0 9 14 h32 812.5\n4 0 2 1 12 11 h256 97.0\n")
    c.tune_load(str(p))
    t = c.tune_table()
    assert (0, 0, 2, 0, 9, 14, "h32", 812.5) in t and (4, 0, 2, 1, 12, 11, "h256", 97.0) in t
    q = tmp_path / "out.txt"
    c.tune_save(str(q))
    c2 = _ctx_handle(mg)
    c2.tune_load(str(q))
    assert sorted(c2.tune_table()) == sorted(t)
    c2.close()
    for mode in (mg.TUNE_OFF, mg.TUNE_CACHED, mg.TUNE_ON):
        c.tune_mode(mode)
    with pytest.raises(mg.MGError):
        c.tune_mode(7)
    c.close()


@pytest.mark.gpu
@pytest.mark.parametrize("line", ["0 0 2 0 9 14 t2 1.0", "0 0 2 0 13 14 h512 1.0", "0 0 2 0 9 14 h33 1.0", "bad"])
def test_tune_load_refuses_bad_lines(mg, tmp_path, line):
    c = _ctx_handle(mg)
    p = tmp_path / "bad.txt"
    p.write_text(line + "\n")
    with pytest.raises(mg.MGError):
        c.tune_load(str(p))
    assert c.tune_table() == []
    c.close()


def test_tune_calls_reject_null(mg):
    lib = mg.lib()
    assert lib.mg_tune_mode(None, 0) != 0
    assert lib.mg_tune_save(None, b"x") != 0
    assert lib.mg_tune_load(None, b"x") != 0
    n = ct.c_size_t()
    assert lib.mg_tune_table(None, None, 0, ct.byref(n)) != 0
