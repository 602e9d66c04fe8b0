"""The reference's entry surface: the .mtx loader and the MG_GCD command line.

Each golden case (tests/golden/) holds what the reference's own loader
(src/mmio/mmio_wrapper.cu:76-295, built from its sources by
oracle/build_ref.sh) produced from a Matrix Market file, and the table its
MG_GCD binary printed for versions 0, 1 and 2 (src/main.cu:20-131, rows
printed at src/louvain/louvain.cu:1536-1538 and :1654).  The file itself is
not stored: it is the lower triangle of the loaded graph in row order
(make_golden.write_mtx), so it is rewritten here byte for byte from the
loaded CSR.

CPU: the engine's host loader (mg_csr_from_mtx) against the reference's
loaded CSR -- identical rows in identical order for symmetric pattern files
(the reference's stable row sort keeps file order), identical rows as sets
for general files (the reference fills them from 80 OpenMP threads, so its
order inside a row is unspecified).
GPU: MG_GCD -path_of_graph <file> -version v prints the reference's table:
same phases, same loop numbers, Q and dQ to the printed six decimals.
"""
import glob
import json
import os
import re
import subprocess
import sys

import numpy as np
import pytest

from conftest import GOLDEN, ROOT

sys.path.insert(0, GOLDEN)
import make_golden  # noqa: E402

CASES = sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN, "*.npz")))
CLI = os.path.join(ROOT, "mg-alphagcd_b200", "MG_GCD")


def _case(O, name, tmp_path):
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    meta = json.load(open(os.path.join(GOLDEN, name + ".json")))
    off = z["load_offsets"].astype(np.uint64)
    g = O.CSR(len(off) - 1, off, z["load_cols"], z["load_weights"]).sorted_rows()
    path = str(tmp_path / (name + ".mtx"))
    make_golden.write_mtx(path, g, meta["weighted"])
    return z, meta, path


def _row_sets(off, cols, w):
    row = np.repeat(np.arange(len(off) - 1), np.diff(off).astype(np.int64))
    o = np.lexsort((w, cols, row))
    return cols[o], w[o]


@pytest.mark.parametrize("name", CASES)
def test_loader_equals_reference_loader(O, mg, name, tmp_path):
    z, meta, path = _case(O, name, tmp_path)
    got = mg.load_mtx(path)
    off, cols = z["load_offsets"].astype(np.uint64), z["load_cols"]
    w = z["load_weights"]
    assert got["n"] == len(off) - 1
    assert (got["offsets"] == off).all()
    gw = np.ones(len(cols)) if got["weights"] is None else got["weights"]
    if not meta["weighted"]:
        # symmetric pattern: the reference stores 1.0 for every entry
        assert got["weights"] is None and (w == 1.0).all()
        assert (got["cols"] == cols).all()
    else:
        ca, wa = _row_sets(off, got["cols"], gw)
        cb, wb = _row_sets(off, cols, w)
        assert (ca == cb).all() and (wa == wb).all()


def _parse(out):
    rows, phase = [], -1
    for line in out.splitlines():
        m = re.match(r"Phase (\d+)", line)
        if m:
            phase = int(m.group(1))
            continue
        m = re.match(r"\|\s*(\d+)\s*\|\s*(-?[\d.]+)\s*\|\s*(-?[\d.]+)\s*\|", line)
        if m and phase >= 0:
            rows.append([phase, int(m.group(1)), float(m.group(2)), float(m.group(3))])
    return rows


@pytest.mark.gpu
@pytest.mark.parametrize("name", CASES)
def test_mg_gcd_prints_reference_tables(O, name, tmp_path):
    z, meta, path = _case(O, name, tmp_path)
    for version in (0, 1, 2):
        out = subprocess.run([CLI, "-path_of_graph", path, "-version", str(version)], capture_output=True,
                             text=True, timeout=300)
        assert out.returncode == 0, out.stderr[-2000:]
        got = _parse(out.stdout)
        want = meta["trace"][str(version)]
        assert len(got) == len(want), (version, len(got), len(want))
        for a, b in zip(got, want):
            assert a[:2] == b[:2], (version, a, b)
            # printed with %f: six decimals on both sides
            assert abs(a[2] - b[2]) <= 1.5e-6 and abs(a[3] - b[3]) <= 1.5e-6, (version, a, b)
        assert "Modularity" in out.stdout


def test_mg_gcd_rejects_unknown_version(tmp_path):
    # the reference prints this and exits 0 (src/main.cu:124-128); needs no GPU
    out = subprocess.run([CLI, "-version", "7"], capture_output=True, text=True, timeout=60)
    assert out.returncode == 0 and "unsupported" in out.stdout
