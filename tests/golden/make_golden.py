"""Generate the golden vectors under tests/golden/ from the reference itself.

Runs oracle/_ref/ref_harness (the reference's own sources built by
oracle/build_ref.sh with the single-PE shim) on small seeded graphs:
  * the reference's .mtx loader            (src/mmio/mmio_wrapper.cu:76-295)
  * BIN::bin_create, all three schemes     (src/bin/BIN.cu:468-575)
  * one local-move sweep, versions 1 and 2 (src/louvain/louvain.cu:1032, louvain_gl.cu:1018)
  * coarsen_graph_mg::coarsen_graph        (src/coarsen_graph/coarsen_graph_mg.cu:2054)
  * louvain*::run printed tables           (src/louvain/louvain*.cu run())
and, with --traces, the printed tables alone (versions 0, 1 and 2) on two
larger seeded graphs -- the 65,536-vertex SBM of the plain-Louvain workload and
R-MAT scale 16 -- into traces.json (the graphs are regenerated from their
seeds by the oracle's and the engine's generators, so only the tables and a
checksum of each graph are stored).
The inputs (graphs, assignments, sigma, k) come from the CPU oracle's seeded
generators and are stored with the outputs, so the fixtures are
self-contained.  Needs a CUDA GPU for everything but the loader.

Usage: python tests/golden/make_golden.py [--out DIR] [--traces]
"""
from __future__ import annotations

import argparse
import json
import os
import re
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import oracle_py as O  # noqa: E402

HARNESS = os.path.join(ROOT, "oracle", "_ref", "ref_harness")


def write_mtx(path, g, weighted):
    """Lower triangle of a symmetric CSR: pattern/symmetric or real/general."""
    row = np.repeat(np.arange(g.n), np.diff(g.offsets).astype(np.int64))
    m = row > g.cols
    with open(path, "w") as f:
        if weighted:
            f.write("%%MatrixMarket matrix coordinate real general\n")
            f.write(f"{g.n} {g.n} {int(m.sum())}\n")
            for r, c, w in zip(row[m], g.cols[m], g.weights[m]):
                f.write(f"{r + 1} {c + 1} {float(w)!r}\n")
        else:
            f.write("%%MatrixMarket matrix coordinate pattern symmetric\n")
            f.write(f"{g.n} {g.n} {int(m.sum())}\n")
            for r, c in zip(row[m], g.cols[m]):
                f.write(f"{r + 1} {c + 1}\n")


def read_graph(path):
    b = open(path, "rb").read()
    n, nnz = np.frombuffer(b[:8], np.uint32)
    o = 8
    off = np.frombuffer(b[o:o + 4 * (n + 1)], np.uint32).astype(np.uint64)
    o += 4 * (n + 1)
    cols = np.frombuffer(b[o:o + 4 * nnz], np.uint32).copy()
    o += 4 * nnz
    w = np.frombuffer(b[o:o + 8 * nnz], np.float64).copy()
    return int(n), off, cols, w


def run(*args):
    return subprocess.run([HARNESS, *map(str, args)], check=True, capture_output=True, text=True,
                          timeout=300).stdout


def parse_table(out):
    rows = []
    phase = -1
    for line in out.splitlines():
        m = re.match(r"Phase (\d+)", line)
        if m:
            phase = int(m.group(1))
            continue
        m = re.match(r"\|\s*(\d+)\s*\|\s*(-?[\d.]+)\s*\|\s*(-?[\d.]+)\s*\|", line)
        if m and phase >= 0:
            rows.append([phase, int(m.group(1)), float(m.group(2)), float(m.group(3))])
    return rows


def cases():
    rng = np.random.default_rng(2024)
    out = []
    out.append(("sbm2k", O.gen_sbm(2048, 16, 16.0, 0.8, seed=7), False))
    out.append(("rmat12", O.gen_rmat(12, seed=2), False))
    # degrees on every bin threshold (local move up to the global-table bin)
    degs = [0, 1, 2, 3, 4, 5, 8, 9, 16, 17, 32, 33, 128, 129, 512, 513, 2048, 2049, 4094, 4095, 4096, 5000,
            8192, 8193, 12288, 12289]
    u, v = [], []
    nc = len(degs)
    for i, d in enumerate(degs):
        for j in range(d):
            u.append(i)
            v.append(nc + (j * 7 + i) % (max(degs) + 1))
    extra = rng.integers(nc, nc + max(degs) + 1, size=(4000, 2))
    u += extra[:, 0].tolist()
    v += extra[:, 1].tolist()
    out.append(("bounds", O.csr_from_pairs(nc + max(degs) + 1, np.array(u), np.array(v)), False))
    base = O.gen_rmat(11, seed=4)
    row = np.repeat(np.arange(base.n), np.diff(base.offsets).astype(np.int64))
    m = row < base.cols
    w = rng.integers(1, 9, m.sum()).astype(np.float64)
    out.append(("rmat11w", O.csr_from_pairs(base.n, row[m], base.cols[m], w), True))
    out.append(("chunglu4k", O.gen_chunglu(4096, max_degree=400.0, seed=5), True))
    return out


# larger graphs whose reference traces are kept (generator, arguments)
TRACE_CASES = (
    ("sbm64k", "sbm", dict(n=65536, blocks=64, mean_degree=16.0, intra_frac=0.8, seed=1)),
    ("rmat16", "rmat", dict(scale=16, seed=2)),
)


def trace_graph(kind, kw):
    return O.gen_sbm(**kw) if kind == "sbm" else O.gen_rmat(**kw)


def graph_checksum(g):
    """Order-sensitive digest of a CSR (offsets and column ids), the same on every host."""
    import hashlib
    h = hashlib.sha256()
    h.update(np.asarray(g.offsets, np.uint64).tobytes())
    h.update(np.asarray(g.cols, np.uint32).tobytes())
    return h.hexdigest()


def make_traces(out):
    tmp = tempfile.mkdtemp()
    res = {}
    for name, kind, kw in TRACE_CASES:
        g = trace_graph(kind, kw)
        mtx = os.path.join(tmp, name + ".mtx")
        write_mtx(mtx, g, False)
        entry = {"generator": kind, "args": kw, "n": int(g.n), "nnz": int(len(g.cols)),
                 "sha256": graph_checksum(g), "trace": {}}
        for version in (0, 1, 2):
            entry["trace"][str(version)] = parse_table(run("louvain", mtx, version))
        res[name] = entry
        print("trace", name, g.n, len(g.cols), flush=True)
    with open(os.path.join(out, "traces.json"), "w") as f:
        json.dump(res, f, indent=1)


def states(g, k, mass):
    res = [("start", np.arange(g.n, dtype=np.uint32), k.copy())]
    C = np.arange(g.n, dtype=np.uint32)
    sig = k.copy()
    for it in range(3):
        Cn, _ = O.local_move(g, C, sig, k, mass, 2, it % 2 == 0)
        sig = np.zeros(g.n)
        np.add.at(sig, Cn, k)
        C = Cn
    res.append(("mid", C, sig))
    return res


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=HERE)
    ap.add_argument("--traces", action="store_true", help="only the larger graphs' printed tables")
    a = ap.parse_args()
    os.makedirs(a.out, exist_ok=True)
    if a.traces:
        make_traces(a.out)
        return
    tmp = tempfile.mkdtemp()
    for name, g, weighted in cases():
        mtx = os.path.join(tmp, name + ".mtx")
        write_mtx(mtx, g, weighted)
        arrays = {}
        meta = {"name": name, "weighted": weighted}
        # what the reference loaded (the engine and the oracle load the same file)
        run("load", mtx, os.path.join(tmp, "l.bin"))
        n, off, cols, w = read_graph(os.path.join(tmp, "l.bin"))
        arrays.update(load_offsets=off, load_cols=cols, load_weights=w)
        lg = O.CSR(n, off, cols, w)
        # bins, all schemes
        run("bins", mtx, os.path.join(tmp, "b.bin"))
        b = open(os.path.join(tmp, "b.bin"), "rb").read()
        o = 0
        for scheme in range(3):
            nb = int(np.frombuffer(b[o:o + 4], np.uint32)[0])
            o += 4
            arrays[f"bins{scheme}_sizes"] = np.frombuffer(b[o:o + 4 * nb], np.uint32).copy()
            o += 4 * nb
            arrays[f"bins{scheme}_offsets"] = np.frombuffer(b[o:o + 4 * nb], np.uint32).copy()
            o += 4 * nb
            arrays[f"bins{scheme}_maxdeg"] = np.frombuffer(b[o:o + 4], np.uint32).copy()
            o += 4
            nn = int(np.frombuffer(b[o:o + 4], np.uint32)[0])
            o += 4
            arrays[f"bins{scheme}_perm"] = np.frombuffer(b[o:o + 4 * nn], np.uint32).copy()
            o += 4 * nn
        # local move sweeps
        k = O.vertex_weights(lg)
        mass = O.mass(lg)
        for sname, C, sig in states(lg, k, mass):
            arrays[f"move_{sname}_C"] = C
            arrays[f"move_{sname}_sigma"] = sig
            arrays[f"move_{sname}_k"] = k
            for fn, arr in (("C", C), ("s", sig), ("k", k)):
                arr.tofile(os.path.join(tmp, fn + ".bin"))
            for version in (1, 2):
                for up in (1, 0):
                    run("move", mtx, os.path.join(tmp, "C.bin"), os.path.join(tmp, "s.bin"),
                        os.path.join(tmp, "k.bin"), up, version, os.path.join(tmp, "m.bin"))
                    r = np.fromfile(os.path.join(tmp, "m.bin"), np.uint32)
                    arrays[f"move_{sname}_v{version}_up{up}"] = r[1:]
        # coarsening by the mid-run assignment and by the final oracle assignment
        final = O.louvain(lg, max_phases=1)["assignment"]
        for cname, C in (("mid", arrays["move_mid_C"]), ("final", final)):
            arrays[f"coarsen_{cname}_C"] = C
            C.astype(np.uint32).tofile(os.path.join(tmp, "C.bin"))
            run("coarsen", mtx, os.path.join(tmp, "C.bin"), os.path.join(tmp, "c.bin"))
            n2, off2, cols2, w2 = read_graph(os.path.join(tmp, "c.bin"))
            arrays[f"coarsen_{cname}_offsets"] = off2
            arrays[f"coarsen_{cname}_cols"] = cols2
            arrays[f"coarsen_{cname}_weights"] = w2
        # full runs: the reference's printed tables
        meta["trace"] = {}
        for version in (0, 1, 2):
            meta["trace"][str(version)] = parse_table(run("louvain", mtx, version))
        np.savez_compressed(os.path.join(a.out, f"{name}.npz"), **arrays)
        spec = {"write_mtx": "lower triangle in CSR row order; pattern symmetric (unit) or real general (weighted)"}
        meta.update(spec)
        with open(os.path.join(a.out, f"{name}.json"), "w") as f:
            json.dump(meta, f, indent=1)
        print("golden", name, n, len(cols), flush=True)


if __name__ == "__main__":
    main()
