"""Host-side Matrix Market loader (mg_csr_from_mtx): the reference's rules,
checked against the oracle's serial loader, plus the binary CSR cache.  No GPU."""
import os

import numpy as np
import pytest


def _write(path, banner, n, lines):
    with open(path, "w") as f:
        f.write(banner + "\n% comment\n")
        f.write(f"{n} {n} {len(lines)}\n")
        f.write("\n".join(lines))
        f.write("\n")


def _same(a, b):
    assert a["n"] == b.n
    assert (a["offsets"] == b.offsets).all()
    assert (a["cols"] == b.cols).all()
    if a["weights"] is None:
        assert b.weights is None or (b.weights == 1).all()
    else:
        assert (a["weights"] == b.weights).all()


def test_small_files_match_oracle(O, mg, tmp_path):
    sym = tmp_path / "s.mtx"
    sym.write_text("%%MatrixMarket matrix coordinate pattern symmetric\n% c\n5 5 6\n2 1\n3 1\n3 3\n4 2\n5 4\n5 1\n")
    a = mg.load_mtx(str(sym))
    assert a["weights"] is None and list(a["offsets"]) == [0, 3, 5, 7, 9, 11]
    _same(a, O.load_mtx(str(sym)))
    gen = tmp_path / "g.mtx"
    gen.write_text("%%MatrixMarket matrix coordinate real general\n5 5 7\n2 1 0.5\n1 2 0.5\n3 1 2.25\n3 3 9\n"
                   "4 2 1\n5 4 3\n5 1\n")
    a = mg.load_mtx(str(gen))
    _same(a, O.load_mtx(str(gen)))
    assert a["weights"].sum() == 2 * (0.5 + 2.25 + 1 + 3 + 1)


@pytest.mark.parametrize("symmetric", [True, False])
def test_multithreaded_parse_matches_oracle(O, mg, tmp_path, symmetric):
    """A file of several MiB (parsed in many chunks), entries in random order,
    diagonal entries and repeated rows: same CSR as the serial oracle."""
    g = O.gen_rmat(14, 16, seed=9)
    row = np.repeat(np.arange(g.n), np.diff(g.offsets).astype(np.int64))
    m = row > g.cols
    r, c = row[m], g.cols[m].astype(np.int64)
    rng = np.random.default_rng(4)
    p = rng.permutation(len(r))
    r, c = r[p], c[p]
    path = tmp_path / ("s.mtx" if symmetric else "g.mtx")
    if symmetric:
        diag = rng.choice(g.n, 50, replace=False)
        r = np.concatenate([r[:1000], diag, r[1000:]])
        c = np.concatenate([c[:1000], diag, c[1000:]])
        lines = [f"{x + 1} {y + 1}" for x, y in zip(r.tolist(), c.tolist())]
        _write(path, "%%MatrixMarket matrix coordinate pattern symmetric", g.n, lines)
    else:
        # both triangles and the diagonal are written; the loader keeps c < r
        w = rng.integers(1, 400, len(r)) / 8
        lines = [f"{x + 1} {y + 1} {v}" for x, y, v in zip(r.tolist(), c.tolist(), w.tolist())]
        lines += [f"{y + 1} {x + 1} 7" for x, y in zip(r[:500].tolist(), c[:500].tolist())]
        lines += [f"{x + 1} {x + 1} 5" for x in range(20)]
        _write(path, "%%MatrixMarket matrix coordinate real general", g.n, lines)
    assert os.path.getsize(path) > (1 << 20)  # parsed in one chunk per thread
    a = mg.load_mtx(str(path))
    assert a["weights"] is None if symmetric else a["weights"] is not None
    _same(a, O.load_mtx(str(path)))


def test_binary_cache_round_trip(O, mg, tmp_path):
    g = O.gen_sbm(3000, 10, 8.0, 0.8, seed=6)
    row = np.repeat(np.arange(g.n), np.diff(g.offsets).astype(np.int64))
    m = row > g.cols
    path = tmp_path / "c.mtx"
    rng = np.random.default_rng(2)
    lines = [f"{x + 1} {y + 1} {v}" for x, y, v in zip(row[m].tolist(), g.cols[m].tolist(),
                                                      (rng.integers(1, 100, m.sum()) / 4).tolist())]
    _write(path, "%%MatrixMarket matrix coordinate real general", g.n, lines)
    cache = str(path) + ".mgcsr"
    a = mg.load_mtx(str(path))
    assert not a["from_cache"] and not a["cache_written"] and not os.path.exists(cache)
    b = mg.load_mtx(str(path), cache_read=True, cache_write=True)
    assert not b["from_cache"] and b["cache_written"] and os.path.exists(cache)
    c = mg.load_mtx(str(path), cache_read=True)
    assert c["from_cache"]
    for x in (b, c):
        assert (x["offsets"] == a["offsets"]).all() and (x["cols"] == a["cols"]).all()
        assert (x["weights"] == a["weights"]).all()
    # a newer .mtx makes the cache stale
    st = os.stat(path)
    os.utime(path, ns=(st.st_atime_ns, st.st_mtime_ns + 1_000_000))
    assert not mg.load_mtx(str(path), cache_read=True)["from_cache"]
    # a rewritten cache is used again; a truncated one is ignored
    assert mg.load_mtx(str(path), cache_read=True, cache_write=True)["cache_written"]
    assert mg.load_mtx(str(path), cache_read=True)["from_cache"]
    with open(cache, "r+b") as f:
        f.truncate(os.path.getsize(cache) - 8)
    d = mg.load_mtx(str(path), cache_read=True)
    assert not d["from_cache"] and (d["cols"] == a["cols"]).all()


def test_symmetric_cache_has_no_weights(mg, tmp_path):
    path = tmp_path / "s.mtx"
    path.write_text("%%MatrixMarket matrix coordinate pattern symmetric\n4 4 3\n2 1\n3 2\n4 4\n")
    assert mg.load_mtx(str(path), cache_write=True)["cache_written"]
    a = mg.load_mtx(str(path), cache_read=True)
    assert a["from_cache"] and a["weights"] is None
    assert list(a["offsets"]) == [0, 1, 3, 4, 5] and list(a["cols"]) == [1, 0, 2, 1, 3]


def test_malformed_files(mg, tmp_path):
    cases = {
        "count": "%%MatrixMarket matrix coordinate pattern symmetric\n3 3 2\n2 1\n",
        "range": "%%MatrixMarket matrix coordinate pattern symmetric\n3 3 1\n4 1\n",
        "zero": "%%MatrixMarket matrix coordinate pattern symmetric\n3 3 1\n0 1\n",
        "nospace": "%%MatrixMarket matrix coordinate pattern symmetric\n3 3 1\n21\n",
        "size": "%%MatrixMarket matrix coordinate pattern symmetric\nthree\n",
        "empty": "",
    }
    for name, text in cases.items():
        p = tmp_path / f"{name}.mtx"
        p.write_text(text)
        with pytest.raises(mg.MGError) as e:
            mg.load_mtx(str(p))
        assert e.value.status == 5, name  # MG_ERR_FORMAT
    with pytest.raises(mg.MGError) as e:
        mg.load_mtx(str(tmp_path / "missing.mtx"))
    assert e.value.status == 4  # MG_ERR_IO


def test_crlf_and_blank_padding_match_oracle(O, mg, tmp_path):
    """Windows line ends and spaces before the first field: the same entries as
    the oracle's atoi/atof reading.  A leading space is the "first space" of
    the reference's field rule, so " 3 1 2.25" reads as row 3, column 3 (a
    diagonal entry, dropped on the general path), as the reference does."""
    text = ("%%MatrixMarket matrix coordinate real general\r\n% c\r\n6 6 6\r\n"
            "2 1 0.5\r\n 3 1 2.25\r\n4 2 1\r\n  5 4 3\r\n6 5\r\n6 1 7.5\r\n")
    p = tmp_path / "crlf.mtx"
    p.write_bytes(text.encode())
    a = mg.load_mtx(str(p))
    _same(a, O.load_mtx(str(p)))
    assert a["weights"].sum() == 2 * (0.5 + 1 + 1 + 7.5)
