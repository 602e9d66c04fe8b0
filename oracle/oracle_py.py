"""ctypes front end of the CPU oracle (oracle/liboracle.so).

Test infrastructure only: imported by tests/, by ``__graft_entry__.smoke()``
as the checker and by ``bench.py``'s CPU baseline.  The product never
imports this module.
"""
from __future__ import annotations

import ctypes as ct
import os
import subprocess
from dataclasses import dataclass
from typing import Optional

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None


@dataclass
class CSR:
    """Symmetric CSR graph: offsets[n+1] uint64, cols[nnz] uint32, weights or None (unit)."""

    n: int
    offsets: np.ndarray
    cols: np.ndarray
    weights: Optional[np.ndarray] = None

    @property
    def nnz(self) -> int:
        return int(self.offsets[-1]) if len(self.offsets) else 0

    def degrees(self) -> np.ndarray:
        return np.diff(self.offsets)

    def weight_array(self) -> np.ndarray:
        if self.weights is None:
            return np.ones(self.nnz, dtype=np.float64)
        return self.weights

    def sorted_rows(self) -> "CSR":
        """Rows sorted by (col, weight): a canonical form for comparisons."""
        cols = self.cols.astype(np.uint32).copy()
        w = self.weight_array().astype(np.float64).copy()
        row = np.repeat(np.arange(self.n, dtype=np.uint64), np.diff(self.offsets).astype(np.int64))
        order = np.lexsort((w, cols, row))
        return CSR(self.n, self.offsets.copy(), cols[order], w[order])


class _OrGraph(ct.Structure):
    _fields_ = [
        ("n", ct.c_uint32),
        ("nnz", ct.c_uint64),
        ("offsets", ct.POINTER(ct.c_uint64)),
        ("cols", ct.POINTER(ct.c_uint32)),
        ("weights", ct.POINTER(ct.c_double)),
    ]


class _OrResult(ct.Structure):
    _fields_ = [
        ("modularity", ct.c_double),
        ("phases", ct.c_int),
        ("levels", ct.c_int),
        ("iterations", ct.c_int),
        ("trace_rows", ct.c_int),
        ("communities", ct.c_uint32),
    ]


def build() -> str:
    path = os.path.join(_HERE, "liboracle.so")
    src = os.path.join(_HERE, "oracle.c")
    if not os.path.exists(path) or os.path.getmtime(path) < os.path.getmtime(src):
        subprocess.check_call(["make", "-s", "-C", _HERE])
    return path


def lib():
    global _LIB
    if _LIB is None:
        _LIB = ct.CDLL(build())
        L = _LIB
        L.or_mix64.restype = ct.c_uint64
        L.or_mix64.argtypes = [ct.c_uint64]
        L.or_mass.restype = ct.c_double
        L.or_modularity.restype = ct.c_double
        L.or_modularity_sigma.restype = ct.c_double
        L.or_time_phase0.restype = ct.c_double
        L.or_gen_rmat.argtypes = [ct.c_int, ct.c_int, ct.c_double, ct.c_double, ct.c_double,
                                  ct.c_uint64, ct.POINTER(_OrGraph)]
        L.or_gen_sbm.argtypes = [ct.c_uint32, ct.c_uint32, ct.c_double, ct.c_double, ct.c_uint64,
                                 ct.POINTER(_OrGraph)]
        L.or_gen_chunglu.argtypes = [ct.c_uint32, ct.c_double, ct.c_double, ct.c_double, ct.c_int,
                                     ct.c_uint64, ct.POINTER(_OrGraph)]
        L.or_local_move.argtypes = [ct.POINTER(_OrGraph), ct.c_int, ct.c_int, ct.c_void_p, ct.c_void_p,
                                    ct.c_void_p, ct.c_double, ct.c_void_p, ct.POINTER(ct.c_uint64)]
        L.or_modularity_sigma.argtypes = [ct.POINTER(_OrGraph), ct.c_void_p, ct.c_void_p, ct.c_double,
                                          ct.c_int]
        L.or_louvain.argtypes = [ct.POINTER(_OrGraph), ct.c_int, ct.c_double, ct.c_int, ct.c_void_p,
                                 ct.c_void_p, ct.c_int, ct.c_void_p, ct.c_int, ct.POINTER(_OrResult)]
        L.or_time_phase0.argtypes = [ct.POINTER(_OrGraph), ct.c_int, ct.c_int, ct.POINTER(ct.c_uint64)]
    return _LIB


def _ptr(a):
    return a.ctypes.data_as(ct.c_void_p) if a is not None else None


class _Borrow:
    """or_graph view of a CSR (keeps the numpy arrays alive)."""

    def __init__(self, g: CSR):
        self.off = np.ascontiguousarray(g.offsets, dtype=np.uint64)
        self.cols = np.ascontiguousarray(g.cols, dtype=np.uint32)
        self.w = None if g.weights is None else np.ascontiguousarray(g.weights, dtype=np.float64)
        self.s = _OrGraph()
        self.s.n = g.n
        self.s.nnz = int(self.off[-1])
        self.s.offsets = self.off.ctypes.data_as(ct.POINTER(ct.c_uint64))
        self.s.cols = self.cols.ctypes.data_as(ct.POINTER(ct.c_uint32))
        self.s.weights = (self.w.ctypes.data_as(ct.POINTER(ct.c_double)) if self.w is not None
                          else ct.POINTER(ct.c_double)())

    def ref(self):
        return ct.byref(self.s)


def _take(s: _OrGraph) -> CSR:
    """Copy an oracle-allocated graph into numpy arrays and free it."""
    n, nnz = s.n, s.nnz
    off = np.ctypeslib.as_array(s.offsets, shape=(n + 1,)).copy()
    cols = np.ctypeslib.as_array(s.cols, shape=(max(nnz, 1),))[:nnz].copy()
    w = None
    if bool(s.weights):
        w = np.ctypeslib.as_array(s.weights, shape=(max(nnz, 1),))[:nnz].copy()
    lib().or_graph_free(ct.byref(s))
    return CSR(n, off, cols, w)


def set_threads(n: int) -> int:
    return lib().or_set_threads(int(n))


def get_threads() -> int:
    return int(lib().or_get_threads())


def mix64(x: int) -> int:
    return int(lib().or_mix64(x & 0xFFFFFFFFFFFFFFFF))


def load_mtx(path: str) -> CSR:
    s = _OrGraph()
    rc = lib().or_load_mtx(path.encode(), ct.byref(s))
    if rc != 0:
        raise ValueError(f"or_load_mtx({path}) failed: {rc}")
    return _take(s)


def gen_rmat(scale: int, edge_factor: int = 16, a=0.57, b=0.19, c=0.19, seed: int = 2) -> CSR:
    s = _OrGraph()
    rc = lib().or_gen_rmat(scale, edge_factor, a, b, c, seed, ct.byref(s))
    if rc != 0:
        raise ValueError(rc)
    return _take(s)


def gen_sbm(n: int, blocks: int, mean_degree: float = 16.0, intra_frac: float = 0.8, seed: int = 1) -> CSR:
    s = _OrGraph()
    rc = lib().or_gen_sbm(n, blocks, mean_degree, intra_frac, seed, ct.byref(s))
    if rc != 0:
        raise ValueError(rc)
    return _take(s)


def gen_chunglu(n: int, exponent=2.1, mean_degree=20.0, max_degree=200000.0, lognormal=True, seed=3) -> CSR:
    s = _OrGraph()
    rc = lib().or_gen_chunglu(n, exponent, mean_degree, max_degree, int(lognormal), seed, ct.byref(s))
    if rc != 0:
        raise ValueError(rc)
    return _take(s)


def csr_from_pairs(n: int, u, v, w=None) -> CSR:
    u = np.ascontiguousarray(u, dtype=np.uint32)
    v = np.ascontiguousarray(v, dtype=np.uint32)
    wa = None if w is None else np.ascontiguousarray(w, dtype=np.float64)
    s = _OrGraph()
    rc = lib().or_csr_from_pairs(ct.c_uint32(n), ct.c_uint64(len(u)), _ptr(u), _ptr(v), _ptr(wa), ct.byref(s))
    if rc != 0:
        raise ValueError(rc)
    return _take(s)


def bins(scheme: int, offsets) -> dict:
    off = np.ascontiguousarray(offsets, dtype=np.uint64)
    n = len(off) - 1
    sizes = np.zeros(11, np.uint32)
    boff = np.zeros(11, np.uint32)
    perm = np.zeros(max(n, 1), np.uint32)
    md = ct.c_uint32(0)
    rc = lib().or_bins(scheme, ct.c_uint32(n), _ptr(off), _ptr(sizes), _ptr(boff), _ptr(perm), ct.byref(md))
    if rc != 0:
        raise ValueError(rc)
    nb = {0: 10, 1: 11, 2: 9}[scheme]
    return {"sizes": sizes[:nb], "offsets": boff[:nb], "perm": perm[:n], "max_degree": int(md.value)}


def vertex_weights(g: CSR) -> np.ndarray:
    b = _Borrow(g)
    k = np.zeros(max(g.n, 1), np.float64)
    lib().or_vertex_weights(b.ref(), _ptr(k))
    return k[: g.n]


def mass(g: CSR) -> float:
    b = _Borrow(g)
    return float(lib().or_mass(b.ref()))


def is_integral(g: CSR) -> bool:
    b = _Borrow(g)
    return bool(lib().or_is_integral(b.ref()))


def local_move(g: CSR, C, sigma, k, mass_: float, version: int = 2, up: bool = True):
    b = _Borrow(g)
    C = np.ascontiguousarray(C, dtype=np.uint32)
    sigma = np.ascontiguousarray(sigma, dtype=np.float64)
    k = np.ascontiguousarray(k, dtype=np.float64)
    out = np.zeros(max(g.n, 1), np.uint32)
    d = ct.c_uint64(0)
    rc = lib().or_local_move(b.ref(), version, int(up), _ptr(C), _ptr(sigma), _ptr(k), mass_, _ptr(out),
                             ct.byref(d))
    if rc != 0:
        raise ValueError(rc)
    return out[: g.n], int(d.value)


def modularity_sigma(g: CSR, C, sigma, mass_: float, integral: bool) -> float:
    b = _Borrow(g)
    C = np.ascontiguousarray(C, dtype=np.uint32)
    sigma = np.ascontiguousarray(sigma, dtype=np.float64)
    return float(lib().or_modularity_sigma(b.ref(), _ptr(C), _ptr(sigma), mass_, int(integral)))


def modularity(g: CSR, C) -> float:
    b = _Borrow(g)
    C = np.ascontiguousarray(C, dtype=np.uint32)
    return float(lib().or_modularity(b.ref(), _ptr(C)))


def coarsen(g: CSR, C):
    b = _Borrow(g)
    C = np.ascontiguousarray(C, dtype=np.uint32)
    cd = np.zeros(max(g.n, 1), np.uint32)
    s = _OrGraph()
    up = np.zeros(g.n + 1, np.uint64)
    rc = lib().or_coarsen(b.ref(), _ptr(C), _ptr(cd), ct.byref(s), _ptr(up))
    if rc != 0:
        raise ValueError(rc)
    out = _take(s)
    return cd[: g.n], out, up[: out.n + 1]


def louvain(g: CSR, version: int = 2, threshold: float = 1e-6, max_phases: int = 1000, max_trace: int = 100000):
    b = _Borrow(g)
    assign = np.zeros(max(g.n, 1), np.uint32)
    trace = np.zeros((max_trace, 4), np.float64)
    levels = np.zeros(256, np.uint32)
    res = _OrResult()
    rc = lib().or_louvain(b.ref(), version, threshold, max_phases, _ptr(assign), _ptr(trace), max_trace,
                          _ptr(levels), 256, ct.byref(res))
    if rc != 0:
        raise ValueError(rc)
    rows = min(res.trace_rows, max_trace)
    return {
        "modularity": res.modularity,
        "phases": res.phases,
        "levels": res.levels,
        "iterations": res.iterations,
        "communities": res.communities,
        "level_sizes": levels[: min(res.levels, 256)].copy(),
        "trace": trace[:rows].copy(),
        "assignment": assign[: g.n].copy(),
    }


def time_phase0(g: CSR, version: int = 2, iters: int = 1):
    b = _Borrow(g)
    done = ct.c_uint64(0)
    t = float(lib().or_time_phase0(b.ref(), version, iters, ct.byref(done)))
    return t, int(done.value)
