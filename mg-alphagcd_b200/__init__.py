"""Python front end of the B200 Louvain engine (ctypes over libmgagcd.so).

The engine itself is CUDA C++ behind the C ABI in include/mgagcd.h; this
module only marshals numpy arrays.  It fails loudly when the shared library
is missing -- there is no CPU fallback.

The directory name is not a Python identifier; load it with
``importlib.import_module("mg-alphagcd_b200")`` after putting the repository
root on ``sys.path``.

Interfaces mirror the reference's stage boundaries (MG-alphaGCD):
  Graph.from_mtx          -> loadMMSparseMatrix        (src/mmio/mmio_wrapper.cu:297)
  Graph.bins              -> BIN::bin_create x3         (src/bin/BIN.cu:468-575)
  Graph.local_move        -> calculate_eicj_and_move_vertex_bin (src/louvain/louvain.cu:1032)
  Graph.modularity        -> compute_modularity         (src/louvain/louvain.cu:105-238)
  Graph.coarsen           -> coarsen_graph_mg::coarsen_graph (src/coarsen_graph/coarsen_graph_mg.cu:2054)
  Graph.louvain           -> louvain::run               (src/louvain/louvain.cu:1401)
  Batch.run               -> louvain::run for every graph of a packed batch (no reference
                             counterpart: the reference runs one graph per process)
"""
from __future__ import annotations

import ctypes as ct
import os
import weakref
from typing import Optional

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libmgagcd.so")
CLI_PATH = os.path.join(_HERE, "MG_GCD")

MG_OK = 0
WEIGHT_UNIT, WEIGHT_F32, WEIGHT_F64 = 0, 1, 2
PREC_FP64, PREC_INT64, PREC_FP32 = 0, 1, 2
_PREC = {"fp64": PREC_FP64, "int64": PREC_INT64, "fp32": PREC_FP32}

_lib = None


class MGError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"[{status}] {msg}")
        self.status = status


class _Opts(ct.Structure):
    _fields_ = [("device", ct.c_int), ("verbose", ct.c_int), ("hbm_budget_bytes", ct.c_size_t)]


class _SweepOpts(ct.Structure):
    _fields_ = [("cluster_fill", ct.c_int), ("giant_class", ct.c_int), ("coarsen_combine", ct.c_int),
                ("light_streams", ct.c_int), ("table_first_sweep", ct.c_int)]


class _RunOpts(ct.Structure):
    _fields_ = [("version", ct.c_int), ("threshold", ct.c_double), ("max_phases", ct.c_int),
                ("precision", ct.c_int), ("verbose", ct.c_int), ("keep_levels", ct.c_int)]


class _Summary(ct.Structure):
    _fields_ = [("modularity", ct.c_double), ("phases", ct.c_int), ("levels", ct.c_int),
                ("iterations", ct.c_int), ("communities", ct.c_uint32), ("seconds_total", ct.c_double),
                ("seconds_local_move", ct.c_double), ("seconds_coarsen", ct.c_double),
                ("edges_swept", ct.c_uint64), ("phase0_edges_swept", ct.c_uint64),
                ("phase0_seconds", ct.c_double), ("distinct_pairs", ct.c_uint64),
                ("seconds_sweep_kernels", ct.c_double), ("sweep_bytes", ct.c_double),
                ("kernel_launches", ct.c_uint64), ("sweeps", ct.c_uint64)]


class SbmParams(ct.Structure):
    _fields_ = [("n", ct.c_uint32), ("blocks", ct.c_uint32), ("mean_degree", ct.c_double),
                ("intra_frac", ct.c_double), ("seed", ct.c_uint64)]


class _BatchGraph(ct.Structure):
    _fields_ = [("modularity", ct.c_double), ("n", ct.c_uint32), ("nnz", ct.c_uint64), ("phases", ct.c_int),
                ("levels", ct.c_int), ("iterations", ct.c_uint64), ("communities", ct.c_uint32)]


class GenParams(ct.Structure):
    _fields_ = [("kind", ct.c_int), ("n", ct.c_uint32), ("blocks", ct.c_uint32), ("mean_degree", ct.c_double),
                ("intra_frac", ct.c_double), ("scale", ct.c_int), ("edge_factor", ct.c_int), ("a", ct.c_double),
                ("b", ct.c_double), ("c", ct.c_double), ("seed", ct.c_uint64)]


class _ServeOpts(ct.Structure):
    _fields_ = [("device", ct.c_int), ("slots", ct.c_int), ("hbm_budget_bytes", ct.c_size_t),
                ("max_batch_jobs", ct.c_uint32), ("batch_flags", ct.c_int)]


class _JobInfo(ct.Structure):
    _fields_ = [("state", ct.c_int), ("status", ct.c_int), ("graph", _BatchGraph), ("submitted_s", ct.c_double),
                ("started_s", ct.c_double), ("finished_s", ct.c_double), ("batch", ct.c_uint64),
                ("batch_jobs", ct.c_uint32)]


class _ServeCounters(ct.Structure):
    _fields_ = [("submitted", ct.c_uint64), ("completed", ct.c_uint64), ("failed", ct.c_uint64),
                ("cancelled", ct.c_uint64), ("queued", ct.c_uint64), ("running", ct.c_uint64),
                ("batches", ct.c_uint64), ("elapsed_s", ct.c_double), ("jobs_per_s", ct.c_double),
                ("p50_latency_s", ct.c_double), ("p99_latency_s", ct.c_double), ("mean_latency_s", ct.c_double),
                ("max_latency_s", ct.c_double), ("budget_bytes", ct.c_size_t), ("reserved_bytes", ct.c_size_t)]


BATCH_GRAPHS = 1
GEN_SBM, GEN_RMAT = 0, 1
JOB_QUEUED, JOB_RUNNING, JOB_DONE, JOB_FAILED, JOB_CANCELLED = 0, 1, 2, 3, 4
MG_ERR_TIMEOUT = 7

EXPORTED = [
    "mg_status_string", "mg_version", "mg_init", "mg_destroy", "mg_last_error", "mg_graph_from_csr",
    "mg_graph_from_device_csr", "mg_graph_from_mtx", "mg_graph_generate_rmat", "mg_graph_generate_sbm",
    "mg_graph_info", "mg_graph_properties", "mg_graph_copy_csr", "mg_graph_destroy", "mg_bins", "mg_bins_offsets", "mg_local_move",
    "mg_modularity", "mg_coarsen", "mg_louvain_run", "mg_result_summary", "mg_result_assignment",
    "mg_result_level_sizes", "mg_result_trace", "mg_result_destroy", "mg_local_move_noalloc",
    "mg_batch_draw_sbm_params", "mg_batch_generate_sbm", "mg_batch_from_csr", "mg_batch_info",
    "mg_batch_graph_info", "mg_batch_destroy", "mg_batch_run", "mg_batch_result_summary", "mg_batch_result_graph",
    "mg_batch_result_assignment", "mg_batch_result_destroy", "mg_batch_generate", "mg_serve_start",
    "mg_serve_submit", "mg_serve_submit_csr", "mg_serve_poll", "mg_serve_wait", "mg_serve_assignment",
    "mg_serve_cancel", "mg_serve_release", "mg_serve_stats", "mg_serve_last_error", "mg_serve_stop",
    "mg_tune_mode", "mg_tune_table", "mg_tune_save", "mg_tune_load", "mg_graph_generate_chunglu",
    "mg_graph_from_mtx_ex", "mg_csr_from_mtx", "mg_csr_info", "mg_csr_arrays", "mg_csr_free",
    "mg_result_level_map", "mg_result_level_csr", "mg_sweep_options", "mg_test_fail_allocation",
]
TUNE_OFF, TUNE_CACHED, TUNE_ON = 0, 1, 2
FILL_AUTO, FILL_OWN, FILL_SPLIT = 0, 1, 2
COMBINE_AUTO, COMBINE_OFF, COMBINE_ON = 0, 1, 2
LOAD_CACHE_READ, LOAD_CACHE_WRITE = 1, 2


def lib():
    """Load libmgagcd.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is missing: build it with `python mg-alphagcd_b200/build.py` "
                           "(the engine has no CPU fallback)")
    L = ct.CDLL(LIB_PATH)
    vp, u32, u64, i32, dbl = ct.c_void_p, ct.c_uint32, ct.c_uint64, ct.c_int, ct.c_double
    pp = ct.POINTER(ct.c_void_p)
    L.mg_status_string.restype = ct.c_char_p
    L.mg_status_string.argtypes = [i32]
    L.mg_version.restype = ct.c_char_p
    L.mg_last_error.restype = ct.c_char_p
    L.mg_last_error.argtypes = [vp]
    L.mg_init.argtypes = [pp, ct.POINTER(_Opts)]
    L.mg_destroy.argtypes = [vp]
    L.mg_graph_from_csr.argtypes = [vp, u32, vp, vp, vp, i32, pp]
    L.mg_graph_from_device_csr.argtypes = [vp, u32, u64, vp, vp, vp, i32, pp]
    L.mg_graph_from_mtx.argtypes = [vp, ct.c_char_p, pp]
    L.mg_graph_from_mtx_ex.argtypes = [vp, ct.c_char_p, i32, pp]
    L.mg_csr_from_mtx.argtypes = [ct.c_char_p, i32, pp]
    L.mg_csr_info.argtypes = [vp, ct.POINTER(u32), ct.POINTER(u64), ct.POINTER(i32), ct.POINTER(i32),
                              ct.POINTER(i32)]
    L.mg_csr_arrays.argtypes = [vp, pp, pp, pp]
    L.mg_csr_free.argtypes = [vp]
    L.mg_graph_generate_rmat.argtypes = [vp, i32, i32, dbl, dbl, dbl, u64, pp]
    L.mg_graph_generate_sbm.argtypes = [vp, u32, u32, dbl, dbl, u64, pp]
    L.mg_graph_generate_chunglu.argtypes = [vp, u32, dbl, dbl, dbl, i32, u64, pp]
    L.mg_graph_info.argtypes = [vp, ct.POINTER(u32), ct.POINTER(u64), ct.POINTER(dbl), ct.POINTER(i32)]
    L.mg_graph_properties.argtypes = [vp, ct.POINTER(i32), ct.POINTER(i32)]
    L.mg_graph_copy_csr.argtypes = [vp, vp, vp, vp]
    L.mg_graph_destroy.argtypes = [vp]
    L.mg_bins.argtypes = [vp, i32, vp, vp, vp, ct.POINTER(u32)]
    L.mg_bins_offsets.argtypes = [vp, i32, u32, vp, vp, vp, vp, ct.POINTER(u32)]
    L.mg_local_move.argtypes = [vp, i32, i32, i32, vp, vp, vp, vp, ct.POINTER(u64)]
    L.mg_modularity.argtypes = [vp, vp, ct.POINTER(dbl)]
    L.mg_coarsen.argtypes = [vp, vp, vp, pp]
    L.mg_louvain_run.argtypes = [vp, ct.POINTER(_RunOpts), pp]
    L.mg_result_summary.argtypes = [vp, ct.POINTER(_Summary)]
    L.mg_result_assignment.argtypes = [vp, vp]
    L.mg_result_level_sizes.argtypes = [vp, vp, i32, ct.POINTER(i32)]
    L.mg_result_trace.argtypes = [vp, vp, i32, ct.POINTER(i32)]
    L.mg_result_level_map.argtypes = [vp, i32, vp, u32, ct.POINTER(u32)]
    L.mg_result_level_csr.argtypes = [vp, i32, ct.POINTER(u32), ct.POINTER(u64), vp, vp, vp]
    L.mg_result_destroy.argtypes = [vp]
    L.mg_batch_draw_sbm_params.argtypes = [u32, u32, u32, u32, u32, dbl, dbl, dbl, dbl, u64, vp]
    L.mg_batch_generate_sbm.argtypes = [vp, u32, vp, pp]
    L.mg_batch_from_csr.argtypes = [vp, u32, vp, vp, vp, vp, i32, pp]
    L.mg_batch_info.argtypes = [vp, ct.POINTER(u32), ct.POINTER(u64), ct.POINTER(u64)]
    L.mg_batch_graph_info.argtypes = [vp, u32, ct.POINTER(u32), ct.POINTER(u64), ct.POINTER(dbl)]
    L.mg_batch_destroy.argtypes = [vp]
    L.mg_batch_run.argtypes = [vp, ct.POINTER(_RunOpts), i32, pp]
    L.mg_batch_result_summary.argtypes = [vp, ct.POINTER(_Summary)]
    L.mg_batch_result_graph.argtypes = [vp, u32, ct.POINTER(_BatchGraph)]
    L.mg_batch_result_assignment.argtypes = [vp, u32, vp]
    L.mg_batch_result_destroy.argtypes = [vp]
    L.mg_batch_generate.argtypes = [vp, u32, vp, pp]
    L.mg_tune_mode.argtypes = [vp, i32]
    L.mg_sweep_options.argtypes = [vp, ct.POINTER(_SweepOpts)]
    L.mg_test_fail_allocation.argtypes = [u64, ct.POINTER(u64)]
    L.mg_tune_table.argtypes = [vp, ct.c_char_p, ct.c_size_t, ct.POINTER(ct.c_size_t)]
    L.mg_tune_save.argtypes = [vp, ct.c_char_p]
    L.mg_tune_load.argtypes = [vp, ct.c_char_p]
    L.mg_serve_start.argtypes = [ct.POINTER(_ServeOpts), pp]
    L.mg_serve_submit.argtypes = [vp, ct.POINTER(GenParams), ct.POINTER(_RunOpts), i32, ct.POINTER(u64)]
    L.mg_serve_submit_csr.argtypes = [vp, u32, vp, vp, vp, i32, ct.POINTER(_RunOpts), i32, ct.POINTER(u64)]
    L.mg_serve_poll.argtypes = [vp, u64, ct.POINTER(_JobInfo)]
    L.mg_serve_wait.argtypes = [vp, u64, dbl, ct.POINTER(_JobInfo)]
    L.mg_serve_assignment.argtypes = [vp, u64, vp]
    L.mg_serve_cancel.argtypes = [vp, u64]
    L.mg_serve_release.argtypes = [vp, u64]
    L.mg_serve_stats.argtypes = [vp, ct.POINTER(_ServeCounters)]
    L.mg_serve_last_error.restype = ct.c_char_p
    L.mg_serve_last_error.argtypes = [vp]
    L.mg_serve_stop.argtypes = [vp]
    _lib = L
    return L


def _p(a: Optional[np.ndarray]):
    return None if a is None else a.ctypes.data_as(ct.c_void_p)


class Context:
    """A CUDA device context of the engine (mg_init / mg_destroy)."""

    def __init__(self, device: int = 0, verbose: bool = False):
        self.h = ct.c_void_p()
        opts = _Opts(device, int(verbose), 0)
        st = lib().mg_init(ct.byref(self.h), ct.byref(opts))
        if st != MG_OK:
            raise MGError(st, lib().mg_last_error(None).decode())

    def check(self, st: int, what: str):
        if st != MG_OK:
            raise MGError(st, f"{what}: {lib().mg_last_error(self.h).decode()}")

    def close(self):
        """Destroy the context -- after the graphs and batches made on it,
        which the C ABI requires to go first (they use its streams)."""
        if self.h:
            for child in list(getattr(self, "_children", ())):
                child.close()
            lib().mg_destroy(self.h)
            self.h = ct.c_void_p()

    def _adopt(self, child):
        if not hasattr(self, "_children"):
            self._children = weakref.WeakSet()
        self._children.add(child)
        return child

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- graph constructors ----------------------------------------------
    def graph_from_csr(self, n: int, offsets, cols, weights=None) -> "Graph":
        off = np.ascontiguousarray(offsets, dtype=np.uint64)
        col = np.ascontiguousarray(cols, dtype=np.uint32)
        if weights is None:
            w, wt = None, WEIGHT_UNIT
        elif np.asarray(weights).dtype == np.float32:
            w, wt = np.ascontiguousarray(weights, dtype=np.float32), WEIGHT_F32
        else:
            w, wt = np.ascontiguousarray(weights, dtype=np.float64), WEIGHT_F64
        h = ct.c_void_p()
        self.check(lib().mg_graph_from_csr(self.h, n, _p(off), _p(col), _p(w), wt, ct.byref(h)),
                   "mg_graph_from_csr")
        return Graph(self, h)

    def graph_from_mtx(self, path: str, cache_read: bool = False, cache_write: bool = False) -> "Graph":
        """Load a Matrix Market file (mg_graph_from_mtx; with the binary CSR
        cache flags, mg_graph_from_mtx_ex)."""
        h = ct.c_void_p()
        flags = (LOAD_CACHE_READ if cache_read else 0) | (LOAD_CACHE_WRITE if cache_write else 0)
        if flags:
            self.check(lib().mg_graph_from_mtx_ex(self.h, path.encode(), flags, ct.byref(h)), "mg_graph_from_mtx_ex")
        else:
            self.check(lib().mg_graph_from_mtx(self.h, path.encode(), ct.byref(h)), "mg_graph_from_mtx")
        return Graph(self, h)

    def generate_rmat(self, scale: int, edge_factor: int = 16, a=0.57, b=0.19, c=0.19, seed: int = 2) -> "Graph":
        h = ct.c_void_p()
        self.check(lib().mg_graph_generate_rmat(self.h, scale, edge_factor, a, b, c, seed, ct.byref(h)),
                   "mg_graph_generate_rmat")
        return Graph(self, h)

    def generate_sbm(self, n: int, blocks: int, mean_degree: float = 16.0, intra_frac: float = 0.8,
                     seed: int = 1) -> "Graph":
        h = ct.c_void_p()
        self.check(lib().mg_graph_generate_sbm(self.h, n, blocks, mean_degree, intra_frac, seed, ct.byref(h)),
                   "mg_graph_generate_sbm")
        return Graph(self, h)

    def generate_chunglu(self, n: int, exponent: float = 2.1, mean_degree: float = 20.0,
                         max_degree: float = 200000.0, lognormal: bool = True, seed: int = 3) -> "Graph":
        h = ct.c_void_p()
        self.check(lib().mg_graph_generate_chunglu(self.h, n, exponent, mean_degree, max_degree, int(lognormal), seed,
                                                   ct.byref(h)), "mg_graph_generate_chunglu")
        return Graph(self, h)

    def bins_offsets(self, scheme: int, offsets) -> dict:
        off = np.ascontiguousarray(offsets, dtype=np.uint64)
        n = len(off) - 1
        sizes = np.zeros(11, np.uint32)
        boff = np.zeros(11, np.uint32)
        perm = np.zeros(max(n, 1), np.uint32)
        md = ct.c_uint32()
        self.check(lib().mg_bins_offsets(self.h, scheme, n, _p(off), _p(sizes), _p(boff), _p(perm), ct.byref(md)),
                   "mg_bins_offsets")
        nb = {0: 10, 1: 11, 2: 9}[scheme]
        return {"sizes": sizes[:nb], "offsets": boff[:nb], "perm": perm[:n], "max_degree": int(md.value)}


    # ---- autotuner ------------------------------------------------------------
    def tune_mode(self, mode: int):
        """TUNE_OFF: built-in shapes; TUNE_CACHED: table only; TUNE_ON: also time new classes."""
        self.check(lib().mg_tune_mode(self.h, mode), "mg_tune_mode")

    def sweep_options(self, cluster_fill: int = FILL_AUTO, giant_class: int = 0,
                      coarsen_combine: int = COMBINE_AUTO, light_streams: int = 0,
                      table_first_sweep: bool = False):
        """Sweep and coarsening policy (mg_sweep_options): the cluster-table
        fill (FILL_*), the first degree class (13..18, 0 = default) sent to
        the global-table path, and warp combining of equal keys in the
        coarsening (COMBINE_*), and the number of streams the light degree
        classes are spread over (1..7, 0 = default 2), and whether a level's
        first sweep uses the table kernels (default: table-free kernels).
        Results do not depend on it."""
        o = _SweepOpts(cluster_fill, giant_class, coarsen_combine, light_streams, int(table_first_sweep))
        self.check(lib().mg_sweep_options(self.h, ct.byref(o)), "mg_sweep_options")

    def tune_table(self) -> list:
        """Entries: (weight kind, precision, version, batched, class, size bucket, shape, microseconds)."""
        n = ct.c_size_t()
        self.check(lib().mg_tune_table(self.h, None, 0, ct.byref(n)), "mg_tune_table")
        buf = ct.create_string_buffer(n.value + 1)
        self.check(lib().mg_tune_table(self.h, buf, n.value + 1, ct.byref(n)), "mg_tune_table")
        out = []
        for line in buf.value.decode().splitlines():
            f = line.split()
            out.append(tuple(int(x) for x in f[:6]) + (f[6], float(f[7])))
        return out

    def tune_save(self, path: str):
        self.check(lib().mg_tune_save(self.h, path.encode()), "mg_tune_save")

    def tune_load(self, path: str):
        self.check(lib().mg_tune_load(self.h, path.encode()), "mg_tune_load")

    # ---- batches ------------------------------------------------------------
    def batch_generate_sbm(self, params) -> "Batch":
        """Batch of seeded SBMs; graph g equals generate_sbm(**params[g])."""
        arr = (SbmParams * len(params))(*[p if isinstance(p, SbmParams) else SbmParams(
            p["n"], p["blocks"], p["mean_degree"], p["intra_frac"], p["seed"]) for p in params])
        h = ct.c_void_p()
        self.check(lib().mg_batch_generate_sbm(self.h, len(params), ct.cast(arr, ct.c_void_p), ct.byref(h)),
                   "mg_batch_generate_sbm")
        return Batch(self, h)

    def batch_generate(self, params) -> "Batch":
        """Batch of generated graphs [GenParams, ...] (SBM and R-MAT mixed)."""
        arr = (GenParams * len(params))(*params)
        h = ct.c_void_p()
        self.check(lib().mg_batch_generate(self.h, len(params), ct.cast(arr, ct.c_void_p), ct.byref(h)),
                   "mg_batch_generate")
        return Batch(self, h)

    def batch_from_csr(self, graphs) -> "Batch":
        """Pack host graphs [(n, offsets, cols, weights|None), ...] (local ids)."""
        G = len(graphs)
        voff = np.zeros(G + 1, np.uint64)
        for g, (n, _, _, _) in enumerate(graphs):
            voff[g + 1] = voff[g] + n
        total = int(voff[-1])
        off = np.zeros(total + 1, np.uint64)
        cols, ws = [], []
        base = 0
        weighted = any(w is not None for _, _, _, w in graphs)
        f32 = weighted and all(w is None or np.asarray(w).dtype == np.float32 for _, _, _, w in graphs)
        for g, (n, o, c, w) in enumerate(graphs):
            o = np.asarray(o, np.uint64)
            off[int(voff[g]) + 1: int(voff[g]) + n + 1] = o[1:] + base
            cols.append(np.asarray(c, np.uint32))
            if weighted:
                ws.append(np.ones(len(c)) if w is None else np.asarray(w, np.float64))
            base += int(o[-1])
        col = np.ascontiguousarray(np.concatenate(cols) if cols else np.zeros(0, np.uint32), dtype=np.uint32)
        if weighted:
            wt = WEIGHT_F32 if f32 else WEIGHT_F64
            w = np.ascontiguousarray(np.concatenate(ws), dtype=np.float32 if f32 else np.float64)
        else:
            wt, w = WEIGHT_UNIT, None
        h = ct.c_void_p()
        self.check(lib().mg_batch_from_csr(self.h, G, _p(voff), _p(off), _p(col), _p(w), wt, ct.byref(h)),
                   "mg_batch_from_csr")
        return Batch(self, h)


def gen_params(kind: str, **kw) -> GenParams:
    """A generated job: gen_params("sbm", n=, blocks=, mean_degree=, intra_frac=, seed=) or
    gen_params("rmat", scale=, edge_factor=16, a=.57, b=.19, c=.19, seed=)."""
    if kind == "sbm":
        return GenParams(GEN_SBM, kw["n"], kw["blocks"], kw.get("mean_degree", 16.0), kw.get("intra_frac", 0.8),
                         0, 0, 0.0, 0.0, 0.0, kw.get("seed", 1))
    return GenParams(GEN_RMAT, 0, 0, 0.0, 0.0, kw["scale"], kw.get("edge_factor", 16), kw.get("a", 0.57),
                     kw.get("b", 0.19), kw.get("c", 0.19), kw.get("seed", 2))


class Server:
    """Continuous-batching Louvain server (mg_serve_*): thread-safe submit / wait."""

    def __init__(self, device: int = 0, slots: int = 4, hbm_budget_bytes: int = 150 * 10**9,
                 max_batch_jobs: int = 4096, graphs: bool = True):
        self.h = ct.c_void_p()
        o = _ServeOpts(device, slots, hbm_budget_bytes, max_batch_jobs, BATCH_GRAPHS if graphs else 0)
        st = lib().mg_serve_start(ct.byref(o), ct.byref(self.h))
        if st != MG_OK:
            raise MGError(st, lib().mg_last_error(None).decode())

    def _check(self, st, what):
        if st != MG_OK:
            raise MGError(st, f"{what}: {lib().mg_serve_last_error(self.h).decode()}")

    def submit(self, job: GenParams, keep_assignment: bool = False, version: int = 2, threshold: float = 1e-6,
               max_phases: int = 1000, precision: str = "fp64") -> int:
        o = _RunOpts(version, threshold, max_phases, _PREC[precision], 0)
        jid = ct.c_uint64()
        self._check(lib().mg_serve_submit(self.h, ct.byref(job), ct.byref(o), int(keep_assignment), ct.byref(jid)),
                    "mg_serve_submit")
        return jid.value

    def submit_csr(self, n, offsets, cols, weights=None, keep_assignment: bool = False, **run) -> int:
        off = np.ascontiguousarray(offsets, dtype=np.uint64)
        col = np.ascontiguousarray(cols, dtype=np.uint32)
        w, wt = (None, WEIGHT_UNIT) if weights is None else (np.ascontiguousarray(weights, np.float64), WEIGHT_F64)
        o = _RunOpts(run.get("version", 2), run.get("threshold", 1e-6), run.get("max_phases", 1000),
                     _PREC[run.get("precision", "fp64")], 0)
        jid = ct.c_uint64()
        self._check(lib().mg_serve_submit_csr(self.h, n, _p(off), _p(col), _p(w), wt, ct.byref(o),
                                              int(keep_assignment), ct.byref(jid)), "mg_serve_submit_csr")
        return jid.value

    @staticmethod
    def _info(i: _JobInfo) -> dict:
        d = {f: getattr(i, f) for f, _ in _JobInfo._fields_ if f != "graph"}
        d.update({f: getattr(i.graph, f) for f, _ in _BatchGraph._fields_})
        return d

    def poll(self, jid: int) -> dict:
        i = _JobInfo()
        self._check(lib().mg_serve_poll(self.h, jid, ct.byref(i)), "mg_serve_poll")
        return self._info(i)

    def wait(self, jid: int, timeout: float = 600.0) -> dict:
        i = _JobInfo()
        st = lib().mg_serve_wait(self.h, jid, timeout, ct.byref(i))
        if st == MG_ERR_TIMEOUT:
            raise TimeoutError(f"job {jid} not done after {timeout} s")
        self._check(st, "mg_serve_wait")
        return self._info(i)

    def assignment(self, jid: int, n: int) -> np.ndarray:
        a = np.zeros(max(n, 1), np.uint32)
        self._check(lib().mg_serve_assignment(self.h, jid, _p(a)), "mg_serve_assignment")
        return a[:n]

    def cancel(self, jid: int) -> bool:
        return lib().mg_serve_cancel(self.h, jid) == MG_OK

    def release(self, jid: int) -> bool:
        return lib().mg_serve_release(self.h, jid) == MG_OK

    def stats(self) -> dict:
        c = _ServeCounters()
        self._check(lib().mg_serve_stats(self.h, ct.byref(c)), "mg_serve_stats")
        return {f: getattr(c, f) for f, _ in _ServeCounters._fields_}

    def stop(self):
        if self.h:
            lib().mg_serve_stop(self.h)
            self.h = ct.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.stop()

    def __del__(self):
        try:
            self.stop()
        except Exception:
            pass


def fail_allocation(nth: int) -> int:
    """Test hook (mg_test_fail_allocation): the nth device allocation of the
    library from now on fails as out of memory (0 disarms).  Returns what was
    left of the previous countdown (0: it fired, or was not armed)."""
    left = ct.c_uint64()
    lib().mg_test_fail_allocation(nth, ct.byref(left))
    return int(left.value)


def load_mtx(path: str, cache_read: bool = False, cache_write: bool = False) -> dict:
    """Parse a Matrix Market file on the host (mg_csr_from_mtx; no GPU needed).

    Returns {"n", "offsets" (uint64), "cols" (uint32), "weights" (float64 or
    None for unit weights), "from_cache", "cache_written"}; the arrays are
    copies."""
    L = lib()
    h = ct.c_void_p()
    flags = (LOAD_CACHE_READ if cache_read else 0) | (LOAD_CACHE_WRITE if cache_write else 0)
    st = L.mg_csr_from_mtx(path.encode(), flags, ct.byref(h))
    if st != MG_OK:
        raise MGError(st, L.mg_last_error(None).decode())
    try:
        n, nnz = ct.c_uint32(), ct.c_uint64()
        wt, fc, cw = ct.c_int(), ct.c_int(), ct.c_int()
        L.mg_csr_info(h, ct.byref(n), ct.byref(nnz), ct.byref(wt), ct.byref(fc), ct.byref(cw))
        po, pc, pw = ct.c_void_p(), ct.c_void_p(), ct.c_void_p()
        L.mg_csr_arrays(h, ct.byref(po), ct.byref(pc), ct.byref(pw))

        def copy(ptr, count, ctype, dtype):
            if count == 0:
                return np.zeros(0, dtype)
            return np.ctypeslib.as_array(ct.cast(ptr, ct.POINTER(ctype)), (count,)).astype(dtype, copy=True)

        off = copy(po, n.value + 1, ct.c_uint64, np.uint64)
        cols = copy(pc, nnz.value, ct.c_uint32, np.uint32)
        w = copy(pw, nnz.value, ct.c_double, np.float64) if wt.value else None
        return {"n": n.value, "offsets": off, "cols": cols, "weights": w, "from_cache": bool(fc.value),
                "cache_written": bool(cw.value)}
    finally:
        L.mg_csr_free(h)


def draw_sbm_params(graphs: int, n_range=(1000, 200000), blocks_range=(4, 256), deg_range=(8.0, 32.0),
                    intra_range=(0.7, 0.9), seed: int = 4) -> list:
    """Per-graph SBM parameters of a batch (mg_batch_draw_sbm_params)."""
    arr = (SbmParams * max(graphs, 1))()
    st = lib().mg_batch_draw_sbm_params(graphs, n_range[0], n_range[1], blocks_range[0], blocks_range[1],
                                        deg_range[0], deg_range[1], intra_range[0], intra_range[1], seed,
                                        ct.cast(arr, ct.c_void_p))
    if st != MG_OK:
        raise MGError(st, lib().mg_last_error(None).decode())
    return [{"n": p.n, "blocks": p.blocks, "mean_degree": p.mean_degree, "intra_frac": p.intra_frac,
             "seed": p.seed} for p in arr[:graphs]]


class Batch:
    """Many graphs packed on the device (mg_batch)."""

    def __init__(self, ctx: Context, h: ct.c_void_p):
        self.ctx = ctx
        self.h = h
        ctx._adopt(self)

    def close(self):
        if self.h:
            lib().mg_batch_destroy(self.h)
            self.h = ct.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def info(self) -> dict:
        g, n, nnz = ct.c_uint32(), ct.c_uint64(), ct.c_uint64()
        self.ctx.check(lib().mg_batch_info(self.h, ct.byref(g), ct.byref(n), ct.byref(nnz)), "mg_batch_info")
        return {"graphs": g.value, "n": n.value, "nnz": nnz.value}

    def graph_info(self, g: int) -> dict:
        n, nnz, mass = ct.c_uint32(), ct.c_uint64(), ct.c_double()
        self.ctx.check(lib().mg_batch_graph_info(self.h, g, ct.byref(n), ct.byref(nnz), ct.byref(mass)),
                       "mg_batch_graph_info")
        return {"n": n.value, "nnz": nnz.value, "mass": mass.value}

    def run(self, version: int = 2, threshold: float = 1e-6, max_phases: int = 1000, precision: str = "fp64",
            graphs: bool = True, assignments: bool = True) -> dict:
        opts = _RunOpts(version, threshold, max_phases, _PREC[precision], 0)
        r = ct.c_void_p()
        self.ctx.check(lib().mg_batch_run(self.h, ct.byref(opts), BATCH_GRAPHS if graphs else 0, ct.byref(r)),
                       "mg_batch_run")
        try:
            s = _Summary()
            lib().mg_batch_result_summary(r, ct.byref(s))
            out = {f: getattr(s, f) for f, _ in _Summary._fields_}
            G = self.info()["graphs"]
            per = {f: [] for f, _ in _BatchGraph._fields_}
            assign = []
            bg = _BatchGraph()
            for g in range(G):
                lib().mg_batch_result_graph(r, g, ct.byref(bg))
                for f, _ in _BatchGraph._fields_:
                    per[f].append(getattr(bg, f))
                if assignments:
                    a = np.zeros(max(bg.n, 1), np.uint32)
                    lib().mg_batch_result_assignment(r, g, _p(a))
                    assign.append(a[: bg.n])
            out["graphs"] = {f: np.array(v) for f, v in per.items()}
            out["assignments"] = assign
            return out
        finally:
            lib().mg_batch_result_destroy(r)


class Graph:
    """A graph resident in device memory (mg_graph)."""

    def __init__(self, ctx: Context, h: ct.c_void_p):
        self.ctx = ctx
        self.h = h
        ctx._adopt(self)

    def close(self):
        if self.h:
            lib().mg_graph_destroy(self.h)
            self.h = ct.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def info(self) -> dict:
        n, nnz, mass, integ = ct.c_uint32(), ct.c_uint64(), ct.c_double(), ct.c_int()
        self.ctx.check(lib().mg_graph_info(self.h, ct.byref(n), ct.byref(nnz), ct.byref(mass), ct.byref(integ)),
                       "mg_graph_info")
        return {"n": n.value, "nnz": nnz.value, "mass": mass.value, "integral": bool(integ.value)}

    def properties(self) -> dict:
        """Row properties found by the engine: sorted rows, symmetric (integral) entries."""
        so, sy = ct.c_int(), ct.c_int()
        self.ctx.check(lib().mg_graph_properties(self.h, ct.byref(so), ct.byref(sy)), "mg_graph_properties")
        return {"sorted_rows": bool(so.value), "symmetric": bool(sy.value)}

    @property
    def n(self) -> int:
        return self.info()["n"]

    def csr(self):
        i = self.info()
        off = np.zeros(i["n"] + 1, np.uint64)
        cols = np.zeros(max(i["nnz"], 1), np.uint32)
        w = np.zeros(max(i["nnz"], 1), np.float64)
        self.ctx.check(lib().mg_graph_copy_csr(self.h, _p(off), _p(cols), _p(w)), "mg_graph_copy_csr")
        return off, cols[: i["nnz"]], w[: i["nnz"]]

    def bins(self, scheme: int = 0) -> dict:
        n = self.info()["n"]
        sizes = np.zeros(11, np.uint32)
        boff = np.zeros(11, np.uint32)
        perm = np.zeros(max(n, 1), np.uint32)
        md = ct.c_uint32()
        self.ctx.check(lib().mg_bins(self.h, scheme, _p(sizes), _p(boff), _p(perm), ct.byref(md)), "mg_bins")
        nb = {0: 10, 1: 11, 2: 9}[scheme]
        return {"sizes": sizes[:nb], "offsets": boff[:nb], "perm": perm[:n], "max_degree": int(md.value)}

    def local_move(self, C, sigma, k, version: int = 2, up: bool = True, precision: str = "fp64"):
        n = self.info()["n"]
        C = np.ascontiguousarray(C, dtype=np.uint32)
        sigma = np.ascontiguousarray(sigma, dtype=np.float64)
        k = np.ascontiguousarray(k, dtype=np.float64)
        out = np.zeros(max(n, 1), np.uint32)
        d = ct.c_uint64()
        self.ctx.check(lib().mg_local_move(self.h, version, int(up), _PREC[precision], _p(C), _p(sigma), _p(k),
                                           _p(out), ct.byref(d)), "mg_local_move")
        return out[:n], int(d.value)

    def modularity(self, C) -> float:
        C = np.ascontiguousarray(C, dtype=np.uint32)
        q = ct.c_double()
        self.ctx.check(lib().mg_modularity(self.h, _p(C), ct.byref(q)), "mg_modularity")
        return q.value

    def coarsen(self, C):
        n = self.info()["n"]
        C = np.ascontiguousarray(C, dtype=np.uint32)
        cd = np.zeros(max(n, 1), np.uint32)
        h = ct.c_void_p()
        self.ctx.check(lib().mg_coarsen(self.h, _p(C), _p(cd), ct.byref(h)), "mg_coarsen")
        return cd[:n], Graph(self.ctx, h)

    def louvain(self, version: int = 2, threshold: float = 1e-6, max_phases: int = 1000,
                precision: str = "fp64", verbose: bool = False, keep_levels: int = 0) -> dict:
        """mg_louvain_run; with keep_levels >= 1 the result also holds
        "level_maps", the dendrogram (one community map per level,
        mg_result_level_map); with keep_levels = 2 also "level_csr", the
        (offsets, cols, weights) of the graph every level worked on."""
        opts = _RunOpts(version, threshold, max_phases, _PREC[precision], int(verbose), int(keep_levels))
        r = ct.c_void_p()
        self.ctx.check(lib().mg_louvain_run(self.h, ct.byref(opts), ct.byref(r)), "mg_louvain_run")
        try:
            s = _Summary()
            lib().mg_result_summary(r, ct.byref(s))
            n = self.info()["n"]
            a = np.zeros(max(n, 1), np.uint32)
            lib().mg_result_assignment(r, _p(a))
            cnt = ct.c_int()
            lib().mg_result_level_sizes(r, None, 0, ct.byref(cnt))
            lv = np.zeros(max(cnt.value, 1), np.uint32)
            lib().mg_result_level_sizes(r, _p(lv), cnt.value, ct.byref(cnt))
            lib().mg_result_trace(r, None, 0, ct.byref(cnt))
            tr = np.zeros((max(cnt.value, 1), 4), np.float64)
            lib().mg_result_trace(r, _p(tr), cnt.value, ct.byref(cnt))
            out = {f: getattr(s, f) for f, _ in _Summary._fields_}
            out.update({"assignment": a[:n], "level_sizes": lv[: len(lv) if cnt.value else 0],
                        "trace": tr[: cnt.value]})
            out["level_sizes"] = lv[: s.levels]
            if keep_levels:
                maps = []
                for lvl in range(s.levels):
                    size = ct.c_uint32()
                    if lib().mg_result_level_map(r, lvl, None, 0, ct.byref(size)) != MG_OK:
                        break
                    m = np.zeros(max(size.value, 1), np.uint32)
                    lib().mg_result_level_map(r, lvl, _p(m), size.value, ct.byref(size))
                    maps.append(m[: size.value])
                out["level_maps"] = maps
            if keep_levels >= 2:
                graphs = []
                for lvl in range(s.levels):
                    ln, lm = ct.c_uint32(), ct.c_uint64()
                    if lib().mg_result_level_csr(r, lvl, ct.byref(ln), ct.byref(lm), None, None, None) != MG_OK:
                        break
                    off = np.zeros(ln.value + 1, np.uint64)
                    cols = np.zeros(max(lm.value, 1), np.uint32)
                    w = np.zeros(max(lm.value, 1), np.float64)
                    lib().mg_result_level_csr(r, lvl, ct.byref(ln), ct.byref(lm), _p(off), _p(cols), _p(w))
                    graphs.append((off, cols[: lm.value], w[: lm.value]))
                out["level_csr"] = graphs
            return out
        finally:
            lib().mg_result_destroy(r)
