#!/usr/bin/env python
"""Benchmark: full Louvain on the seeded R-MAT scale-24 graph (edge factor 16,
(a,b,c,d) = (.57,.19,.19,.05), symmetrised, deduplicated, unit weights).

One step = one Louvain run to convergence (all phases, coarsening included)
on the graph resident in HBM.  value = local-move edges swept per second of
device time (sum over sweeps of the level's directed entries / run time),
summed over ranks and divided by the slowest rank's time.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl engine|reference]

On one GPU the line also carries "batched": the batched form on 4,096 seeded
SBM graphs (vertex counts log-uniform in [1k, 200k], 4-256 planted
communities, mean degree uniform in [8, 32], 70-90% intra-community edges,
unit weights) -- graphs/s of one batched run against the graphs/s of a loop
of single-graph runs over a systematic sample of the same graphs, and a check
that every sampled graph got the same modularity both ways.

Two more single-graph workloads are reported beside it: "sbm64k" (seeded SBM,
65,536 vertices in 64 planted communities, mean degree 16, 80% intra: Q and
the community count of every level) and "precision" (seeded Chung-Lu graph,
4,194,304 vertices, exponent 2.1, mean degree 20, degrees capped at 200,000,
float lognormal(0, 1) weights: FP32 gains against FP64 gains, the FP64
modularity recomputed from the FP32 run's assignment, and exact int64 gains
against FP64 gains on the unit-weight copy of the same graph).  "loader"
times the host Matrix Market loader on an R-MAT-20 file: parse, parse with
the binary CSR cache written, load from the cache, and a graph built from it.

It also carries "serving": a Poisson stream of Louvain jobs (default 200
requests/s for 60 s; half SBM, half R-MAT with edge factor 16 and the
R-MAT-24 probabilities; vertex counts log-uniform in [1k, 8M]) submitted to
the continuous-batching server (8 slots sharing a 150 GB HBM budget):
offered and served jobs/s and the submit-to-done latency percentiles of the
jobs completed within the window (jobs still queued at its end are reported
with their count and age).  Its "rate_ladder" repeats the window at lower
loads (default 6, 10 and 14 requests/s for 15 s each), where the latency
percentiles measure service rather than backlog; "sustained_load" is the
first of them and "max_rate_p99_below_1s" the highest rate of the ladder
that was served completely with p99 below one second.

--impl reference times the reference's Louvain logic on the host cores (the
CPU oracle port under OpenMP, all host threads): each step is one phase-0
sweep (local move + sigma update + modularity) over the same graph, and one
full run to convergence beside the steps gives its time to solution and Q.
The engine arm runs the same full oracle run on the graph it timed
("cpu_baseline.full_run") and reports |Q - Q_oracle|.
Multi-GPU runs are independent replicas (a single graph does not shard).
"""
from __future__ import annotations

import argparse
import importlib
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Louvain edges/s (R-MAT 24, full convergence)"
UNIT = "edges/s"
RMAT = dict(scale=24, edge_factor=16, a=0.57, b=0.19, c=0.19, seed=2)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["engine", "reference"], default="engine")
    ap.add_argument("--scale", type=int, default=RMAT["scale"])
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-full-run", dest="full_run", action="store_false",
                    help="skip the oracle's full run to convergence (Q_oracle, time to solution)")
    ap.add_argument("--no-batched", action="store_true")
    ap.add_argument("--batch-graphs", type=int, default=4096)
    ap.add_argument("--batch-steps", type=int, default=2)
    ap.add_argument("--no-serving", action="store_true")
    ap.add_argument("--no-extra", action="store_true", help="skip the sbm64k and precision lines")
    ap.add_argument("--tune", choices=["on", "cached", "off"], default="on",
                    help="autotuner of the kernel shapes per degree class (on: time new classes)")
    ap.add_argument("--serve-rate", type=float, default=200.0)
    ap.add_argument("--serve-seconds", type=float, default=60.0)
    ap.add_argument("--serve-slots", type=int, default=SERVE["slots"], help="worker slots of the server")
    ap.add_argument("--sustain-rates", default="6,10,14",
                    help="serving windows at lower loads (comma-separated req/s; empty: skip): the first is "
                         "'sustained_load', all form 'rate_ladder' with the highest rate whose p99 stays below 1 s")
    ap.add_argument("--sustain-seconds", type=float, default=15.0)
    return ap.parse_args()


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        backend = "nccl" if torch.cuda.is_available() else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
        pg = dist
    return world, rank, local, pg


def reduce_max_sum(pg, world, local, t, x):
    """max of t and sum of x over ranks (identity on one process)."""
    if pg is None or world == 1:
        return t, x
    import torch

    dev = torch.device("cuda", local) if torch.cuda.is_available() else torch.device("cpu")
    a = torch.tensor([t], dtype=torch.float64, device=dev)
    b = torch.tensor([x], dtype=torch.float64, device=dev)
    pg.all_reduce(a, op=pg.ReduceOp.MAX)
    pg.all_reduce(b, op=pg.ReduceOp.SUM)
    return float(a.item()), float(b.item())


def barrier(pg):
    if pg is not None:
        pg.barrier()


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, local_rank):
        vis = os.environ.get("CUDA_VISIBLE_DEVICES")
        idx = str(local_rank)
        if vis:
            parts = [p.strip() for p in vis.split(",") if p.strip()]
            if local_rank < len(parts):
                idx = parts[local_rank]
        self.idx = idx
        self.lines = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                          "-i", self.idx, "-lms", "200"], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except (OSError, FileNotFoundError):
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"], "samples": 0}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.t.join(timeout=2)
        sm, smax, power = [], [], []
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
                power.append(float(f[3]))
            except ValueError:
                continue
            for nm, val in zip(names, f[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(smax), "reasons": sorted(reasons),
                "samples": len(sm), "power_w_max": max(power)}


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


TRAFFIC_PROFILE = "local_move_level0_sweep_traffic"


def traffic_per_sweep():
    """DRAM bytes of one level-0 table sweep of R-MAT-24 (the second sweep)
    from the committed ncu summary (measured on smaller R-MATs and scaled by
    the entry count), the algorithmic bytes bound of that sweep, and where the
    figures come from."""
    try:
        with open(os.path.join(ROOT, "profiles", TRAFFIC_PROFILE + ".json")) as f:
            p = json.load(f)
        src = {"profile": p["key"], "measured_at_commit": p["measured_at_commit"], "sweep": p["sweep"],
               "scaling": p["scaling"],
               "captures": {k: {"dram_bytes": v["dram_bytes"], "first_sweep_dram_bytes": v["first_sweep_dram_bytes"]}
                            for k, v in p["captures"].items()}}
        return p["rmat24_dram_bytes_scaled"], p["rmat24_algorithmic_bytes_bound"], src
    except (OSError, ValueError, KeyError):
        return None, None, None


def pinned_csr(g):
    """The graph's CSR (offsets u64, cols u32) copied into page-locked host
    memory, as a caller that streams graphs to the GPU would hold it."""
    import numpy as np
    import torch

    off_d, cols_d, _ = g.csr()
    off = torch.empty(len(off_d), dtype=torch.int64).pin_memory().numpy().view(np.uint64)
    cols = torch.empty(len(cols_d), dtype=torch.int32).pin_memory().numpy().view(np.uint32)
    off[:] = off_d
    cols[:] = cols_d
    return off, cols


def cpu_baseline_sample(csr, threads):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle_py as O

    O.set_threads(threads)
    t, edges = O.time_phase0(csr, 2, 1)
    return edges / t, t


def rmat_config(scale, n, nnz):
    """The workload description both arms report (identical dicts)."""
    return {"workload": f"rmat{scale}_ef16_louvain_full", "vertices": n, "directed_entries": nnz,
            "abcd": [RMAT["a"], RMAT["b"], RMAT["c"], 0.05], "seed": RMAT["seed"],
            "l2": "inputs larger than L2 (2.1 GB of column ids)"}


def oracle_full_run(O, csr):
    """The oracle's Louvain to convergence (version 2, threshold 1e-6) on the
    host cores: time to solution, Q, levels and iterations."""
    t0 = time.perf_counter()
    r = O.louvain(csr)
    t = time.perf_counter() - t0
    return {"seconds": t, "modularity": r["modularity"], "levels": [int(x) for x in r["level_sizes"]],
            "iterations": int(r["iterations"]), "communities": int(r["communities"]),
            "threads": O.get_threads()}


def run_reference(args, world, rank, local, pg):
    if rank != 0:
        return None
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle_py as O

    threads = os.cpu_count() or 1
    O.set_threads(threads)
    g = O.gen_rmat(args.scale, RMAT["edge_factor"], RMAT["a"], RMAT["b"], RMAT["c"], RMAT["seed"])
    for _ in range(args.warmup):
        O.time_phase0(g, 2, 1)
    tot_t, tot_e = 0.0, 0
    for _ in range(args.steps):
        t, e = O.time_phase0(g, 2, 1)
        tot_t += t
        tot_e += e
    v = tot_e / tot_t
    sample = (f"one phase-0 sweep (local move + sigma update + modularity) per step over the full "
              f"R-MAT-{args.scale} graph ({g.nnz} directed entries), version 2")
    full = oracle_full_run(O, g) if args.full_run else None
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * tot_t / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded R-MAT generator)",
        "config": rmat_config(args.scale, g.n, g.nnz),
        "parallelism": f"host threads ({threads})",
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        # time to solution beside the sweep samples: one run to convergence
        "full_run": full,
    }
    if full is not None:
        line["convergence_s"] = full["seconds"]
        line["modularity"] = full["modularity"]
    return line


def _timed_runs(g, k, **kw):
    g.louvain(**kw)  # warm-up (and autotuning of new degree classes)
    runs = [g.louvain(**kw) for _ in range(k)]
    return runs, statistics.median(r["seconds_total"] for r in runs)


def run_sbm64k(ctx, with_oracle=True):
    g = ctx.generate_sbm(65536, 64, 16.0, 0.8, 1)
    info = g.info()
    runs, t = _timed_runs(g, 3)
    r = runs[-1]
    ref = None
    if with_oracle:
        O = _oracle()
        off, cols, _ = g.csr()
        ref = oracle_full_run(O, O.CSR(len(off) - 1, off, cols, None))
    g.close()
    out = {"workload": "SBM 65,536 vertices, 64 blocks, mean degree 16, 80% intra, seed 1, unit weights",
           "directed_entries": info["nnz"], "modularity": r["modularity"], "communities": r["communities"],
           "vertices_per_level": [int(x) for x in r["level_sizes"]], "phases": r["phases"],
           "iterations": r["iterations"], "run_s": t, "edges_per_s": r["edges_swept"] / r["seconds_total"]}
    if ref is not None:
        out["oracle"] = ref
        out["abs_error_vs_oracle"] = abs(r["modularity"] - ref["modularity"])
        out["levels_equal_oracle"] = out["vertices_per_level"] == ref["levels"]
    return out


def _oracle():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle_py as O

    O.set_threads(os.cpu_count() or 1)
    return O


def run_precision(ctx, with_oracle=True):
    """Chung-Lu 4M: FP32 gains (FP64 sigma and Q) and FP64 gains on the
    lognormal weights, FP64 and exact int64 gains on the unit-weight copy.
    Each result's error is stated against the FP64 oracle twice: Q
    recomputed by the oracle from the returned assignment (the reported
    number's own error) and the oracle's own FP64 run to convergence on the
    same graph (the algorithm's error)."""
    import numpy as np

    n = 4_194_304
    O = _oracle() if with_oracle else None

    def one(g, runs, t, prec, csr, ref):
        r = runs[-1]
        out = {"precision": prec, "modularity": r["modularity"], "run_s": t, "levels": len(r["level_sizes"])}
        if O is not None:
            qo = O.modularity(csr, r["assignment"])
            out["modularity_oracle_fp64_from_assignment"] = qo
            out["abs_error_vs_oracle_recomputed"] = abs(r["modularity"] - qo)
            out["abs_error_vs_oracle_run"] = abs(r["modularity"] - ref["modularity"])
        return out

    def oracle_run(g):
        if O is None:
            return None, None
        off, cols, w = g.csr()
        csr = O.CSR(len(off) - 1, off, cols, None if bool(np.all(w == 1.0)) else w)
        return csr, oracle_full_run(O, csr)

    gw = ctx.generate_chunglu(n, 2.1, 20.0, 200000.0, lognormal=True, seed=3)
    info = gw.info()
    csr_w, ref_w = oracle_run(gw)
    r64, t64 = _timed_runs(gw, 2, precision="fp64")
    r32, t32 = _timed_runs(gw, 2, precision="fp32")
    w64 = one(gw, r64, t64, "fp64", csr_w, ref_w)
    w32 = one(gw, r32, t32, "fp32", csr_w, ref_w)
    gw.close()
    del csr_w
    gu = ctx.generate_chunglu(n, 2.1, 20.0, 200000.0, lognormal=False, seed=3)
    csr_u, ref_u = oracle_run(gu)
    u64, tu64 = _timed_runs(gu, 2, precision="fp64")
    ui, tui = _timed_runs(gu, 2, precision="int64")
    x64 = one(gu, u64, tu64, "fp64", csr_u, ref_u)
    xi = one(gu, ui, tui, "int64", csr_u, ref_u)
    gu.close()
    del csr_u
    return {"workload": "Chung-Lu 4,194,304 vertices, exponent 2.1, mean degree 20, max degree 200,000, seed 3",
            "directed_entries": info["nnz"],
            "lognormal_f32_weights": {"fp64": w64, "fp32": w32, "oracle_fp64_run": ref_w,
                                      "fp32_vs_fp64_abs_error": abs(w32["modularity"] - w64["modularity"])},
            "unit_weights": {"fp64": x64, "int64": xi, "oracle_fp64_run": ref_u,
                             "int64_vs_fp64_abs_error": abs(xi["modularity"] - x64["modularity"]),
                             "same_assignment": bool((ui[-1]["assignment"] == u64[-1]["assignment"]).all())}}


def run_loader(mg, ctx, scale=20):
    """Host .mtx loader: an R-MAT-20 graph written as a symmetric pattern
    Matrix Market file, then parsed (mmap, all host threads), parsed with the
    binary CSR cache written, loaded from that cache, and uploaded from it."""
    import shutil
    import tempfile

    import numpy as np
    import pandas as pd

    g = ctx.generate_rmat(scale, RMAT["edge_factor"], RMAT["a"], RMAT["b"], RMAT["c"], RMAT["seed"])
    off, cols, _ = g.csr()
    g.close()
    n = len(off) - 1
    row = np.repeat(np.arange(n, dtype=np.int64), np.diff(off.astype(np.int64)))
    m = row > cols
    d = tempfile.mkdtemp(prefix="mgload")
    try:
        path = os.path.join(d, f"rmat{scale}.mtx")
        with open(path, "w") as f:
            f.write("%%MatrixMarket matrix coordinate pattern symmetric\n")
            f.write(f"{n} {n} {int(m.sum())}\n")
        pd.DataFrame({"r": row[m] + 1, "c": cols[m].astype(np.int64) + 1}).to_csv(
            path, mode="a", sep=" ", header=False, index=False)
        size = os.path.getsize(path)
        del row, m
        L = mg.lib()
        import ctypes as ct

        def timed(flags):
            h = ct.c_void_p()
            t0 = time.perf_counter()
            st = L.mg_csr_from_mtx(path.encode(), flags, ct.byref(h))
            t = time.perf_counter() - t0
            L.mg_csr_free(h)
            if st != 0:
                raise RuntimeError(f"mg_csr_from_mtx: status {st}")
            return t

        parse = min(timed(0) for _ in range(3))
        write = timed(mg.LOAD_CACHE_WRITE)
        cached = min(timed(mg.LOAD_CACHE_READ) for _ in range(3))
        ups, same = [], False
        for rep in range(3):  # the first call also pays device allocations and page faults
            t0 = time.perf_counter()
            h = ctx.graph_from_mtx(path, cache_read=True)
            ups.append(time.perf_counter() - t0)
            if rep == 0:
                same = bool((h.csr()[1] == cols).all())
            h.close()
        return {"workload": f"R-MAT-{scale} (edge factor 16) as a symmetric pattern .mtx, {size / 1e6:.0f} MB, "
                            f"{len(cols)} directed entries", "threads": os.cpu_count(),
                "parse_s": parse, "parse_mb_per_s": size / 1e6 / parse, "parse_entries_per_s": len(cols) / parse,
                "parse_and_cache_write_s": write, "cache_load_s": cached,
                "graph_from_cache_s": min(ups), "graph_from_cache_first_s": ups[0],
                "graph_equals_generator": same}
    finally:
        shutil.rmtree(d, ignore_errors=True)


BATCH = dict(n_range=(1000, 200000), blocks_range=(4, 256), deg_range=(8.0, 32.0), intra_range=(0.7, 0.9), seed=4)


def run_batched(mg, ctx, args):
    """Batched form vs a per-graph loop of the plain path on the same GPU."""
    params = mg.draw_sbm_params(args.batch_graphs, **BATCH)
    b = ctx.batch_generate_sbm(params)
    info = b.info()
    b.run(assignments=False)  # warm-up
    walls, devs, runs = [], [], []
    for _ in range(max(args.batch_steps, 1)):
        t0 = time.perf_counter()
        r = b.run(assignments=False)
        walls.append(time.perf_counter() - t0)
        devs.append(r["seconds_total"])
        runs.append(r)
    q = runs[-1]["graphs"]["modularity"]
    b.close()
    # per-graph loop over a systematic sample (every step-th graph)
    step = max(1, args.batch_graphs // 64)
    loop_wall, loop_dev, same, k = 0.0, 0.0, 0, 0
    for i in range(0, args.batch_graphs, step):
        p = params[i]
        g = ctx.generate_sbm(p["n"], p["blocks"], p["mean_degree"], p["intra_frac"], p["seed"])
        g.louvain()  # first run of a size may grow buffers; time the second
        t0 = time.perf_counter()
        r = g.louvain()
        loop_wall += time.perf_counter() - t0
        loop_dev += r["seconds_total"]
        same += int(r["modularity"] == q[i])
        k += 1
        g.close()
    wall = statistics.median(walls)
    return {
        "workload": f"{args.batch_graphs} SBM graphs, one batched run", "graphs": args.batch_graphs,
        "vertices": info["n"], "directed_entries": info["nnz"], "params": BATCH,
        "graphs_per_s": args.batch_graphs / wall, "run_s": wall, "device_s": statistics.median(devs),
        "sweeps": runs[-1]["sweeps"], "levels": runs[-1]["levels"],
        "gpu_launches": runs[-1]["kernel_launches"],
        "loop_graphs_per_s": k / loop_wall, "loop_sample": k, "loop_device_graphs_per_s": k / loop_dev,
        "loop_sample_wall_s": loop_wall, "loop_sample_device_s": loop_dev,
        "loop_extrapolated_wall_s": loop_wall * args.batch_graphs / k,
        "speedup_vs_loop": (args.batch_graphs / wall) / (k / loop_wall),
        "modularity_equal": f"{same}/{k}", "mean_modularity": float(q.mean()),
        "mode": "CUDA-graph iteration loop (MG_BATCH_GRAPHS)",
    }


SERVE = dict(n_range=(1000, 8_000_000), blocks_range=(4, 256), deg_range=(8.0, 32.0), intra_range=(0.7, 0.9),
             rmat_edge_factor=16, abc=(0.57, 0.19, 0.19), slots=8, budget=150 * 10**9, seed=5)


def serve_jobs(mg, count, seed):
    """Job stream of the serving workload: alternating SBM / R-MAT, vertex
    counts log-uniform (R-MAT: the nearest power of two)."""
    import numpy as np

    rng = np.random.default_rng(seed)
    lo, hi = SERVE["n_range"]
    jobs = []
    for i in range(count):
        v = float(np.exp(rng.uniform(np.log(lo), np.log(hi))))
        if i % 2 == 0:
            n = int(round(v))
            blocks = int(rng.integers(SERVE["blocks_range"][0], min(SERVE["blocks_range"][1], n) + 1))
            jobs.append(mg.gen_params("sbm", n=n, blocks=blocks, mean_degree=float(rng.uniform(*SERVE["deg_range"])),
                                      intra_frac=float(rng.uniform(*SERVE["intra_range"])), seed=1000 + i))
        else:
            scale = int(min(23, max(10, round(np.log2(v)))))
            a, b, c = SERVE["abc"]
            jobs.append(mg.gen_params("rmat", scale=scale, edge_factor=SERVE["rmat_edge_factor"], a=a, b=b, c=c,
                                      seed=1000 + i))
    return jobs


def run_serving(mg, rate, seconds, local, slots=None):
    """Poisson arrivals into the continuous-batching server for a fixed window."""
    import numpy as np

    rng = np.random.default_rng(SERVE["seed"])
    expected = int(rate * seconds * 1.2) + 16
    jobs = serve_jobs(mg, expected, SERVE["seed"])
    gaps = rng.exponential(1.0 / rate, expected)
    slots = slots or SERVE["slots"]
    srv = mg.Server(device=local, slots=slots, hbm_budget_bytes=SERVE["budget"])
    ids, t_sub = [], []
    t0 = time.perf_counter()
    t_next = 0.0
    for i in range(expected):
        t_next += gaps[i]
        if t_next >= seconds:
            break
        delay = t0 + t_next - time.perf_counter()
        if delay > 0:
            time.sleep(delay)
        ids.append(srv.submit(jobs[i]))
    window = max(time.perf_counter() - t0, seconds)
    if window > time.perf_counter() - t0:
        time.sleep(window - (time.perf_counter() - t0))
    st = srv.stats()
    infos = [srv.poll(j) for j in ids]
    done = [i for i in infos if i["state"] == mg.JOB_DONE]
    lat = np.array([i["finished_s"] - i["submitted_s"] for i in done]) if done else np.zeros(1)
    now = st["elapsed_s"]
    waiting = [now - i["submitted_s"] for i in infos if i["state"] in (mg.JOB_QUEUED, mg.JOB_RUNNING)]
    edges = sum(i["nnz"] for i in done)
    t_stop = time.perf_counter()
    srv.stop()  # cancels the queue, lets running batches finish
    return {
        "workload": f"Poisson {rate:g} req/s for {seconds:g} s, SBM + R-MAT, "
                    f"vertices log-uniform in [1k, 8M]", "params": dict(SERVE, slots=slots),
        "offered_jobs_per_s": len(ids) / window, "served_jobs_per_s": len(done) / window,
        "submitted": len(ids), "completed": len(done), "failed": st["failed"],
        "unfinished": len(waiting), "unfinished_max_age_s": max(waiting) if waiting else 0.0,
        "p50_latency_s": float(np.percentile(lat, 50)), "p99_latency_s": float(np.percentile(lat, 99)),
        "mean_latency_s": float(lat.mean()), "served_edges_per_s": edges / window,
        "batches": st["batches"], "stop_s": time.perf_counter() - t_stop,
    }


def run_engine(args, world, rank, local, pg):
    mg = importlib.import_module("mg-alphagcd_b200")
    ctx = mg.Context(local)
    ctx.tune_mode({"on": mg.TUNE_ON, "cached": mg.TUNE_CACHED, "off": mg.TUNE_OFF}[args.tune])
    g = ctx.generate_rmat(args.scale, RMAT["edge_factor"], RMAT["a"], RMAT["b"], RMAT["c"], RMAT["seed"])
    info = g.info()
    for _ in range(max(args.warmup, 0)):
        g.louvain()
    barrier(pg)
    clocks = ClockSampler(local)
    clocks.start()
    runs = [g.louvain() for _ in range(args.steps)]
    barrier(pg)
    clk = clocks.stop()
    t = sum(r["seconds_total"] for r in runs)
    e = sum(r["edges_swept"] for r in runs)
    t_max, e_sum = reduce_max_sum(pg, world, local, t, e)
    value = e_sum / t_max
    last = runs[-1]
    sweep_s = sum(r["seconds_sweep_kernels"] for r in runs)
    sweep_b = sum(r["sweep_bytes"] for r in runs)
    sweeps = sum(r["sweeps"] for r in runs)
    achieved = sweep_b / sweep_s / 1e9
    peak, peak_kind = peaks()
    traffic, traffic_alg, traffic_src = traffic_per_sweep()

    # end to end through the public API with host buffers: upload the CSR
    # from pinned host memory, run, read the assignment back
    off, cols = pinned_csr(g)
    e2e_t, e2e_e = 0.0, 0
    for i in range(args.e2e_steps + 1 if args.e2e_steps > 0 else 0):
        t0 = time.perf_counter()
        h = ctx.graph_from_csr(info["n"], off, cols, None)
        r = h.louvain()
        t1 = time.perf_counter()
        h.close()
        if i > 0:
            e2e_t += t1 - t0
            e2e_e += r["edges_swept"]
    e2e_tmax, e2e_esum = reduce_max_sum(pg, world, local, e2e_t, e2e_e)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        O = _oracle()
        threads = os.cpu_count() or 1
        cg = O.CSR(info["n"], off, cols, None)
        cv, ct_ = cpu_baseline_sample(cg, threads)
        cpu = {"value": cv, "unit": UNIT, "cores": threads, "kind": "port",
               "sample": f"one phase-0 sweep (local move + sigma update + modularity) over the same graph, "
                         f"{ct_:.1f} s on {threads} threads"}
        if args.full_run:
            # the oracle to convergence on the graph the engine ran: Q_oracle
            # and its time to solution
            cpu["full_run"] = oracle_full_run(O, cg)
        del cg
    batched = serving = sbm64k = precision = loader = None
    if world == 1 and not args.no_extra:
        g.close()
        sbm64k = run_sbm64k(ctx, with_oracle=not args.no_cpu_baseline)
        precision = run_precision(ctx, with_oracle=not args.no_cpu_baseline)
        loader = run_loader(mg, ctx)
    if world == 1 and not args.no_batched:
        g.close()
        batched = run_batched(mg, ctx, args)
    if world == 1 and not args.no_serving:
        g.close()
        ctx.close()  # the server's slots take the HBM budget
        serving = run_serving(mg, args.serve_rate, args.serve_seconds, local, args.serve_slots)
        rates = [float(x) for x in args.sustain_rates.split(",") if x.strip()]
        if rates:
            # the same job mix at loads one GPU keeps up with: latency is
            # service time plus short queueing, not backlog
            ladder = [run_serving(mg, r, args.sustain_seconds, local, args.serve_slots) for r in rates]
            serving["sustained_load"] = ladder[0]
            serving["rate_ladder"] = [{"offered_jobs_per_s": x["offered_jobs_per_s"],
                                       "served_jobs_per_s": x["served_jobs_per_s"],
                                       "p50_latency_s": x["p50_latency_s"], "p99_latency_s": x["p99_latency_s"],
                                       "unfinished": x["unfinished"]} for x in ladder]
            ok = [x["offered_jobs_per_s"] for x in ladder if x["p99_latency_s"] < 1.0 and x["unfinished"] == 0]
            serving["max_rate_p99_below_1s"] = max(ok) if ok else None
    if rank != 0:
        return None
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * t_max / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded R-MAT generator, graph built on the device)",
        "config": rmat_config(args.scale, info["n"], info["nnz"]),
        "parallelism": f"replicas ({world} GPUs)" if world > 1 else "single GPU",
        "modularity": last["modularity"], "communities": last["communities"],
        "levels": [int(x) for x in last["level_sizes"]], "iterations": last["iterations"],
        "first_pass_edges_per_s": last["phase0_edges_swept"] / last["phase0_seconds"],
        "convergence_s": last["seconds_total"],
        "local_move_s": last["seconds_local_move"], "coarsen_s": last["seconds_coarsen"],
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic,
                     "traffic_sweep": traffic_src["sweep"] if traffic_src else None,
                     "traffic_sweep_algorithmic_bytes_bound": traffic_alg,
                     "traffic_source": traffic_src,
                     "kernel": "local-move sweep (all bins)", "peak_kind": peak_kind,
                     "sweeps": sweeps, "algorithmic_bytes_per_sweep": sweep_b / max(sweeps, 1)},
        "cpu_baseline": cpu,
        "modularity_vs_oracle": None if not (cpu and cpu.get("full_run")) else {
            "q_oracle": cpu["full_run"]["modularity"],
            "abs_error": abs(last["modularity"] - cpu["full_run"]["modularity"]),
            "levels_equal": [int(x) for x in last["level_sizes"]] == cpu["full_run"]["levels"],
            "iterations_equal": last["iterations"] == cpu["full_run"]["iterations"],
            "oracle_convergence_s": cpu["full_run"]["seconds"],
            "engine_convergence_s": last["seconds_total"]},
        "e2e": None if args.e2e_steps <= 0 else {"value": e2e_esum / e2e_tmax, "unit": UNIT,
                "h2d_bytes_per_step": 8 * (info["n"] + 1) + 4 * info["nnz"],
                "d2h_bytes_per_step": 4 * info["n"]},
        "clocks": clk,
        "gpu_launches": int(sum(r["kernel_launches"] for r in runs)),
        "sbm64k": sbm64k,
        "precision": precision,
        "loader": loader,
        "batched": batched,
        "serving": serving,
    }
    return line


def main():
    args = parse()
    if args.impl == "reference":
        # host-only arm: rank 0 runs, the other ranks exit without work
        rank = int(os.environ.get("RANK", "0"))
        line = run_reference(args, int(os.environ.get("WORLD_SIZE", "1")), rank, 0, None)
        if line is not None:
            print(json.dumps(line), flush=True)
        return
    world, rank, local, pg = dist_setup(args)
    try:
        if args.impl == "reference":
            line = run_reference(args, world, rank, local, pg)
        else:
            line = run_engine(args, world, rank, local, pg)
        if line is not None and rank == 0:
            print(json.dumps(line), flush=True)
    finally:
        if pg is not None:
            pg.destroy_process_group()


if __name__ == "__main__":
    main()
