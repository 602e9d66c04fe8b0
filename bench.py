#!/usr/bin/env python
"""Benchmark: full Louvain on the seeded R-MAT scale-24 graph (edge factor 16,
(a,b,c,d) = (.57,.19,.19,.05), symmetrised, deduplicated, unit weights).

One step = one Louvain run to convergence (all phases, coarsening included)
on the graph resident in HBM.  value = local-move edges swept per second of
device time (sum over sweeps of the level's directed entries / run time),
summed over ranks and divided by the slowest rank's time.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl engine|reference]

--impl reference times the reference's Louvain logic on the host cores (the
CPU oracle port under OpenMP, all host threads): each step is one phase-0
sweep (local move + sigma update + modularity) over the same graph.
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


def traffic_per_sweep():
    """DRAM bytes of one phase-0 sweep from the committed ncu summary, if any."""
    path = os.path.join(ROOT, "profiles", "local_move_rmat24_traffic.json")
    try:
        with open(path) as f:
            return json.load(f).get("dram_bytes_per_sweep")
    except (OSError, ValueError):
        return None


def cpu_baseline_sample(csr, threads):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle_py as O

    O.set_threads(threads)
    t, edges = O.time_phase0(csr, 2, 1)
    return edges / t, t


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
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * tot_t / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded R-MAT generator)",
        "config": {"workload": f"rmat{args.scale}_ef16_louvain", "vertices": g.n, "directed_entries": g.nnz,
                   "parallelism": "host threads"},
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    return line


def run_engine(args, world, rank, local, pg):
    mg = importlib.import_module("mg-alphagcd_b200")
    ctx = mg.Context(local)
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
    traffic = traffic_per_sweep()

    # end to end through the public API with host buffers: upload the CSR,
    # run, read the assignment back
    off, cols, _ = g.csr()
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
        import types

        csr = types.SimpleNamespace(n=info["n"], offsets=off, cols=cols, weights=None)
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle_py as O

        threads = os.cpu_count() or 1
        cg = O.CSR(info["n"], off, cols, None)
        cv, ct_ = cpu_baseline_sample(cg, threads)
        cpu = {"value": cv, "unit": UNIT, "cores": threads, "kind": "port",
               "sample": f"one phase-0 sweep (local move + sigma update + modularity) over the same graph, "
                         f"{ct_:.1f} s on {threads} threads"}
        del csr
    if rank != 0:
        return None
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * t_max / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded R-MAT generator, graph built on the device)",
        "config": {"workload": f"rmat{args.scale}_ef16_louvain_full", "vertices": info["n"],
                   "directed_entries": info["nnz"], "abcd": [RMAT["a"], RMAT["b"], RMAT["c"], 0.05],
                   "seed": RMAT["seed"], "l2": "inputs larger than L2 (2.1 GB of column ids)",
                   "parallelism": "replicas" if world > 1 else "single GPU"},
        "modularity": last["modularity"], "communities": last["communities"],
        "levels": [int(x) for x in last["level_sizes"]], "iterations": last["iterations"],
        "first_pass_edges_per_s": last["phase0_edges_swept"] / last["phase0_seconds"],
        "convergence_s": last["seconds_total"],
        "local_move_s": last["seconds_local_move"], "coarsen_s": last["seconds_coarsen"],
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic,
                     "kernel": "local-move sweep (all bins)", "peak_kind": peak_kind,
                     "sweeps": sweeps, "algorithmic_bytes_per_sweep": sweep_b / max(sweeps, 1)},
        "cpu_baseline": cpu,
        "e2e": None if args.e2e_steps <= 0 else {"value": e2e_esum / e2e_tmax, "unit": UNIT,
                "h2d_bytes_per_step": 8 * (info["n"] + 1) + 4 * info["nnz"],
                "d2h_bytes_per_step": 4 * info["n"]},
        "clocks": clk,
        "gpu_launches": int(sum(r["kernel_launches"] for r in runs)),
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
