"""bench.py's reference arm on the host cores (no GPU): one JSON line with the
keys the benchmark contract asks for, the same workload config as the engine
arm, and a torchrun-style run where only rank 0 prints."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _run(args, env=None):
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py")] + args, capture_output=True, text=True,
                         timeout=600, env=env, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    return [l for l in out.stdout.splitlines() if l.startswith("{")]


def test_reference_arm_line():
    lines = _run(["--impl", "reference", "--scale", "14", "--steps", "2", "--warmup", "1"])
    assert len(lines) == 1
    d = json.loads(lines[0])
    for k in ("impl", "metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
              "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["impl"] == "reference" and d["steps"] == 2 and d["warmup"] == 1
    assert d["value"] > 0 and d["higher_is_better"] is True
    assert d["e2e"]["value"] == d["value"] and d["e2e"]["h2d_bytes_per_step"] == 0
    assert d["cpu_baseline"]["kind"] == "port" and d["cpu_baseline"]["cores"] >= 1
    # time to solution: one oracle run to convergence beside the sweep samples
    full = d["full_run"]
    assert full["seconds"] > 0 and full["iterations"] > 0 and full["levels"][0] == d["config"]["vertices"]
    assert d["modularity"] == full["modularity"] and d["convergence_s"] == full["seconds"]
    sys.path.insert(0, ROOT)
    import bench

    # the engine arm reports the identical workload description
    assert d["config"] == bench.rmat_config(14, d["config"]["vertices"], d["config"]["directed_entries"])


def test_reference_arm_other_ranks_print_nothing():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2")
    assert _run(["--impl", "reference", "--scale", "12", "--steps", "1", "--warmup", "0"], env=env) == []
