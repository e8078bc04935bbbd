"""bench.py --impl reference on the CPU: the JSON line of the reference arm.

The reference arm times the oracle (the CPU restatement of the reference
path) over the same window as the GPU arm.  Its line must carry the same
metric, unit and config dict as the GPU arm's, `impl: reference`, a
`cpu_baseline` describing the run and an `e2e` with zero copy bytes; under
torchrun only rank 0 runs and prints.  A 0.1 sim-time window keeps each run
to seconds.
"""
import json
import os
import subprocess
import sys

import pytest

from conftest import REPO

ARGS = ["--impl", "reference", "--steps", "1", "--warmup", "0", "--dt", "0.1"]


def _lines(out):
    return [json.loads(l) for l in out.splitlines() if l.startswith("{")]


def _bench():
    sys.path.insert(0, REPO)
    import bench
    return bench


def test_reference_arm_line_matches_the_gpu_arm_contract():
    r = subprocess.run([sys.executable, os.path.join(REPO, "bench.py")] + ARGS, cwd=REPO, capture_output=True,
                       text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = _lines(r.stdout)
    assert len(lines) == 1
    d = lines[0]
    bench = _bench()

    class A:
        dt, steps, warmup = 0.1, 1, 0

    assert d["impl"] == "reference"
    assert d["metric"] == bench.METRIC and d["unit"] == bench.UNIT and d["higher_is_better"] is True
    assert d["config"] == bench.bench_config(A, 1)
    assert d["value"] > 0.0 and d["steps"] == 1 and d["warmup"] == 0 and d["n_gpus"] == 1
    assert d["e2e"] == {"value": d["value"], "unit": bench.UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    cb = d["cpu_baseline"]
    assert cb["kind"] == "port" and cb["value"] == d["value"] and cb["cores"] >= 1
    assert d["solver_counters"]["nst"] > 0


def test_reference_arm_under_torchrun_prints_on_rank_0_only():
    env = dict(os.environ, MASTER_ADDR="127.0.0.1", OMP_NUM_THREADS="4")
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node=2",
           "--master-addr", "127.0.0.1", "--master-port", "29631", os.path.join(REPO, "bench.py"),
           "--gpus", "2"] + ARGS
    r = subprocess.run(cmd, cwd=REPO, capture_output=True, text=True, timeout=900, env=env)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = _lines(r.stdout)
    assert len(lines) == 1
    assert lines[0]["impl"] == "reference" and lines[0]["n_gpus"] == 2
