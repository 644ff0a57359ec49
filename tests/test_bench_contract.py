"""bench.py on the host: the reference arm's JSON line and the CPU timings of the reference's
own methods that the B200 line reports beside its rates (no GPU)."""

from __future__ import annotations

import json
import subprocess
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT))


def test_reference_arm_prints_the_contract_line():
    out = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference",
                          "--steps", "2", "--warmup", "1"], cwd=ROOT, capture_output=True,
                         text=True, timeout=300, check=True).stdout
    line = json.loads(out.strip().splitlines()[-1])
    assert line["impl"] == "reference"
    for key in ("metric", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "scaling",
                "vs_baseline", "dtype", "data", "config"):
        assert key in line, key
    assert line["value"] > 0 and line["higher_is_better"] is True
    assert line["steps"] == 2 and line["warmup"] == 1
    cpu = line["cpu_baseline"]
    assert cpu["kind"] == "port" and cpu["cores"] >= 1 and cpu["value"] == line["value"]
    assert line["e2e"] == {"value": line["value"], "unit": line["unit"],
                           "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}


def small_case():
    from pyeulerale_b200 import grid

    X = grid.naca_ogrid(33, 33, 0.12, 1.0, 20.0, 0.01)
    rng = np.random.default_rng(3)
    U = grid.perturbed_states(32, 32, 0.5, 1.25, 0.01, rng)
    return X, np.zeros_like(X), U


def test_cpu_reference_methods_run_on_a_small_grid():
    import bench

    X, V, U = small_case()
    lin = bench.cpu_linear_rates(X, V, U, 0.5)
    for key in ("jacobian_states", "vjp", "jvp", "bsr_conversion", "bsr_spmv"):
        assert lin[key]["value"] > 0, key
    assert lin["cores"] == 1 and lin["kind"] == "port"
    so = bench.cpu_second_order_rate(X, V, U, 0.5)
    assert so["value"] > 0
    res = bench.cpu_resolvent_rate(X, V, U, 0.5, 0.05j)
    assert res["value"] > 0 and "relative residual" in res["sample"]
    rel = float(res["sample"].split("relative residual ")[1].split(")")[0])
    assert rel < 1e-8


def test_gpus_flag_starts_that_many_ranks():
    """``bench.py --gpus 2`` outside torchrun starts two ranks (here in the gloo dry run, which
    runs the launcher, the rank check, the barrier and the max over ranks without a GPU) and
    prints one JSON line whose n_gpus is 2."""
    import os

    env = {k: v for k, v in os.environ.items()
           if k not in ("WORLD_SIZE", "RANK", "LOCAL_RANK", "MASTER_ADDR", "MASTER_PORT")}
    out = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--gpus", "2", "--dry-run",
                          "--steps", "3", "--warmup", "3"], cwd=ROOT, capture_output=True,
                         text=True, timeout=300, check=True, env=env).stdout
    lines = [json.loads(s) for s in out.strip().splitlines() if s.startswith("{")]
    assert len(lines) == 1, out
    assert lines[0]["n_gpus"] == 2 and lines[0]["dry_run"] is True
    assert lines[0]["config"]["parallelism"] == "replicas x2"


def test_rank_count_mismatch_fails_loudly():
    """A rank whose WORLD_SIZE disagrees with --gpus stops before any timing."""
    import os

    env = dict(os.environ, WORLD_SIZE="1", RANK="0", LOCAL_RANK="0")
    proc = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--gpus", "2", "--dry-run"],
                          cwd=ROOT, capture_output=True, text=True, timeout=120, env=env)
    assert proc.returncode != 0
    assert "2 but 1 ranks" in proc.stderr
