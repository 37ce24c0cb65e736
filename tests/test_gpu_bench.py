"""Every arm of bench.py, end to end, on a small workload.

Each run prints one JSON line; the test checks the keys the benchmark's
contract requires of it (metric, value, unit, timing, the roofline and CPU
baseline objects of the own arm, the reference arm's marker).  The sizes are
small, so the numbers themselves are not checked.
"""
import json
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SMALL = ["--steps", "1", "--warmup", "3", "--e2e-steps", "1"]


def _bench(*args, timeout=900):
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), *args],
                       cwd=ROOT, capture_output=True, text=True, timeout=timeout)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-4000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, r.stdout[-2000:]
    return json.loads(lines[0])


def _check_own(d, workload_key="workload"):
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step",
              "higher_is_better", "scaling", "dtype", "data", "config", "roofline",
              "gpu_launches", "clocks"):
        assert k in d, k
    assert d["value"] > 0 and d["ms_per_step"] > 0
    assert workload_key in d["config"]
    r = d["roofline"]
    assert r["bound"] in ("hbm", "tensor") and r["peak"] > 0 and r["achieved"] > 0
    assert d["gpu_launches"] > 0


@pytest.mark.parametrize("workload,extra", [
    ("ncu_small", []),
    ("prune_ncu_l2000", []),
    ("batch_small", []),
    ("precision_small", ["--cerr-pairs", "2", "--ref-pairs", "1"]),
    ("shard_small", []),
])
def test_bench_own_arm(workload, extra):
    d = _bench("--workload", workload, *SMALL, "--no-cpu-baseline", *extra)
    _check_own(d)
    if workload == "ncu_small":
        # the drop-in call on a host cost matrix, timed beside the plan path
        dr = d["dropin_host_C"]
        assert dr["value"] > 0 and dr["h2d_bytes_per_call"] > 0


def test_bench_own_arm_cpu_baseline():
    # the CPU baseline leg (the oracle, bounded sample) on the single-pair arm
    d = _bench("--workload", "ncu_small", *SMALL)
    _check_own(d)
    cb = d["cpu_baseline"]
    assert cb["value"] > 0 and cb["cores"] >= 1 and cb["kind"] in ("port", "reference")


@pytest.mark.parametrize("workload", ["ncu_small", "prune_ncu_l2000", "batch_small",
                                      "precision_small", "shard_small"])
def test_bench_reference_arm(workload):
    d = _bench("--impl", "reference", "--workload", workload, *SMALL)
    assert d["impl"] == "reference"
    if "unavailable" in d:
        return
    assert d["value"] > 0
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["d2h_bytes_per_step"] == 0
    assert d["cpu_baseline"]["cores"] >= 1
