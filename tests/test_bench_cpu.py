"""bench.py's reference arm on the CPU: the reference's own KT step (its CPU build under
oracle/_ref) timed on the host cores and printed as the benchmark's one JSON line; under
torchrun only rank 0 does the work and prints."""
import json
import os
import subprocess
import sys

import pytest

import oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

pytestmark = pytest.mark.skipif(not oracle.ref_available("fp64_qcd_bulk"),
                                reason="the reference's CPU build (oracle/_ref) is not built")


def run_bench(args, env=None):
    e = dict(os.environ)
    e.update(env or {})
    return subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), *args], capture_output=True, text=True,
                          env=e, timeout=600)


def test_reference_arm_prints_the_json_line():
    r = run_bench(["--impl", "reference", "--steps", "1", "--warmup", "0"])
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, r.stdout
    b = json.loads(lines[0])
    for key in ["metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
                "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"]:
        assert key in b, key
    assert b["impl"] == "reference"
    assert b["metric"] == b["unit"] == "cell-updates/s"
    assert b["value"] > 0 and b["higher_is_better"] is True
    assert b["n_gpus"] == 1 and b["steps"] == 1 and b["warmup"] == 0
    assert b["config"]["workload"].startswith("config2_131x131x61")
    cb = b["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["value"] == b["value"] and cb["cores"] >= 1 and cb["sample"]
    assert b["e2e"] == {"value": b["value"], "unit": b["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}


def test_reference_arm_other_ranks_exit_without_work():
    r = run_bench(["--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "0"],
                  env={"RANK": "1", "WORLD_SIZE": "2", "LOCAL_RANK": "1"})
    assert r.returncode == 0, r.stderr[-2000:]
    assert not r.stdout.strip()
