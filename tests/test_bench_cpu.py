"""bench.py's reference arm (the reference's own CPU code for the path, no
GPU needed): one JSON line with the contract's keys, the reference-arm
additions (impl, cpu_baseline describing the run, e2e with no host-device
bytes) and, for a workload the reference has no CPU code for, the one-line
`unavailable` form."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
KEYS = {"metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
        "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e", "impl"}


def _bench(*args):
    out = subprocess.run([sys.executable, "bench.py", "--impl", "reference", *args], cwd=ROOT, capture_output=True,
                         text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [ln for ln in out.stdout.strip().splitlines() if ln.startswith("{")]
    assert len(lines) == 1, out.stdout[-2000:]
    return json.loads(lines[0])


@pytest.mark.parametrize("workload", ["q11", "q21", "q41"])
def test_reference_arm_line(workload):
    d = _bench("--workload", workload, "--steps", "2", "--warmup", "1")
    assert KEYS <= set(d), KEYS - set(d)
    assert d["impl"] == "reference" and d["n_gpus"] == 1 and d["steps"] == 2 and d["warmup"] == 1
    assert d["metric"] == "fused decode+query rows/s" and d["unit"] == "rows/s" and d["higher_is_better"] is True
    assert d["value"] > 0 and d["ms_per_step"] > 0
    cb = d["cpu_baseline"]
    assert cb["kind"] in ("reference", "port") and cb["cores"] >= 1 and cb["value"] == d["value"] and cb["sample"]
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    assert d["config"]["workload"]


def test_reference_arm_unavailable_for_the_ssb_suite():
    d = _bench("--workload", "ssb", "--steps", "1", "--warmup", "1")
    assert d["impl"] == "reference" and set(d) == {"impl", "unavailable"} and d["unavailable"]
