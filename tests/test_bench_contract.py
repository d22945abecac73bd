"""bench.py's reference arm runs on the host alone (the CPU restatement of the
reference's Newton-Raphson), so its one-line JSON contract is checked here on
a small sample: the keys the harness reads, the arm's own cpu_baseline and
e2e objects, and the metric shared with the measured arm."""

import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.parametrize("workload", ["n1_sweep_case2000_synth", "injection_sweep_case6500_synth",
                                      "single_case118_synth"])
def test_reference_arm_json_line(workload):
    cmd = [sys.executable, "bench.py", "--impl", "reference", "--workload", workload, "--steps", "1", "--warmup", "0",
           "--cpu-budget-s", "0.5"]
    r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.strip().splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    sys.path.insert(0, ROOT)
    import bench
    assert d["impl"] == "reference"
    assert d["metric"] == bench.METRIC and d["unit"] == "solves/s" and d["higher_is_better"] is True
    assert d["value"] > 0 and d["steps"] == 1 and d["warmup"] == 0 and d["n_gpus"] == 1
    assert d["config"]["workload"] == workload
    cb = d["cpu_baseline"]
    assert cb["value"] == d["value"] and cb["kind"] == "port" and cb["cores"] >= 1 and " of " in cb["sample"]
    assert "cpu_nr" in cb["sample"]
    e = d["e2e"]
    assert e["value"] == d["value"] and e["h2d_bytes_per_step"] == 0 and e["d2h_bytes_per_step"] == 0
    # the reference arm never maps this repository's engine (no package import)
    assert d["native_so_loaded"] == []
