"""The bench's reference arm (CPU only, `bench.py --impl reference`): it
times the reference's own FMM::update on the host cores and prints exactly
one JSON line with the keys the driver reads, for every workload."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
KEYS = ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
        "vs_baseline", "dtype", "data", "config", "impl", "cpu_baseline", "e2e")


@pytest.mark.parametrize("workload", ["plummer", "mixture", "disk2d"])
def test_reference_arm_prints_one_contract_line(workload):
    if not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "libref.so")):
        pytest.skip("the reference is not built here (oracle/_ref)")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "0", "--workload", workload], capture_output=True, text=True, timeout=600,
                       cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.strip()]
    assert len(lines) == 1, r.stdout[-2000:]
    line = json.loads(lines[0])
    for k in KEYS:
        assert k in line, k
    assert line["impl"] == "reference" and line["value"] > 0 and line["higher_is_better"] is True
    assert line["e2e"] == {"value": line["value"], "unit": line["unit"], "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}
    cb = line["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["cores"] >= 1 and cb["value"] == line["value"]
    assert ("mixture" in line["config"]["workload"]) == (workload == "mixture")
    assert ("mixture" in cb["sample"]) == (workload == "mixture")
    assert ("2D" in line["config"]["workload"]) == (workload == "disk2d")
    # the reference's own force error on its sample is stated beside its speed
    assert cb["reference_force_rel_l2"] > 0
