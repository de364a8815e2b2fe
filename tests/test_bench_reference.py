"""CPU test of bench.py's reference arm (`--impl reference`): on a small
grid it runs the CPU restatement on the host cores and prints the
contract's JSON line (impl, metric, unit, value, e2e with no host-device
bytes, cpu_baseline), with the workload named after the grid it ran."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_prints_the_contract_line():
    r = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--grid", "40", "--steps", "1",
                        "--warmup", "3"], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads(r.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference"
    assert line["metric"] == "time to 1e-6 rel. KKT (s)" and line["unit"] == "s"
    assert line["higher_is_better"] is False and line["value"] > 0
    assert line["config"]["workload"] == "grid_qp_40x40" and line["config"]["n"] == 1600
    assert line["e2e"]["value"] == line["value"]
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["d2h_bytes_per_step"] == 0
    assert line["cpu_baseline"]["cores"] >= 1 and line["cpu_baseline"]["kind"] == "port"
