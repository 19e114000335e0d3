"""bench.py's reference arm on the CPU: the JSON line the contract asks for, and no product library
in the process (the arm times the float64 oracle alone)."""
import json
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]

CHILD = r"""
import runpy, sys
sys.argv = ["bench.py", "--impl", "reference", "--steps", "1", "--warmup", "1"]
runpy.run_path("bench.py", run_name="__main__")
with open("/proc/self/maps") as f:
    print("LOADED_PRODUCT", any("libshaderous_b200" in line for line in f))
"""


def test_reference_arm_line_and_process():
    out = subprocess.run([sys.executable, "-c", CHILD], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = out.stdout.strip().splitlines()
    assert lines[-1] == "LOADED_PRODUCT False"
    rec = json.loads(next(ln for ln in lines if ln.startswith("{")))
    assert rec["impl"] == "reference" and rec["steps"] == 1 and rec["warmup"] == 1
    assert rec["metric"].startswith("zone-updates/s") and rec["unit"] == "zone-updates/s"
    assert rec["value"] > 0 and rec["higher_is_better"] is True
    assert rec["cpu_baseline"]["value"] == rec["value"] and rec["cpu_baseline"]["cores"] >= 1
    assert rec["e2e"] == {"value": rec["value"], "unit": rec["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
