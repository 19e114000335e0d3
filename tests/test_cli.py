"""The command-line runner (python -m shaderous_b200): setup parsing on CPU, and runs on the GPU
that write diag.jsonl and manifest.json at the output times."""
import argparse
import json
import math
import subprocess
import sys
from pathlib import Path

import pytest

from shaderous_b200.cli import PRESETS, build, parse_setup

ROOT = Path(__file__).resolve().parent.parent


def ns(**kw):
    base = dict(problem=None, dim=None, n=None, amr=None, set=None)
    base.update(kw)
    return argparse.Namespace(**base)


def test_setup_from_query_flags_and_set():
    s = parse_setup("https://x/?problem=sedov&dim=2&n=256", ns(set=["gamma=1.4", "limiter=mc"]))
    assert s == {"problem": "sedov", "dim": 2, "n": 256, "gamma": 1.4, "limiter": "mc"}
    s = parse_setup(None, ns(problem="kh", n=64))
    assert s["problem"] == "kelvin-helmholtz" and s["dim"] == 2 and s["n"] == 64
    with pytest.raises(SystemExit):
        parse_setup("problem=nope", ns())
    with pytest.raises(SystemExit):
        parse_setup(None, ns(set=["novalue"]))


def test_build_configs():
    cls, cfg, prob, t_end = build({"problem": "taylor-green", "dim": 3, "n": 64})
    assert cls.__name__ == "Sim" and cfg.n == (64, 64, 64) and cfg.dx == pytest.approx(2 * math.pi / 64)
    assert cfg.recon == "ppm" and prob.kind == "tgv" and t_end == 1.0
    cls, cfg, prob, _ = build({"problem": "sedov", "dim": 3, "n": 32, "amr": 3})
    assert cls.__name__ == "AmrSim" and cfg.nr == 2 and cfg.max_level == 2 and cfg.hydro.bc_lo == (1, 1, 1)
    assert cfg.time_bins == 0
    # the reference's link parameter for per-block timesteps (tests/unit/levels.test.ts:37)
    s = parse_setup("problem=sedov&dim=2&n=2048&amr=7&tbins=5", ns())
    _, cfg, _, _ = build(s)
    assert cfg.time_bins == 5 and cfg.max_level == 6 and cfg.nr == 128
    cls, cfg, _, _ = build({"problem": "sod", "dim": 1, "n": 512})
    assert cfg.n == (512, 1, 1) and cfg.bc_lo == (1, 0, 0) and cfg.recon == "minmod"
    assert set(PRESETS) >= {"sod", "kelvin-helmholtz", "sedov", "taylor-green", "blast"}


def test_describe_lists_the_problems():
    r = subprocess.run([sys.executable, "-m", "shaderous_b200", "describe"], capture_output=True, text=True, cwd=ROOT,
                       check=True)
    assert "sedov" in json.loads(r.stdout)


@pytest.mark.gpu
def test_run_writes_outputs(tmp_path):
    out = tmp_path / "sod"
    r = subprocess.run([sys.executable, "-m", "shaderous_b200", "run", "problem=sod&dim=1&n=512", "--until", "0.2",
                        "--every", "0.05", "--out", str(out), "--state", "--quiet"],
                       capture_output=True, text=True, cwd=ROOT, timeout=600)
    assert r.returncode == 0, r.stderr
    lines = [json.loads(x) for x in (out / "diag.jsonl").read_text().splitlines()]
    assert [round(x["t"], 9) for x in lines] == [0.0, 0.05, 0.1, 0.15, 0.2]
    assert all(abs(x["mass"] - lines[0]["mass"]) < 1e-6 * lines[0]["mass"] for x in lines[:2])
    man = json.loads((out / "manifest.json").read_text())
    assert man["stopped"] == "time" and len(man["outputs"]) == 5
    assert (out / man["outputs"][-1]["state"]).exists()
    # an adaptive run
    out2 = tmp_path / "sedov"
    r = subprocess.run([sys.executable, "-m", "shaderous_b200", "run", "problem=sedov&dim=2&n=32&amr=3", "--steps", "20",
                        "--out", str(out2), "--quiet"], capture_output=True, text=True, cwd=ROOT, timeout=600)
    assert r.returncode == 0, r.stderr
    lines = [json.loads(x) for x in (out2 / "diag.jsonl").read_text().splitlines()]
    assert lines[-1]["steps"] == 20


@pytest.mark.gpu
def test_run_writes_snapshots_and_restarts_from_one(tmp_path):
    """--athdf writes an Athena++ snapshot at each output; --from starts a run from one, which then
    goes on from the file's time and steps (the reference's headless checkpoints and --from)."""
    out = tmp_path / "blast"
    r = subprocess.run([sys.executable, "-m", "shaderous_b200", "run", "problem=blast&dim=2&n=32&amr=2", "--steps", "12",
                        "--out", str(out), "--athdf", "--gzip", "1", "--quiet"],
                       capture_output=True, text=True, cwd=ROOT, timeout=600)
    assert r.returncode == 0, r.stderr
    man = json.loads((out / "manifest.json").read_text())
    last = out / man["outputs"][-1]["athdf"]
    from shaderous_b200.athdf import read_athdf

    snap = read_athdf(last)
    assert snap.steps == 12 and snap.meta["program"] == "shaderous" and "problem=blast" in snap.meta["query"]
    out2 = tmp_path / "again"
    r = subprocess.run([sys.executable, "-m", "shaderous_b200", "run", "problem=blast&dim=2&n=32&amr=2", "--steps", "4",
                        "--from", str(last), "--out", str(out2), "--quiet"], capture_output=True, text=True, cwd=ROOT,
                       timeout=600)
    assert r.returncode == 0, r.stderr
    lines = [json.loads(x) for x in (out2 / "diag.jsonl").read_text().splitlines()]
    assert lines[0]["steps"] == 12 and lines[-1]["steps"] == 16
    assert abs(lines[0]["t"] - snap.time) < 1e-12
