"""The MCP server's tools on the GPU, against the library called directly: a loaded setup runs to
the same state (diagnostics equal to the float64 bit), slices and probes read the cells that hold
the points, a snapshot written by save_athdf restarts a run at its time, and the adaptive mesh's
stats count its leaves."""
import json
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

from shaderous_b200 import cli
from shaderous_b200.mcp import Server

pytestmark = pytest.mark.gpu


def call(srv, name, **args):
    r = srv.handle({"jsonrpc": "2.0", "id": 1, "method": "tools/call", "params": {"name": name, "arguments": args}})
    res = r["result"]
    assert not res.get("isError"), res["content"][0]["text"]
    return json.loads(res["content"][0]["text"])


def test_uniform_run_diagnostics_slice_probe_and_snapshot(tmp_path):
    setup = "problem=kelvin-helmholtz&dim=2&n=128&limiter=mc&cfl=0.4"
    srv = Server()
    call(srv, "load", setup=setup)
    r = call(srv, "run", steps=25)
    assert r["taken"] == 25 and r["stopped"] == "steps"
    d = call(srv, "diagnostics")
    # the same setup through the library directly
    class NS:
        problem = dim = n = amr = None
        set = None

    cls, cfg, prob, _ = cli.build(cli.parse_setup(setup, NS()))
    with cls(cfg) as s:
        s.reset(prob)
        s.run(steps=25)
        want = s.diagnostics()
        u1, u2 = s.read_state()
    assert d["steps"] == 25
    assert d["mass"] == pytest.approx(want.mass, rel=1e-6) and d["eTot"] == pytest.approx(want.e_tot, rel=1e-6)
    # a slice of density at full resolution is the state's density, cell for cell (its values are
    # given to 5 significant digits, as the reference's mcp.mjs gives them)
    sl = call(srv, "slice", variable="rho", axis=2, pos=0.5, res=128, include_values=True)
    rho = np.asarray(sl["values"])
    np.testing.assert_allclose(rho, u1[:, 0].reshape(128, 128), rtol=1e-4)
    assert sl["min"] == pytest.approx(float(u1[:, 0].min()), rel=1e-6)
    # probes at cell centres
    pts = [[(5 + 0.5) / 128, (70 + 0.5) / 128, 0.5], [(100 + 0.5) / 128, (3 + 0.5) / 128, 0.5]]
    pr = call(srv, "probe", points=pts)["points"]
    for p, (i, j) in zip(pr, [(5, 70), (100, 3)]):
        o = j * 128 + i
        assert p["rho"] == pytest.approx(float(u1[o, 0]), rel=1e-6)
        assert p["v"][0] == pytest.approx(float(u1[o, 1] / u1[o, 0]), rel=1e-5, abs=1e-7)
    # a snapshot, then more steps, then a restart from the snapshot lands back at its time
    f = tmp_path / "kh.athdf"
    saved = call(srv, "save_athdf", path=str(f))
    assert f.exists() and saved["bytes"] > 0
    call(srv, "run", steps=5)
    back = call(srv, "load_athdf", path=str(f))
    assert back["steps"] == 25 and back["t"] == pytest.approx(d["t"], rel=1e-6)
    d2 = call(srv, "diagnostics")
    assert d2["mass"] == pytest.approx(d["mass"], rel=1e-6)
    st = call(srv, "stats")
    assert st["cells"] == 128 * 128
    srv.session._close()


def test_adaptive_run_over_stdio():
    msgs = [
        {"jsonrpc": "2.0", "id": 1, "method": "initialize", "params": {}},
        {"jsonrpc": "2.0", "id": 2, "method": "tools/call",
         "params": {"name": "load", "arguments": {"setup": "problem=blast&dim=3&n=32&amr=3&cap=2000"}}},
        {"jsonrpc": "2.0", "id": 3, "method": "tools/call", "params": {"name": "run", "arguments": {"until": 0.002}}},
        {"jsonrpc": "2.0", "id": 4, "method": "tools/call", "params": {"name": "stats", "arguments": {}}},
        {"jsonrpc": "2.0", "id": 5, "method": "tools/call",
         "params": {"name": "slice", "arguments": {"variable": "pressure", "axis": 2, "pos": 0.5, "res": 16}}},
    ]
    p = subprocess.run([sys.executable, "-m", "shaderous_b200.mcp"], input="\n".join(json.dumps(m) for m in msgs) + "\n",
                       capture_output=True, text=True, cwd=Path(__file__).resolve().parent.parent, timeout=600)
    by = {r["id"]: r for r in map(json.loads, p.stdout.splitlines())}
    for k in (2, 3, 4, 5):
        assert not by[k]["result"].get("isError"), by[k]["result"]["content"][0]["text"]
    run = json.loads(by[3]["result"]["content"][0]["text"])
    assert run["stopped"] == "time" and run["t"] == pytest.approx(0.002, rel=1e-9)
    st = json.loads(by[4]["result"]["content"][0]["text"])
    assert st["leaves"] > 8 and len(st["leavesPerLevel"]) == 3
    sl = json.loads(by[5]["result"]["content"][0]["text"])
    assert sl["max"] > sl["min"] > 0 and len(sl["values"]) == 16
