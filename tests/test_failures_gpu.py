"""The failure surface of the boundary, made on the host (no GPU is faulted):

- a state with a NaN in it: run() stops with SHZ_E_NAN, "the clock is NaN" (src/sim.ts:3708; the
  reference's run() throws on a NaN clock, src/ui/api.ts settle), uniform grid and blocks;
- RunOptions.timeoutMs (src/ui/api.ts:188-196): run() gives up after that much wall time and
  returns where the run got to, stopped = "timeout";
- cancel on the server: a queued request and a running one are taken off, their results report
  SHZ_E_CANCELLED, and every other request's result is the same, bit for bit, as without them.
"""
import numpy as np
import pytest

from shaderous_b200 import Config, Problem, ShaderousError, Sim, _abi
from shaderous_b200.amr import AmrConfig, AmrSim
from shaderous_b200.serve import Request, Server, ServerConfig

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("bits", [0x7FC00000, 0xFFC00000])
def test_nan_state_stops_the_run_with_nan(bits):
    cfg = Config(n=(64, 64, 32), gamma=1.4, recon="mc", cfl=0.4)
    with Sim(cfg) as s:
        s.reset(Problem("blast", a=(1, 10, 1, 0.1, 0.2)))
        u1, u2 = s.read_state()
        u1 = u1.copy()
        u1[12345, 1] = np.array([bits], dtype=np.uint32).view(np.float32)[0]  # a momentum
        s.set_state(u1, u2)
        with pytest.raises(ShaderousError) as e:
            s.run(steps=20)
        assert e.value.code == _abi.SHZ_E_NAN
        assert "NaN" in str(e.value)


def test_nan_state_on_blocks_stops_the_run_with_nan():
    hyd = Config(gamma=5 / 3, bc_lo=(1, 1, 1), bc_hi=(1, 1, 1), recon="mc", cfl=0.4)
    cfg = AmrConfig(hydro=hyd, ndim=3, nr=2, max_level=1, cap=200, regrid_every=0)
    with AmrSim(cfg) as a:
        a.reset(Problem("blast", a=(1, 10, 1, 0.1, 0.2)))
        u1, u2 = a.leaves_state()
        u1 = u1.copy()
        u1[0, 77, 2] = np.nan
        a.set_leaves_state(u1, u2)
        with pytest.raises(ShaderousError) as e:
            a.run(steps=10)
        assert e.value.code == _abi.SHZ_E_NAN


def test_timeout_returns_where_the_run_got_to():
    cfg = Config(n=(256, 256, 256), gamma=5 / 3, recon="mc", cfl=0.4)
    with Sim(cfg) as s:
        s.reset(Problem("blast", a=(1, 10, 1, 0.1, 0.2)))
        s.run(steps=3)  # tuned and warm
        r = s.run(steps=100000, timeout_ms=300)
        assert r.stopped == "timeout"
        assert 0 < r.taken < 100000
        # batches are paced to about 50 ms of GPU time, so the run ends soon after the limit
        assert 0.3 <= r.seconds < 1.0, r.seconds
        t, _, steps = s.clock()
        assert steps == 3 + r.taken and t == r.t


def test_timeout_on_blocks():
    hyd = Config(gamma=5 / 3, bc_lo=(1, 1, 1), bc_hi=(1, 1, 1), recon="mc", cfl=0.4)
    cfg = AmrConfig(hydro=hyd, ndim=3, nr=4, max_level=2, cap=4000, regrid_every=8)
    with AmrSim(cfg) as a:
        a.reset(Problem("blast", a=(1, 10, 1, 0.1, 0.2)))
        a.run(steps=2)
        r = a.run(steps=100000, timeout_ms=300)
        assert r.stopped == "timeout" and 0 < r.taken < 100000
        assert 0.3 <= r.seconds < 2.0, r.seconds


def _reqs():
    return [
        Request(ndim=2, n=64, steps=60, problem=Problem("kh", a=(2, 1, 0.5, 2.5, 0.01, 1e-3), seed=3), gamma=1.4, bc=0),
        Request(ndim=3, n=48, steps=40, problem=Problem("blast", a=(3, 50, 1, 1, 0.15)), gamma=5 / 3, bc=1),
        Request(ndim=2, n=96, steps=50, problem=Problem("sod", a=(4, 0, 20, 1, 0, 1)), gamma=5 / 3, bc=1),
        Request(ndim=3, n=32, steps=70, problem=Problem("sod", a=(2, 0, 5, 1, 0, 1)), gamma=1.4, bc=2),
    ]


def _cfg(max_grids):
    return ServerConfig(hydro=Config(recon="mc", cfl=0.4), budget_bytes=2e9, max_grids=max_grids, round_steps=4,
                        keep_states=True)


def test_cancel_running_and_queued_requests():
    reqs = _reqs()
    with Server(_cfg(1)) as s:  # one request at a time per engine (2D, 3D): two run, two wait
        ids = [s.submit(r) for r in reqs]
        s.drain(max_rounds=2)  # 0 (2D) and 1 (3D) are running, 2 and 3 queued
        assert [s.poll(i)[0] for i in ids] == ["running", "running", "queued", "queued"]
        assert 0 < s.poll(ids[0])[1] < reqs[0].steps
        s.cancel(ids[1])  # running
        s.cancel(ids[3])  # queued
        assert s.poll(ids[1])[0] == "cancelled" and s.poll(ids[3])[0] == "cancelled"
        with pytest.raises(ShaderousError) as e:
            s.cancel(ids[1])
        assert e.value.code == _abi.SHZ_E_CONFIG
        with pytest.raises(ShaderousError) as e:
            s.cancel(12345)
        assert e.value.code == _abi.SHZ_E_CONFIG
        s.drain()
        for k in (1, 3):
            with pytest.raises(ShaderousError) as e:
                s.result(ids[k])
            assert e.value.code == _abi.SHZ_E_CANCELLED
            with pytest.raises(ShaderousError) as e:
                s.state(ids[k], reqs[k])
            assert e.value.code == _abi.SHZ_E_CANCELLED
        assert s.poll(ids[0]) == ("finished", reqs[0].steps) and s.poll(ids[2]) == ("finished", reqs[2].steps)
        got = {k: s.state(ids[k], reqs[k]) for k in (0, 2)}
        for k in (0, 2):
            assert s.result(ids[k]).steps == reqs[k].steps
    with Server(_cfg(1)) as s:
        ids = [s.submit(reqs[k]) for k in (0, 2)]
        s.drain()
        for i, k in zip(ids, (0, 2)):
            a1, a2 = s.state(i, reqs[k])
            assert np.array_equal(a1, got[k][0]) and np.array_equal(a2, got[k][1])
