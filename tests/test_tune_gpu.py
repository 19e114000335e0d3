"""The launch-shape autotuner: tuning picks among launch shapes only, so a run that tunes gives the
same state, bit for bit, as a run with the tuner off; and the choices land in the table."""
import numpy as np
import pytest

from shaderous_b200 import Config, Problem, Sim, tune
from shaderous_b200.amr import AmrConfig, AmrSim

pytestmark = pytest.mark.gpu


def _uniform_state(tuned: bool):
    tune.reset()
    tune.enable(tuned)
    try:
        cfg = Config(n=(64, 64, 64), dx=2 * np.pi / 64, gamma=5 / 3, recon="ppm", cfl=0.4)
        with Sim(cfg) as s:
            s.reset(Problem("tgv", a=(1.0, 100.0, 1.0)))
            s.run(steps=6)
            return s.read_state()
    finally:
        tune.enable(True)


def test_uniform_sweep_tuning_is_exact():
    a1, a2 = _uniform_state(True)
    ent = [e for e in tune.entries() if e["kernel"] == "uniform_sweep"]
    b1, b2 = _uniform_state(False)
    assert np.array_equal(a1, b1) and np.array_equal(a2, b2)
    assert len(ent) == 1 and ent[0]["ndim"] == 3
    assert ent[0]["tz"] in (32, 64) and ent[0]["candidates"] == 2  # tz > 64 exceeds the 64 planes
    assert ent[0]["ms"] <= ent[0]["default_ms"]


def _amr_state(tuned: bool):
    tune.reset()
    tune.enable(tuned)
    try:
        hyd = Config(gamma=5 / 3, bc_lo=(1, 1, 1), bc_hi=(2, 2, 2), recon="koren", isentropic=True, cfl=0.4,
                     p_floor=1e-12)
        cfg = AmrConfig(hydro=hyd, ndim=3, nr=2, max_level=2, cap=1200, refine_hi=0.1, refine_lo=0.05, regrid_every=4)
        with AmrSim(cfg) as a:
            a.reset(Problem("blast", a=(1, 10, 1, 0.1, 0.2)))
            a.run(steps=12)
            return a.leaves(), a.leaves_state()
    finally:
        tune.enable(True)


def test_amr_tuning_is_exact():
    (s0, l0, c0), (u0, v0) = _amr_state(True)
    kinds = {e["kernel"] for e in tune.entries()}
    (s1, l1, c1), (u1, v1) = _amr_state(False)
    assert (l0 == l1).all() and (c0 == c1).all()
    assert np.array_equal(u0, u1) and np.array_equal(v0, v1)
    assert {"amr_assemble", "amr_sweep", "amr_fine_flux"} <= kinds
    for e in tune.entries():
        assert e["ms"] <= e["default_ms"]


def test_bounded_wait_reports_timeout():
    """The bounded-wait path of the TMA-staged sweeps, run for real without a fault: a wait on an
    mbarrier phase nothing completes gives up after its limit and sets the timeout code."""
    import ctypes as C

    from shaderous_b200 import _abi

    lib = _abi.load()
    code = C.c_int32(0)
    assert lib.shz_selftest_wait_timeout(0, C.byref(code)) == 0
    assert code.value == 1
