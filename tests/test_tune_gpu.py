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


def _pinned_amr(variant, ndim, two_pass, bcs):
    tune.reset()
    tune.pin("amr_assemble", variant)
    try:
        hyd = Config(gamma=5 / 3, bc_lo=bcs[0], bc_hi=bcs[1], recon="koren", isentropic=True, cfl=0.4, p_floor=1e-12)
        cfg = AmrConfig(hydro=hyd, ndim=ndim, nr=2, max_level=2, cap=1500 if ndim == 3 else 300, refine_hi=0.1,
                        refine_lo=0.05, regrid_every=4, two_pass=two_pass)
        with AmrSim(cfg) as a:
            a.reset(Problem("blast", a=(1, 10, 1, 0.1, 0.2)))
            a.run(steps=14)
            _, lv, co = a.leaves()
            return lv, co, a.leaves_state()
    finally:
        tune.pin("amr_assemble", None)


@pytest.mark.parametrize("ndim,two_pass,bcs", [
    (3, False, ((1, 2, 0), (2, 1, 0))),
    (3, True, ((2, 2, 2), (1, 1, 1))),
    (2, False, ((0, 2, 0), (0, 1, 0))),
    (2, True, ((1, 1, 0), (2, 2, 0))),
])
def test_every_assemble_variant_gives_the_same_state(ndim, two_pass, bcs):
    """The one-pass assemble at each register budget and the split form (a light pass for own cells
    and same-level ghosts, then the ghosts beyond level changes over only the blocks the host lists
    for them; in order, or side by side on two streams) on refined meshes with walls, outflow and
    periodic faces: the same state bit for bit."""
    ref = _pinned_amr(0, ndim, two_pass, bcs)
    assert len(set(ref[0].tolist())) > 1  # the mesh has level changes
    for v in (1, 2, 3, 4, 5, 6):
        lv, co, (u1, u2) = _pinned_amr(v, ndim, two_pass, bcs)
        assert (lv == ref[0]).all() and (co == ref[1]).all()
        assert np.array_equal(u1, ref[2][0]) and np.array_equal(u2, ref[2][1]), v


def test_served_blocks_skip_the_second_pass_and_agree():
    """Served grids are uniform (no level changes): the split form's second pass has no blocks, and
    the results equal the one-pass kernel's."""
    from shaderous_b200.serve import Request, Server, ServerConfig

    reqs = [Request(ndim=2, n=64, steps=21, problem=Problem("kh", a=(2, 1, 0.5, 2.5, 0.01, 1e-3), seed=3), gamma=1.4, bc=0),
            Request(ndim=3, n=32, steps=11, problem=Problem("blast", a=(3, 50, 1, 1, 0.15)), gamma=5 / 3, bc=2),
            Request(ndim=3, n=48, steps=7, problem=Problem("sod", a=(2, 0, 5, 1, 0, 1)), gamma=1.4, bc=1)]
    out = []
    for v in (0, 3):
        tune.reset()
        tune.pin("amr_assemble", v)
        try:
            cfg = ServerConfig(hydro=Config(recon="koren", isentropic=True, cfl=0.4), budget_bytes=2e9, max_grids=8,
                               round_steps=4, keep_states=True)
            with Server(cfg) as s:
                ids = [s.submit(r) for r in reqs]
                s.drain()
                out.append([s.state(i, r) for r, i in zip(reqs, ids)])
        finally:
            tune.pin("amr_assemble", None)
    for (a1, a2), (b1, b2) in zip(*out):
        assert np.array_equal(a1, b1) and np.array_equal(a2, b2)


@pytest.mark.parametrize("ndim,two_pass", [(3, False), (2, False), (2, True)])
def test_substep_assemble_variants_give_the_same_state(ndim, two_pass):
    """With per-block timesteps, the substeps' assemble in one pass and in the split form (its
    second pass over every block, with half-step ghosts of neighbours part way through their step)
    give the same state, bins and work, bit for bit."""
    out = []
    for v in (1, 3):
        tune.reset()
        tune.pin("amr_assemble_bins", v)
        try:
            hyd = Config(gamma=5 / 3, bc_lo=(1, 2, 0), bc_hi=(1, 1, 0), recon="koren", isentropic=True, cfl=0.4,
                         p_floor=1e-12)
            cfg = AmrConfig(hydro=hyd, ndim=ndim, nr=2 if ndim == 3 else 4, max_level=2, cap=1500 if ndim == 3 else 400,
                            refine_hi=0.1, refine_lo=0.05, regrid_every=8, two_pass=two_pass, time_bins=3,
                            time_bins_always=True)
            with AmrSim(cfg) as a:
                a.reset(Problem("blast", a=(1, 10, 1, 0.1, 0.2)))
                a.run(steps=48)
                _, lv, co = a.leaves()
                out.append((lv, co, a.leaves_state(), a.bins()[0], a.bin_work()))
        finally:
            tune.pin("amr_assemble_bins", None)
    (l0, c0, (u0, v0), b0, w0), (l1, c1, (u1, v1), b1, w1) = out
    assert len(set(l0.tolist())) > 1 and w0["cycles"] > 0
    assert (l0 == l1).all() and (c0 == c1).all() and (b0 == b1).all() and w0 == w1
    assert np.array_equal(u0, u1) and np.array_equal(v0, v1)
