"""The 2D step's two forms: the march along y (a CTA owns a row segment and marches it through
many rows) and the tile form (16 x 12 cells with a ring of halo cells). Both run the same per-cell
functions in the same order; being different kernels, they agree to rounding (the compiler may
contract a multiply and an add differently in each), while every depth of the march is the same
kernel and gives the same bits. The depth pin picks the form for the test; grids of 512 cells a
side and more march, smaller ones take the tile form."""
import numpy as np
import pytest

from shaderous_b200 import Config, Problem, Sim, tune

pytestmark = pytest.mark.gpu

KH = Problem("kh", a=(2, 1, 0.5, 2.5, 0.01, 1e-3), seed=7)
BLAST = Problem("blast", a=(1.0, 10.0, 1.0, 0.1, 0.15))


def _state(cfg, prob, rows, steps):
    tune.reset()
    tune.pin("uniform_sweep", 0, rows)
    try:
        with Sim(cfg) as s:
            s.reset(prob)
            s.run(steps=steps)
            return s.read_state(), s.clock()
    finally:
        tune.pin("uniform_sweep", None)


CASES = [
    # periodic Kelvin-Helmholtz, sizes that no segment or row count divides
    dict(n=(300, 170, 1), gamma=1.4, recon="ppm", prob=KH),
    dict(n=(253, 131, 1), gamma=1.4, recon="koren", isentropic=True, prob=KH),
    dict(n=(130, 260, 1), gamma=1.4, recon="mc", isentropic=False, prob=KH, riemann="hll"),
    # blasts against walls and open faces, mixed per axis and side
    dict(n=(200, 150, 1), recon="ppm", prob=BLAST, bc_lo=(1, 2, 0), bc_hi=(2, 1, 0)),
    dict(n=(127, 199, 1), recon="koren", isentropic=True, prob=BLAST, bc_lo=(2, 2, 0), bc_hi=(2, 2, 0)),
    dict(n=(256, 128, 1), recon="minmod", isentropic=False, prob=BLAST, bc_lo=(0, 1, 0), bc_hi=(0, 1, 0)),
    dict(n=(190, 90, 1), recon="vanleer", isentropic=True, prob=BLAST, bc_lo=(1, 0, 0), bc_hi=(1, 0, 0)),
]


@pytest.mark.parametrize("case", CASES, ids=lambda c: f"{c['recon']}-{c['n'][0]}x{c['n'][1]}")
def test_row_march_agrees_with_tile_form(case):
    case = dict(case)
    prob = case.pop("prob")
    cfg = Config(cfl=0.4, **case)
    (t1, t2), clk_t = _state(cfg, prob, 0, 12)
    (a1, a2), clk_a = _state(cfg, prob, 16, 12)
    assert clk_a[2] == clk_t[2] and abs(clk_a[0] - clk_t[0]) <= 1e-6 * clk_t[0]
    # 12 steps from the same state: within a few float32 roundings of each other
    for r, t in ((a1, t1), (a2, t2)):
        np.testing.assert_allclose(r, t, rtol=1e-5, atol=1e-6)
    for rows in (37, 256):
        (r1, r2), clk_r = _state(cfg, prob, rows, 12)
        assert clk_r == clk_a
        assert np.array_equal(r1, a1) and np.array_equal(r2, a2), rows


def test_tuner_tunes_the_march_depth_and_stays_exact():
    cfg = Config(n=(512, 512, 1), gamma=1.4, recon="koren", cfl=0.4)
    tune.reset()
    with Sim(cfg) as s:
        s.reset(KH)
        s.run(steps=5)
        a = s.read_state()
    ent = [e for e in tune.entries() if e["kernel"] == "uniform_sweep" and e["ndim"] == 2]
    assert len(ent) == 1 and ent[0]["candidates"] == 4 and ent[0]["tz"] in (8, 16, 32, 64)
    assert ent[0]["ms"] <= ent[0]["default_ms"]
    tune.enable(False)  # untuned: the march at its default depth
    try:
        with Sim(cfg) as s:
            s.reset(KH)
            s.run(steps=5)
            b = s.read_state()
    finally:
        tune.enable(True)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])


def test_small_2d_grids_take_the_tile_form_untuned():
    cfg = Config(n=(256, 384, 1), gamma=1.4, recon="koren", cfl=0.4)
    tune.reset()
    with Sim(cfg) as s:
        s.reset(KH)
        s.run(steps=3)
        a = s.read_state()
    assert not [e for e in tune.entries() if e["kernel"] == "uniform_sweep"]
    (t1, t2), _ = _state(cfg, KH, 0, 3)
    assert np.array_equal(a[0], t1) and np.array_equal(a[1], t2)
