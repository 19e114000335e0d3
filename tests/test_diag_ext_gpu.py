"""The extended diagnostics channels (ranges of density, temperature, scalar, pressure and speed;
the centre of mass) against the same quantities formed in float64 from the state read back, on a
uniform grid and on a refined block grid (hydro/diagnostics.wgsl channels 10-22)."""
import numpy as np
import pytest

from shaderous_b200 import Config, Problem, Sim
from shaderous_b200.amr import AmrConfig, AmrSim

pytestmark = pytest.mark.gpu


def expected(u1, u2, gamma, rho_floor, p_floor, dv, pos):
    """Ranges and centre of mass as the channels define them, from float32 cells (float64 math)."""
    u1 = u1.astype(np.float64)
    u2 = u2.astype(np.float64)
    gm1 = float(np.float32(gamma - 1.0))
    rho = np.maximum(u1[:, 0], float(np.float32(rho_floor)))
    eint = u2[:, 1]
    p = np.maximum(gm1 * eint, float(np.float32(p_floor)))
    T = gm1 * eint / rho
    s = u2[:, 2] / rho
    v = u1[:, 1:4] / rho[:, None]
    speed = np.sqrt((v ** 2).sum(1))
    fields = {"rho": rho, "temperature": T, "scalar": s, "pressure": p, "speed": speed}
    m = (rho * dv).sum()
    com = tuple((rho * dv * pos[:, a]).sum() / m for a in range(3))
    return {k: (f.min(), f.max()) for k, f in fields.items()}, com


def test_uniform_ranges_and_centre_of_mass():
    n = (32, 16, 16)
    cfg = Config(n=n, dx=1.0 / 32, gamma=1.4, bc_lo=(1, 1, 1), bc_hi=(1, 1, 1), cfl=0.4, recon="mc", p_floor=1e-12)
    with Sim(cfg) as s:
        s.reset(Problem("sod", a=(1, 0.3, 1, 0.125, 0, 0.1), axis=0))
        s.run(steps=10)
        d = s.diagnostics_ext()
        u1, u2 = s.read_state()
    k, j, i = np.meshgrid(np.arange(n[2]), np.arange(n[1]), np.arange(n[0]), indexing="ij")
    pos = np.stack([(i + 0.5 - n[0] / 2) / 32, (j + 0.5 - n[1] / 2) / 32, (k + 0.5 - n[2] / 2) / 32], -1).reshape(-1, 3)
    ranges, com = expected(u1, u2, 1.4, cfg.rho_floor, cfg.p_floor, (1 / 32) ** 3, pos)
    for name, (lo, hi) in ranges.items():
        assert d.ranges[name][0] == pytest.approx(lo, rel=1e-12, abs=1e-300), name
        assert d.ranges[name][1] == pytest.approx(hi, rel=1e-12, abs=1e-300), name
    assert com[0] < -0.05  # the dense left half pulls the centre of mass left
    assert d.com == pytest.approx(com, rel=1e-10, abs=1e-12)
    assert d.e_grav == 0.0 and d.jeans_unresolved == 0.0 and d.nuclear_heating == 0.0
    assert d.totals.mass == pytest.approx((np.maximum(u1[:, 0].astype(np.float64), 1e-10) * (1 / 32) ** 3).sum(),
                                          rel=1e-12)


def test_amr_ranges_and_centre_of_mass():
    hyd = Config(gamma=5 / 3, bc_lo=(1, 1, 0), bc_hi=(1, 1, 0), recon="koren", cfl=0.4, p_floor=1e-12)
    cfg = AmrConfig(hydro=hyd, ndim=2, nr=2, max_level=2, cap=400, refine_hi=0.1, refine_lo=0.05, regrid_every=4)
    with AmrSim(cfg) as a:
        a.reset(Problem("sod", a=(1, 0, 1, 0.125, 0, 0.1), axis=1))
        a.run(steps=12)
        d = a.diagnostics_ext()
        slots, lv, co = a.leaves()
        u1, u2 = a.leaves_state()
    assert lv.max() == 2
    dx0 = 1.0 / (2 * 16)
    pos, dvs = [], []
    j, i = np.meshgrid(np.arange(16), np.arange(16), indexing="ij")
    for b in range(len(slots)):
        dx = dx0 / (1 << int(lv[b]))
        x = (co[b, 0] * 16 + i + 0.5) * dx - 0.5
        y = (co[b, 1] * 16 + j + 0.5) * dx - 0.5
        pos.append(np.stack([x, y, np.zeros_like(x)], -1).reshape(-1, 3))
        dvs.append(np.full(256, dx * dx))
    ranges, com = expected(u1.reshape(-1, 4), u2.reshape(-1, 4), 5 / 3, hyd.rho_floor, hyd.p_floor,
                           np.concatenate(dvs), np.concatenate(pos))
    for name, (lo, hi) in ranges.items():
        assert d.ranges[name][0] == pytest.approx(lo, rel=1e-12, abs=1e-300), name
        assert d.ranges[name][1] == pytest.approx(hi, rel=1e-12, abs=1e-300), name
    assert com[1] < -0.05  # dense gas below y = 0
    assert d.com == pytest.approx(com, rel=1e-10, abs=1e-12)
