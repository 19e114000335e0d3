"""The float64 oracle pinned against the reference's own unit tests for its CPU scheme,
tests/unit/reference.test.ts, case by case with the same thresholds (citations per test)."""
import math

import numpy as np
import pytest

from oracle.oracle import RefHydro, exact_riemann, limiter

LIMITERS = ["mc", "vanleer", "minmod", "koren"]


def base(**over):
    """reference.test.ts:6-13 base()."""
    cfg = dict(n=(128, 1, 1), dx=1 / 128, gamma=1.4, bc_lo=(1, 0, 0), bc_hi=(1, 0, 0), cfl=0.8, rho_floor=1e-10,
               p_floor=1e-12, eta_dual=1e-3, shock_thresh=0.5, riemann="hllc", limiter="mc")
    cfg.update(over)
    return cfg


def tube(l, r):
    """reference.test.ts:14-17 tube()."""
    def f(x, y, z):
        rho, vx, p = l if x < 0 else r
        return (rho, vx, 0.0, 0.0, p, 1.0 if x < 0 else 0.0)
    return f


# --- exact Riemann solver (reference.test.ts:20-36) ----------------------------------------------

def test_exact_sod_star_state():
    sol = lambda xi: exact_riemann((1, 0, 1), (0.125, 0, 0.1), 1.4, xi)[0]
    star = sol(0.5)
    assert star[2] == pytest.approx(0.30313, abs=5e-5)
    assert star[1] == pytest.approx(0.92745, abs=5e-5)
    assert sol(-2)[0] == 1.0
    assert sol(2)[0] == 0.125
    assert sol(1.0)[0] == pytest.approx(0.26557, abs=5e-5)


def test_exact_strong_shock_toro3():
    star = exact_riemann((1, 0, 1000), (1, 0, 0.01), 1.4, 19)[0]
    assert star[2] == pytest.approx(460.894, abs=5e-3)
    assert star[1] == pytest.approx(19.5975, abs=5e-4)


# --- limiters (reference.test.ts:38-60) ----------------------------------------------------------

@pytest.mark.parametrize("kind", LIMITERS)
def test_limiters_vanish_keep_sign_exact_linear(kind):
    assert limiter(kind, 1, -1, 0) == 0
    assert limiter(kind, 0, 3, 0) == 0
    for a, b in [(1, 2), (2, 1), (-1, -4), (0.3, 0.3)]:
        s = limiter(kind, a, b, 0)
        assert math.copysign(1, s) == math.copysign(1, a) and s != 0
        assert abs(s) <= 2 * min(abs(a), abs(b)) + 1e-15
    assert limiter(kind, 0.3, 0.3, 0) == pytest.approx(0.3, abs=1e-14)


def test_koren_unlimited_where_smooth():
    assert limiter("koren", 0.001, -0.002, 1) == pytest.approx((0.001 - 0.004) / 3, abs=1e-14)
    assert limiter("koren", 0.001, -0.002, 0) == 0
    assert limiter("koren", 0.5, -0.5, 1) == 0


# --- the float64 scheme (reference.test.ts:62-150) ---------------------------------------------

def test_converges_on_sod_tube():
    def err(n):
        h = RefHydro(**base(n=(n, 1, 1), dx=1 / n))
        h.init(tube((1, 0, 1), (0.125, 0, 0.1)))
        h.run(0.2)
        assert h.t == pytest.approx(0.2, abs=1e-12)
        x = ((np.arange(n) + 0.5) / n - 0.5) / 0.2
        ex = exact_riemann((1, 0, 1), (0.125, 0, 0.1), 1.4, x)[:, 0]
        return np.abs(h.U[0] - ex).sum() / n

    e64, e128 = err(64), err(128)
    assert e128 < 0.005
    assert e128 < 0.7 * e64


def test_second_order_on_smooth_advection():
    def err(n):
        h = RefHydro(**base(n=(n, 1, 1), dx=1 / n, bc_lo=(0, 0, 0), bc_hi=(0, 0, 0)))
        rho0 = lambda x: 1.5 + 0.2 * math.sin(2 * math.pi * x)
        h.init(lambda x, y, z: (rho0(x), 1.0, 0.0, 0.0, 1.0, 0.0))
        h.run(1)
        xs = (np.arange(n) + 0.5) / n - 0.5
        return np.abs(h.U[0] - (1.5 + 0.2 * np.sin(2 * np.pi * xs))).sum() / n

    assert math.log2(err(32) / err(64)) > 1.7


def test_conserves_in_periodic_box():
    h = RefHydro(**base(n=(16, 16, 4), dx=1 / 16, bc_lo=(0, 0, 0), bc_hi=(0, 0, 0)))
    h.init(lambda x, y, z: (1.5 + math.exp(-(x * x + y * y) / 0.02), 1.0, 0.5, 0.1 * math.sin(8 * math.pi * z),
                            1 + 0.5 * math.exp(-(x * x + y * y) / 0.01), 0.0))
    before = [h.U[i].sum() for i in (0, 1, 2, 4)]
    for _ in range(40):
        h.step()
    after = [h.U[i].sum() for i in (0, 1, 2, 4)]
    for b, a in zip(before, after):
        assert abs(a - b) / abs(b) < 1e-12


def test_positive_through_pressure_ratio_1e5():
    h = RefHydro(**base())
    h.init(tube((1, 0, 1000), (1, 0, 0.01)))
    h.run(0.012)
    U = h.U
    assert (U[0] > 0.5).all()
    assert (0.4 * U[5] > 0.009).all()


def test_same_answer_along_x_y_z():
    def run(axis):
        dims = [1, 1, 1]
        dims[axis] = 48
        bc = [0, 0, 0]
        bc[axis] = 1
        h = RefHydro(**base(n=tuple(dims), dx=1 / 48, bc_lo=tuple(bc), bc_hi=tuple(bc)))

        def f(x, y, z):
            s = (x, y, z)[axis]
            v = [0.0, 0.0, 0.0]
            v[axis] = 0.3
            return (1.0 if s < 0 else 0.125, v[0], v[1], v[2], 1.0 if s < 0 else 0.1, 0.0)

        h.init(f)
        h.run(0.15)
        return h.U[0].copy()

    x = run(0)
    assert np.array_equal(run(1), x)
    assert np.array_equal(run(2), x)


def test_reflecting_walls_symmetric_and_closed():
    h = RefHydro(**base(n=(32, 1, 1), dx=1 / 32, bc_lo=(2, 0, 0), bc_hi=(2, 0, 0)))
    h.init(lambda x, y, z: (1.0, 0.0, 0.0, 0.0, 10.0 if abs(x) < 0.1 else 0.1, 0.0))
    m0 = h.U[0].sum()
    h.run(0.5)
    U = h.U
    assert abs(U[0].sum() - m0) / m0 < 1e-12
    for i in range(16):
        assert U[0][i] == pytest.approx(U[0][31 - i], abs=1e-10)


# --- the switches the reference's GPU path turns on (isentropic reconstruction, koren) ----------

@pytest.mark.parametrize("kind", LIMITERS)
def test_isentropic_sod_converges(kind):
    n = 128
    h = RefHydro(**base(n=(n, 1, 1), dx=1 / n, limiter=kind, isentropic=True))
    h.init(tube((1, 0, 1), (0.125, 0, 0.1)))
    h.run(0.2)
    x = ((np.arange(n) + 0.5) / n - 0.5) / 0.2
    ex = exact_riemann((1, 0, 1), (0.125, 0, 0.1), 1.4, x)[:, 0]
    assert np.abs(h.U[0] - ex).sum() / n < 0.006


def test_ppm_extension_sod_and_smooth_order():
    """PPM (Colella & Woodward 1984) has no reference counterpart: it is held to the same scheme
    properties the reference tests ask of its limiters."""
    n = 128
    h = RefHydro(**base(n=(n, 1, 1), dx=1 / n, limiter="ppm"))
    h.init(tube((1, 0, 1), (0.125, 0, 0.1)))
    h.run(0.2)
    x = ((np.arange(n) + 0.5) / n - 0.5) / 0.2
    ex = exact_riemann((1, 0, 1), (0.125, 0, 0.1), 1.4, x)[:, 0]
    assert np.abs(h.U[0] - ex).sum() / n < 0.005

    def err(n):
        h = RefHydro(**base(n=(n, 1, 1), dx=1 / n, bc_lo=(0, 0, 0), bc_hi=(0, 0, 0), limiter="ppm"))
        h.init(lambda x, y, z: (1.5 + 0.2 * math.sin(2 * math.pi * x), 1.0, 0.0, 0.0, 1.0, 0.0))
        h.run(1)
        xs = (np.arange(n) + 0.5) / n - 0.5
        return np.abs(h.U[0] - (1.5 + 0.2 * np.sin(2 * np.pi * xs))).sum() / n

    assert math.log2(err(32) / err(64)) > 1.7
