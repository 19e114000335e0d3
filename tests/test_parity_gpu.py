"""GPU parity: the CUDA path (through the C ABI) against the float64 oracle on identical inputs.

Both start from the same float32 state (the oracle reads it as float64), take the same number of
steps with their own dt, and are compared per conserved variable by the relative L1 error
sum|gpu - ref| / sum|ref| and the L-infinity error, the measure of the reference's gpu-vs-cpu
validation (src/validation/tests.ts:2365-2403, tolerance 1e-4, recorded 7.8e-8 / 7.8e-9).

Tolerances (float32 state and fluxes against float64):
  - smooth flows: relative L1 of density <= 1e-5 (the stated gate), other variables <= 1e-4;
  - flows with shocks, after tens of steps: relative L1 <= 1e-4 (the reference's own bound).
"""
import math

import numpy as np
import pytest

from oracle.oracle import RefHydro, exact_riemann
from shaderous_b200 import Config, Problem, Sim, problem_prims, prims_to_state

pytestmark = pytest.mark.gpu

VARS = ["rho", "mx", "my", "mz", "E", "eint", "rhos"]


def as7(u1, u2):
    return np.concatenate([np.asarray(u1, np.float64).T, np.asarray(u2, np.float64).T[:3]], axis=0)


def rel_l1(g, r):
    """Relative L1 error per conserved variable; a momentum component is measured against the
    L1 of the momentum's magnitude (a component that starts at zero, as w in the Taylor-Green
    vortex, has no scale of its own)."""
    out = {}
    mom = np.sqrt(r[1] ** 2 + r[2] ** 2 + r[3] ** 2).sum()
    for i, name in enumerate(VARS):
        den = mom if name in ("mx", "my", "mz") else np.abs(r[i]).sum()
        out[name] = np.abs(g[i] - r[i]).sum() / den if den > 0 else np.abs(g[i] - r[i]).max()
    return out


def oracle_for(cfg: Config, threads=8):
    return RefHydro(n=cfg.n, dx=cfg.dx if cfg.dx is not None else 1.0 / cfg.n[0], gamma=cfg.gamma, bc_lo=cfg.bc_lo,
                    bc_hi=cfg.bc_hi, cfl=cfg.cfl, rho_floor=cfg.rho_floor, p_floor=cfg.p_floor, eta_dual=cfg.eta_dual,
                    shock_thresh=cfg.shock_thresh, riemann=cfg.riemann, limiter=cfg.recon,
                    isentropic=cfg.isentropic and cfg.recon != "ppm", signal_dims=cfg.signal_dims, threads=threads)


def run_pair(cfg: Config, prob: Problem, steps: int):
    """Run `steps` steps on the GPU and in the oracle from the same float32 state."""
    u1, u2 = prims_to_state(problem_prims(cfg, prob), cfg.gamma)
    with Sim(cfg) as s:
        s.set_state(u1, u2)
        r = s.run(steps=steps)
        assert r.taken == steps
        g1, g2 = s.read_state()
        t_gpu = r.t
    ref = oracle_for(cfg)
    ref.set_state32(u1, u2)
    for _ in range(steps):
        ref.step()
    return as7(g1, g2), ref.U, t_gpu, ref.t


def check(g, r, tol_rho, tol_other, label):
    e = rel_l1(g, r)
    assert np.isfinite(g).all(), label
    assert e["rho"] <= tol_rho, (label, e)
    for k in ("mx", "my", "mz", "E", "eint"):
        if np.abs(r[VARS.index(k)]).sum() > 1e-6 * np.abs(r[4]).sum():
            assert e[k] <= tol_other, (label, k, e)
    return e


# --- the benchmark configurations, at sizes the oracle finishes in seconds -----------------------

def test_sod_512_minmod_hllc_to_t02():
    """1D Sod, 512 cells on [0,1], minmod + HLLC, CFL 0.4, to t = 0.2 (the first configuration)."""
    cfg = Config(n=(512, 1, 1), gamma=1.4, bc_lo=(1, 0, 0), bc_hi=(1, 0, 0), cfl=0.4, p_floor=1e-12, recon="minmod",
                 riemann="hllc")
    prob = Problem("sod", a=(1, 0, 1, 0.125, 0, 0.1))
    u1, u2 = prims_to_state(problem_prims(cfg, prob), cfg.gamma)
    with Sim(cfg) as s:
        s.set_state(u1, u2)
        r = s.run(until=0.2)
        assert r.stopped == "time"
        assert r.t == pytest.approx(0.2, abs=1e-12)
        g = as7(*s.read_state())
    ref = oracle_for(cfg)
    ref.set_state32(u1, u2)
    ref.run(0.2)
    assert ref.t == pytest.approx(0.2, abs=1e-12)
    assert r.steps == ref.steps
    check(g, ref.U, 1e-5, 1e-4, "sod512")
    # both against the exact solution (the reference test's L1 < 0.005 at 128 cells)
    x = ((np.arange(512) + 0.5) / 512 - 0.5) / 0.2
    ex = exact_riemann((1, 0, 1), (0.125, 0, 0.1), 1.4, x)[:, 0]
    assert np.abs(g[0] - ex).mean() < 0.003


@pytest.mark.parametrize("recon", ["minmod", "mc", "koren"])
def test_kh_2d(recon):
    """2D Kelvin-Helmholtz slab, periodic (the second configuration, at 128^2, 50 steps)."""
    n = 128
    cfg = Config(n=(n, n, 1), gamma=1.4, cfl=0.4, recon=recon)
    prob = Problem("kh", a=(2, 1, 0.5, 2.5, 0.01, 1e-3), seed=1234)
    g, r, tg, tr = run_pair(cfg, prob, 50)
    assert tg == pytest.approx(tr, rel=1e-6)
    check(g, r, 1e-5, 1e-4, f"kh-{recon}")


def test_kh_1024_1000_steps_as_configured():
    """The second configuration as stated: 2D Kelvin-Helmholtz at 1024^2, periodic, gamma 1.4,
    MC + HLLC, CFL 0.4, 1000 steps, against the oracle at 1024^2 from the same float32 state.

    The seeded shear layer amplifies differences, so the tolerance is stated against the step
    count: at 250, 500 and 1000 steps the relative L1 of density stays <= 1e-5 and the relative
    difference of the transverse kinetic energy sum(my^2 / rho) (the instability's growth) <= 1e-4.
    (The reference's own check of this flow is qualitative, src/validation/tests.ts:607-610.)"""
    import os

    n = 1024
    cfg = Config(n=(n, n, 1), dx=1.0 / n, gamma=1.4, cfl=0.4, recon="mc", riemann="hllc", isentropic=False)
    prob = Problem("kh", a=(2, 1, 0.5, 2.5, 0.01, 1e-3), seed=20240601)
    u1, u2 = prims_to_state(problem_prims(cfg, prob), cfg.gamma)
    ref = oracle_for(cfg, threads=os.cpu_count() or 8)
    ref.set_state32(u1, u2)
    lines = ["| steps | t | rel. L1 density | rel. L-inf density | transverse KE (oracle) | rel. diff. transverse KE |",
             "|---|---|---|---|---|---|"]
    failures = []
    with Sim(cfg) as s:
        s.set_state(u1, u2)
        done = 0
        for upto in (250, 500, 1000):
            s.run(steps=upto - done)
            for _ in range(upto - done):
                ref.step()
            done = upto
            g = as7(*s.read_state())
            r = ref.U
            e1 = np.abs(g[0] - r[0]).sum() / np.abs(r[0]).sum()
            ei = np.abs(g[0] - r[0]).max() / np.abs(r[0]).max()
            ke_g = (g[2] ** 2 / g[0]).sum()
            ke_r = (r[2] ** 2 / r[0]).sum()
            dke = abs(ke_g - ke_r) / ke_r
            t, _, steps = s.clock()
            assert steps == upto == ref.steps and t == pytest.approx(ref.t, rel=1e-6)
            lines.append(f"| {upto} | {t:.5f} | {e1:.2e} | {ei:.2e} | {ke_r / n ** 2:.4e} | {dke:.2e} |")
            if not (e1 <= 1e-5 and dke <= 1e-4):
                failures.append((upto, e1, dke))
    table = "\n".join(lines)
    print("\n" + table)
    if os.environ.get("SHZ_KH_REPORT"):
        with open(os.environ["SHZ_KH_REPORT"], "w") as f:
            f.write(table + "\n")
    assert not failures, failures


def test_tgv_3d_ppm():
    """3D Taylor-Green vortex, PPM + HLLC (the third configuration, at 32^3, 20 steps)."""
    n = 32
    cfg = Config(n=(n, n, n), dx=2 * math.pi / n, gamma=5 / 3, cfl=0.4, recon="ppm")
    prob = Problem("tgv", a=(1, 100, 1))
    g, r, tg, tr = run_pair(cfg, prob, 20)
    assert tg == pytest.approx(tr, rel=1e-6)
    check(g, r, 1e-5, 1e-4, "tgv-ppm")


# --- the reference's own gpu-vs-cpu validation cases (tests.ts:2365-2403): 32^3, 20 steps -------

def test_gpu_vs_cpu_sod_diagonal_32():
    n = 32
    cfg = Config(n=(n, n, n), gamma=1.4, bc_lo=(1, 1, 1), bc_hi=(1, 1, 1), p_floor=1e-12, recon="koren")
    # a diagonal tube: x + y + z < 0 on the left
    prims = problem_prims(cfg, Problem("sod", a=(1, 0, 1, 0.125, 0, 0.1)))
    idx = np.arange(n)
    c = (idx + 0.5) / n - 0.5
    X, Y, Z = np.meshgrid(c, c, c, indexing="ij")
    left = (X + Y + Z < 0).transpose(2, 1, 0).reshape(-1)
    prims[:, 0] = np.where(left, 1.0, 0.125)
    prims[:, 4] = np.where(left, 1.0, 0.1)
    prims[:, 5] = left.astype(float)
    u1, u2 = prims_to_state(prims, 1.4)
    with Sim(cfg) as s:
        s.set_state(u1, u2)
        s.run(steps=20)
        g = as7(*s.read_state())
    ref = oracle_for(cfg)
    ref.set_state32(u1, u2)
    for _ in range(20):
        ref.step()
    e = check(g, ref.U, 1e-4, 1e-4, "sod-diag")
    assert e["E"] <= 1e-4


def test_gpu_vs_cpu_sedov_32():
    n = 32
    cfg = Config(n=(n, n, n), gamma=1.4, bc_lo=(1, 1, 1), bc_hi=(1, 1, 1), p_floor=1e-12, recon="koren")
    g, r, _, _ = run_pair(cfg, Problem("sedov", a=(1, 1e-5, 1, 3.5)), 20)
    e = check(g, r, 1e-4, 1e-4, "sedov")
    assert e["E"] <= 1e-4


# --- every reconstruction and switch, boundaries on every face --------------------------------

@pytest.mark.parametrize("recon", ["minmod", "mc", "vanleer", "koren", "ppm"])
@pytest.mark.parametrize("isen", [False, True])
def test_recon_switches_smooth_3d(recon, isen):
    if recon == "ppm" and isen:
        pytest.skip("the density along the adiabat is a PLM switch")
    n = 24
    cfg = Config(n=(n, n, n), gamma=1.4, recon=recon, isentropic=isen, cfl=0.5)
    prob = Problem("gauss", a=(1.5, 0.02, 1.0, 0.5, 0.1, 1.0, 0.01))
    g, r, _, _ = run_pair(cfg, prob, 10)
    check(g, r, 1e-5, 1e-4, f"{recon}-{isen}")


@pytest.mark.parametrize("bc", [(1, 1), (2, 2), (1, 2), (2, 0)])
@pytest.mark.parametrize("recon", ["koren", "ppm"])
def test_boundaries_3d_blast(bc, recon):
    lo, hi = bc
    n = 20
    cfg = Config(n=(n, n + 4, n - 2), gamma=5 / 3, bc_lo=(lo, hi, lo), bc_hi=(hi, lo, hi), recon=recon, cfl=0.5)
    prob = Problem("blast", a=(1, 10, 1, 0.1, 0.2))
    g, r, _, _ = run_pair(cfg, prob, 15)
    check(g, r, 1e-4, 1e-4, f"bc{bc}-{recon}")


@pytest.mark.parametrize("dims", [(300, 1, 1), (70, 45, 1), (40, 20, 70)])
def test_ragged_sizes_and_hll(dims):
    """Grids that no tile divides; HLL; reflecting and outflow walls."""
    cfg = Config(n=dims, gamma=1.4, bc_lo=(2, 1, 0), bc_hi=(1, 2, 0), riemann="hll", recon="mc", cfl=0.6)
    if dims[2] == 1:
        cfg.bc_lo = (2, 1 if dims[1] > 1 else 0, 0)
        cfg.bc_hi = (1, 2 if dims[1] > 1 else 0, 0)
    prob = Problem("blast", a=(1, 10, 0.5, 0.1, 0.15))
    g, r, _, _ = run_pair(cfg, prob, 12)
    check(g, r, 1e-4, 1e-4, f"ragged{dims}")


# --- scheme properties at full sizes ----------------------------------------------------------

def test_conservation_periodic_fp64_totals():
    """Periodic box: mass, momentum and energy totals (float64 compensated sums on the device)
    stay put to float32 round-off; and they match a host float64 sum of the state."""
    n = 64
    cfg = Config(n=(n, n, n), gamma=1.4, recon="koren")
    with Sim(cfg) as s:
        s.reset(Problem("gauss", a=(1.5, 0.02, 1.0, 0.5, 0.1, 1.0, 0.01)))
        d0 = s.diagnostics()
        u1, u2 = s.read_state()
        dv = (1 / n) ** 3
        assert d0.mass == pytest.approx(np.asarray(u1[:, 0], np.float64).sum() * dv, rel=1e-12)
        assert d0.e_tot == pytest.approx(np.asarray(u2[:, 0], np.float64).sum() * dv, rel=1e-12)
        s.run(steps=100)
        d1 = s.diagnostics()
    assert abs(d1.mass - d0.mass) / d0.mass < 2e-6
    assert abs(d1.e_tot - d0.e_tot) / d0.e_tot < 2e-6
    assert abs(d1.momentum[0] - d0.momentum[0]) / abs(d0.momentum[0]) < 2e-6
    assert d1.steps == 100


def test_axis_permutation_3d():
    """sod-axes (tests.ts:523-538): a tube along x, y and z gives the same profile (< 1e-6)."""
    n = 32
    profiles = []
    for axis in range(3):
        cfg = Config(n=(n, n, n), gamma=1.4, bc_lo=(1, 1, 1), bc_hi=(1, 1, 1), recon="koren")
        with Sim(cfg) as s:
            s.reset(Problem("sod", axis=axis, a=(1, 0, 1, 0.125, 0, 0.1)))
            s.run(steps=30)
            u1, _ = s.read_state()
        rho = u1[:, 0].reshape(n, n, n)  # (z, y, x)
        prof = [rho[0, 0, :], rho[0, :, 0], rho[:, 0, 0]][axis]
        # planar: every line along the axis is the same
        line = [rho[n // 2, n // 3, :], rho[n // 2, :, n // 3], rho[:, n // 2, n // 3]][axis]
        assert np.abs(line - prof).max() < 1e-5
        profiles.append(prof.astype(np.float64))
    assert np.abs(profiles[1] - profiles[0]).max() < 1e-6
    assert np.abs(profiles[2] - profiles[0]).max() < 1e-6


def test_run_until_lands_and_holds():
    cfg = Config(n=(64, 64, 1), gamma=1.4, recon="mc", t_end=0.05)
    with Sim(cfg) as s:
        s.reset(Problem("blast", a=(1, 10, 1, 0.1, 0.1)))
        r = s.run(until=0.02)
        assert r.stopped == "time" and r.t == pytest.approx(0.02, abs=1e-12)
        r2 = s.run(steps=100000)
        assert r2.stopped == "end" and r2.t == pytest.approx(0.05, abs=1e-12)
        a1, _ = s.read_state()
        s.step(3)  # held at the end: the state stays as it is
        b1, _ = s.read_state()
        assert np.array_equal(a1, b1)
        assert s.clock()[2] == r2.steps


def test_refusals_as_errors():
    from shaderous_b200 import ShaderousError

    with pytest.raises(ShaderousError):
        Sim(Config(n=(1, 8, 8)))
    with pytest.raises(ShaderousError):
        Sim(Config(n=(64, 1, 1), bc_lo=(1, 2, 0), bc_hi=(1, 2, 0)))
    with Sim(Config(n=(64, 1, 1))) as s:
        with pytest.raises(ValueError):
            s.run()
        with pytest.raises(ShaderousError):
            s.set_state(np.zeros((10, 4), np.float32), np.zeros((10, 4), np.float32))


# --- the per-variable error report of every configuration ------------------------------------------

def rel_linf(g, r):
    """Relative L-infinity error per conserved variable (momentum against the largest momentum
    magnitude, as for L1)."""
    out = {}
    mom = np.sqrt(r[1] ** 2 + r[2] ** 2 + r[3] ** 2).max()
    for i, name in enumerate(VARS):
        den = mom if name in ("mx", "my", "mz") else np.abs(r[i]).max()
        out[name] = np.abs(g[i] - r[i]).max() / den if den > 0 else np.abs(g[i] - r[i]).max()
    return out


# (configuration, steps or None for the Sod run to t = 0.2, L1 bound, L-inf bound): every
# variable's relative L1 error <= 1e-5 (the stated gate, here for shocked flows too) and relative
# L-inf error <= 1e-4. Measured on a B200: L1 <= 5.2e-6, L-inf <= 2.3e-5 (Taylor-Green momentum).
REPORT = [
    ("sod 512, minmod+HLLC, to t=0.2", Config(n=(512, 1, 1), gamma=1.4, bc_lo=(1, 0, 0), bc_hi=(1, 0, 0), cfl=0.4,
                                             p_floor=1e-12, recon="minmod"),
     Problem("sod", a=(1, 0, 1, 0.125, 0, 0.1)), None, 1e-5, 1e-4),
    ("kh 256^2, mc+HLLC, 200 steps", Config(n=(256, 256, 1), gamma=1.4, cfl=0.4, recon="mc"),
     Problem("kh", a=(2, 1, 0.5, 2.5, 0.01, 1e-3), seed=1234), 200, 1e-5, 1e-4),
    ("tgv 128^3, PPM+HLLC, 200 steps", Config(n=(128, 128, 128), dx=2 * math.pi / 128, gamma=5 / 3, cfl=0.4,
                                              recon="ppm"),
     Problem("tgv", a=(1.0, 100.0, 1.0)), 200, 1e-5, 1e-4),
    ("sedov 64^3, koren+HLLC, 40 steps", Config(n=(64, 64, 64), gamma=5 / 3, cfl=0.5, recon="koren",
                                                bc_lo=(1, 1, 1), bc_hi=(1, 1, 1), p_floor=1e-12),
     Problem("sedov", a=(1.0, 1e-5, 1.0, 3.5)), 40, 1e-5, 1e-4),
]


def test_parity_report():
    """L1 and L-infinity error per conserved variable for each configuration, printed as a table
    (and written to $SHZ_PARITY_REPORT when set), each held to its bound."""
    import os

    lines = ["| configuration | variable | rel. L1 | rel. L-inf |", "|---|---|---|---|"]
    failures = []
    for label, cfg, prob, steps, tol1, tolinf in REPORT:
        u1, u2 = prims_to_state(problem_prims(cfg, prob), cfg.gamma)
        with Sim(cfg) as s:
            s.set_state(u1, u2)
            r = s.run(until=0.2) if steps is None else s.run(steps=steps)
            g = as7(*s.read_state())
        ref = oracle_for(cfg, threads=os.cpu_count() or 8)
        ref.set_state32(u1, u2)
        if steps is None:
            ref.run(0.2)
        else:
            for _ in range(steps):
                ref.step()
        assert ref.steps == r.steps, label
        e1, ei = rel_l1(g, ref.U), rel_linf(g, ref.U)
        for k in ("rho", "mx", "my", "mz", "E", "eint"):
            if np.abs(ref.U[VARS.index(k)]).sum() <= 1e-6 * np.abs(ref.U[4]).sum():
                continue  # a variable that stays zero (collapsed axes)
            lines.append(f"| {label} | {k} | {e1[k]:.2e} | {ei[k]:.2e} |")
            if not (e1[k] <= tol1 and ei[k] <= tolinf):
                failures.append((label, k, e1[k], ei[k]))
    table = "\n".join(lines)
    print("\n" + table)
    if os.environ.get("SHZ_PARITY_REPORT"):
        with open(os.environ["SHZ_PARITY_REPORT"], "w") as f:
            f.write(table + "\n")
    assert not failures, failures
