"""Per-block timesteps on the GPU, against the reference's own checks of them (amr-time-bins and
amr-time-bins-32, src/validation/tests.ts:287-340 and :1644-1656): with blocks stepping up to 8
(32) times less often than the fastest, a 2D Sod tube's L1 density error < 0.003 (256 finest, 2
levels; 1024 finest, 4 levels) and a 3D Sedov blast's shock radius within 2% of the similarity
solution (128 finest, 2 levels; 3 levels); mass and energy drift < 1e-6 in both; Sedov makes under
85% of the block updates of single steps. Plus: the device's bins and work equal the oracle's
restatement of the bin passes on the same rates and table, and the pauses of
src/amr/amr_sim.ts:136-151 (16 single steps first; a pause when the cycles save too little)."""
import math

import numpy as np
import pytest

from oracle import bins as ob
from oracle.oracle import exact_riemann
from shaderous_b200 import Config, Problem
from shaderous_b200.amr import AmrConfig, AmrSim

pytestmark = pytest.mark.gpu

BS = 16
LEAF = 2


def used(tab):
    return [s for s in range(tab.shape[0]) if tab[s, 4] & 1]


def drift(d0, d1):
    return abs(d1.mass - d0.mass) / d0.mass, abs(d1.e_tot - d0.e_tot) / abs(d0.e_tot)


def top_bin(a):
    b, _ = a.bins()
    s, _, _ = a.leaves()
    return int(max(b[1 + x] for x in s))


@pytest.mark.parametrize("ndim,two_pass", [(2, False), (3, False), (2, True), (3, True)])
def test_bins_and_work_equal_the_oracle(ndim, two_pass):
    hyd = Config(gamma=1.4, bc_lo=(1, 1, 1), bc_hi=(1, 1, 1), recon="koren", cfl=0.8, p_floor=1e-12)
    K, lev = 3, 2
    cfg = AmrConfig(hydro=hyd, ndim=ndim, nr=4 if ndim == 2 else 2, max_level=lev, cap=400 if ndim == 2 else 1200,
                    regrid_every=0, time_bins=K, time_bins_always=True, two_pass=two_pass)
    with AmrSim(cfg) as a:
        a.reset(Problem("blast", a=(1, 10, 1, 0.1, 0.12)))
        assert a.bin_work()["paused"] == 16
        a.run(steps=16)
        w0 = a.bin_work()
        assert w0["paused"] == 0 and w0["cycles"] == 0
        for _ in range(3):
            w0 = a.bin_work()
            a.step(1)  # one cycle of 2^K substeps
            w1 = a.bin_work()
            tab = a.table()
            kb, rates = a.bins()
            _, dt, steps = a.clock()
            blocks = used(tab)
            want = ob.cycle_bins(tab, blocks, ndim, lev, rates, dt, hyd.cfl, K)
            for s in blocks:
                assert kb[1 + s] == want[1 + s], s
            assert w1["cycles"] == w0["cycles"] + 1
            assert w1["updates"] - w0["updates"] == ob.cycle_updates(tab, blocks, want, K, ndim)
            nleaf = sum(1 for s in blocks if tab[s, 4] & LEAF)
            assert w1["single"] - w0["single"] == nleaf << K
        assert steps == 16 + 3 * (1 << K)
        assert top_bin(a) >= 1  # the blast's surroundings step less often


@pytest.mark.parametrize("K,deeper,two_pass", [(3, 0, False), (5, 2, False), (3, 0, True)])
def test_sod_2d_with_bins_against_exact(K, deeper, two_pass):
    hyd = Config(gamma=1.4, bc_lo=(1, 1, 0), bc_hi=(1, 1, 0), p_floor=1e-12)
    cfg = AmrConfig(hydro=hyd, ndim=2, nr=4, max_level=2 + deeper, cap=3000, time_bins=K, time_bins_always=True,
                    two_pass=two_pass)
    with AmrSim(cfg) as a:
        a.reset(Problem("sod", a=(1, 0, 1, 0.125, 0, 0.1)))
        d0 = a.diagnostics()
        r = a.run(until=0.2)
        assert r.stopped == "time" and r.t == pytest.approx(0.2, rel=1e-9)
        d1 = a.diagnostics()
        slots, lv, co = a.leaves()
        u1, _ = a.leaves_state()
        top = top_bin(a)
        work = a.bin_work()
    assert work["cycles"] > 0 and top >= 1
    err = area = 0.0
    for i in range(len(slots)):
        dx = 1.0 / (4 * BS << lv[i])
        x = (co[i, 0] * BS + np.arange(BS) + 0.5) * dx - 0.5
        ex = exact_riemann((1, 0, 1), (0.125, 0, 0.1), 1.4, x / 0.2)[:, 0]
        rho = u1[i, :, 0].reshape(BS, BS).astype(np.float64)
        err += np.abs(rho - ex[None, :]).sum() * dx * dx
        area += BS * BS * dx * dx
    assert area == pytest.approx(1.0)
    assert err / area < 0.003, err
    assert max(drift(d0, d1)) < 1e-6, drift(d0, d1)


def shock_radius(slots, lv, co, u1, nr, nb=128):
    """tests.ts:268-285 leafShockRadius: the outermost radius at which the shell-averaged density
    falls through half way between its peak and the ambient 1."""
    bw = 0.5 / nb
    s = np.zeros(nb)
    v = np.zeros(nb)
    k, j, i = np.meshgrid(np.arange(BS), np.arange(BS), np.arange(BS), indexing="ij")
    for q in range(len(slots)):
        dx = 1.0 / (nr * BS << lv[q])
        x = (co[q, 0] * BS + i + 0.5) * dx - 0.5
        y = (co[q, 1] * BS + j + 0.5) * dx - 0.5
        z = (co[q, 2] * BS + k + 0.5) * dx - 0.5
        b = np.floor(np.sqrt(x * x + y * y + z * z) / bw).astype(np.int64).ravel()
        rho = u1[q, :, 0].astype(np.float64)
        m = b < nb
        np.add.at(s, b[m], rho[m] * dx ** 3)
        np.add.at(v, b[m], dx ** 3)
    prof = np.where(v > 0, s / np.maximum(v, 1e-300), 1.0)
    half = 0.5 * (prof.max() + 1)
    for b in range(nb - 1, 0, -1):
        if prof[b - 1] >= half:
            return (b - 0.5 + (prof[b - 1] - half) / (prof[b - 1] - prof[b])) * bw
    return math.nan


@pytest.mark.parametrize("K,levels,two_pass", [(3, 2, False), (5, 3, False), (3, 2, True)])
def test_sedov_3d_with_bins(K, levels, two_pass):
    hyd = Config(gamma=1.4, bc_lo=(1, 1, 1), bc_hi=(1, 1, 1), p_floor=1e-12)
    nr = 128 // (BS << levels)  # 128 cells across at the finest level
    cfg = AmrConfig(hydro=hyd, ndim=3, nr=nr, max_level=levels, cap=4000, time_bins=K, time_bins_always=True,
                    two_pass=two_pass)
    with AmrSim(cfg) as a:
        a.reset(Problem("sedov", a=(1.0, 1e-5, 1.0, 3.5)))
        d0 = a.diagnostics()
        r = a.run(until=0.06)
        assert r.stopped == "time"
        d1 = a.diagnostics()
        slots, lv, co = a.leaves()
        u1, _ = a.leaves_state()
        work = a.bin_work()
        top = top_bin(a)
    rad = shock_radius(slots, lv, co, u1, nr)
    want = 1.033 * (0.06 ** 2) ** 0.2
    assert abs(rad - want) / want < 0.02, (rad, want)
    assert max(drift(d0, d1)) < 1e-6, drift(d0, d1)
    assert work["cycles"] > 0 and top >= 1
    assert work["updates"] / work["single"] < 0.85, work


def test_cycles_pause_when_they_save_too_little():
    # a quiet uniform grid: every block in the fastest bin, the cycles save nothing
    hyd = Config(gamma=1.4, bc_lo=(0, 0, 0), bc_hi=(0, 0, 0))
    cfg = AmrConfig(hydro=hyd, ndim=2, nr=2, max_level=0, cap=64, regrid_every=0, time_bins=2)
    with AmrSim(cfg) as a:
        a.reset(Problem("sod", a=(1, 0, 1, 1, 0, 1)))
        assert a.bin_work()["paused"] == 16
        a.step(10)
        assert a.bin_work() == {"cycles": 0, "updates": 0, "single": 0, "paused": 6}
        a.step(6 + 4 * 4)  # the first single steps, then four cycles and the poll
        w = a.bin_work()
        assert w["cycles"] == 4 and w["updates"] == w["single"] == 4 * 4 * 4
        assert w["paused"] == 192
        _, _, steps = a.clock()
        assert steps == 16 + 16


@pytest.mark.parametrize("ndim,recon,bcs", [
    (2, "mc", ((2, 1, 0), (1, 0, 0))),
    (2, "minmod", ((0, 0, 0), (0, 0, 0))),
    (3, "minmod", ((2, 0, 1), (1, 2, 0))),
    (3, "mc", ((1, 1, 1), (2, 2, 2))),
])
def test_fused_cycles_equal_two_pass_cycles(ndim, recon, bcs):
    """The fused form of the cycles (one sweep per leaf, the neighbour-flux pass, the deposits) gives
    the two passes' state bit for bit, remeshes included."""
    hyd = Config(gamma=1.4, bc_lo=bcs[0], bc_hi=bcs[1], recon=recon, isentropic=False, cfl=0.6, p_floor=1e-12)
    out = []
    for two_pass in (False, True):
        cfg = AmrConfig(hydro=hyd, ndim=ndim, nr=2, max_level=2, cap=1200 if ndim == 3 else 300, refine_hi=0.1,
                        refine_lo=0.05, regrid_every=8, time_bins=3, time_bins_always=True, two_pass=two_pass)
        with AmrSim(cfg) as a:
            a.reset(Problem("blast", a=(1, 10, 1, 0.1, 0.15)))
            a.run(steps=16 + 5 * 8)
            out.append((a.leaves(), a.leaves_state(), a.clock(), a.bin_work(), top_bin(a)))
    (sa, la, ca), (ua1, ua2), clka, wa, ta = out[0]
    (sb, lb, cb), (ub1, ub2), clkb, wb, tb = out[1]
    assert ta >= 1 and wa["cycles"] == 5
    assert np.array_equal(la, lb) and np.array_equal(ca, cb)
    assert clka == clkb and wa == wb
    assert np.array_equal(ua1, ub1) and np.array_equal(ua2, ub2)


@pytest.mark.parametrize("case,two_pass", [("kh", False), ("kh", True), ("blast", False), ("blast", True)])
def test_periodic_runs_with_bins_conserve(case, two_pass):
    """Periodic boxes on two refined levels with 4 bins (a Kelvin-Helmholtz layer; a blast whose
    mesh follows it): nothing leaves the box, so mass, momentum and energy stay what they were
    (float32 state, float64 sums)."""
    hyd = Config(gamma=1.4, bc_lo=(0, 0, 0), bc_hi=(0, 0, 0), recon="koren", cfl=0.8)
    cfg = AmrConfig(hydro=hyd, ndim=2, nr=4, max_level=2, cap=800, refine_hi=0.05 if case == "kh" else 0.1,
                    refine_lo=0.02 if case == "kh" else 0.05, regrid_every=8, time_bins=2, time_bins_always=True,
                    two_pass=two_pass)
    with AmrSim(cfg) as a:
        if case == "kh":
            a.reset(Problem("kh", a=(2, 1, 0.5, 2.5, 0.01, 1e-3), seed=5))
        else:
            a.reset(Problem("blast", a=(1, 10, 1, 0.1, 0.12)))
        d0 = a.diagnostics()
        meshes = set()
        for _ in range(12):
            a.run(steps=16)
            _, lv, co = a.leaves()
            meshes.add(frozenset((int(x), *map(int, c)) for x, c in zip(lv, co)))
        d1 = a.diagnostics()
        work = a.bin_work()
        top = top_bin(a)
    assert work["cycles"] >= 40 and top >= 1
    if case == "blast":
        assert len(meshes) > 1  # the mesh followed the blast across re-meshes between cycles
    assert abs(d1.mass - d0.mass) / d0.mass < 1e-6
    assert abs(d1.e_tot - d0.e_tot) / d0.e_tot < 1e-6
    scale = abs(d0.mass)  # momentum per unit of mass moving at 1 (the flows' speeds are of order 1)
    assert abs(d1.momentum[0] - d0.momentum[0]) / scale < 1e-6
    assert abs(d1.momentum[1] - d0.momentum[1]) / scale < 1e-6


@pytest.mark.parametrize("ndim", [2, 3])
def test_bins_on_a_single_periodic_root(ndim):
    """One root block on a periodic box is its own neighbour across every face (the table's
    neighbour entry is the block itself): the bin rules, the flux pass and the deposits skip it as
    a neighbour. The one block is in the fastest bin; the cycles conserve."""
    hyd = Config(gamma=1.4, bc_lo=(0, 0, 0), bc_hi=(0, 0, 0), recon="mc", cfl=0.7)
    cfg = AmrConfig(hydro=hyd, ndim=ndim, nr=1, max_level=0, cap=4, regrid_every=8, time_bins=2,
                    time_bins_always=True)
    with AmrSim(cfg) as a:
        a.reset(Problem("blast", a=(1, 10, 1, 0.1, 0.2)))
        tab = a.table()
        assert all(int(tab[0, 6 + f]) == 0 for f in range(2 * ndim))
        d0 = a.diagnostics()
        a.run(steps=16 + 10 * 4)
        d1 = a.diagnostics()
        work = a.bin_work()
        kb, _ = a.bins()
    assert work["cycles"] == 10 and work["updates"] == work["single"] == 10 * 4 and kb[1] == 0
    assert abs(d1.mass - d0.mass) / d0.mass < 1e-6
    assert abs(d1.e_tot - d0.e_tot) / d0.e_tot < 1e-6
