"""The adaptive block grid on the GPU, against the reference's own checks for it.

- ghost indexing: the device's classification of every ghost texel equals the reference's rule
  (src/amr/grid.wgsl:186-222 ghost_src) evaluated on the same block table;
- amr-unrefined (src/validation/tests.ts:1203): blocks at one level give the uniform grid's
  answer (the reference's bound 1e-5 relative);
- conservation through re-meshes, with fine-flux matching (amr-shock-tube's drift < 1e-6,
  tests.ts:1231, here float32 totals over many steps: < 2e-6);
- a refined Sod tube against the exact solution.
"""
import math

import numpy as np
import pytest

from oracle.oracle import exact_riemann
from shaderous_b200 import Config, Problem, Sim
from shaderous_b200.amr import AmrConfig, AmrSim

pytestmark = pytest.mark.gpu

BS = 16


def ghost_src_ref(tab, slot, l, ndim):
    """amr/grid.wgsl ghost_src restated over a block table: (kind, slot, l0, l1, l2)."""
    out = [a for a in range(ndim) if l[a] < 0 or l[a] >= BS]
    if not out:
        return (0, slot, *l)
    if len(out) > 1:
        return (2, slot, *l)
    axis = out[0]
    upper = 1 if l[axis] >= BS else 0
    nb = int(tab[slot, 6 + 2 * axis + upper])
    ll = list(l)
    if nb >= 0:
        ll[axis] += -BS if upper else BS
        return (0, nb, *ll)
    if nb == -1:
        return (1, int(tab[slot, 20 + 2 * axis + upper]), *l)
    k = -1 - nb
    if k == 2:
        ll[axis] = 2 * BS - 1 - l[axis] if upper else -1 - l[axis]
    else:
        ll[axis] = BS - 1 if upper else 0
    return (0, slot, *ll)


@pytest.mark.parametrize("ndim", [2, 3])
def test_ghost_indexing_matches_reference_rule(ndim):
    hyd = Config(gamma=5 / 3, bc_lo=(1, 2, 0), bc_hi=(2, 1, 0), recon="mc")
    cfg = AmrConfig(hydro=hyd, ndim=ndim, nr=2, max_level=2, cap=600 if ndim == 3 else 200, refine_hi=0.1,
                    refine_lo=0.05, regrid_every=0)
    with AmrSim(cfg) as a:
        a.reset(Problem("blast", a=(1, 10, 1, 0.1, 0.12)))
        slots, levels, _ = a.leaves()
        assert levels.max() == 2  # refined around the blast
        tab = a.table()
        coarse_faces = 0
        for s in slots:
            gm = a.ghost_map(int(s))
            pad = 20
            for t in range(pad ** ndim):
                l = [t % pad - 2, (t // pad) % pad - 2, (t // (pad * pad)) - 2 if ndim == 3 else 0]
                want = ghost_src_ref(tab, int(s), l, ndim)
                assert tuple(gm[t]) == want, (s, l, tuple(gm[t]), want)
                coarse_faces += want[0] == 1
        assert coarse_faces > 0


@pytest.mark.parametrize("case", ["gauss-periodic", "blast-walls"])
def test_unrefined_blocks_equal_uniform_grid(case):
    n = 64
    if case == "gauss-periodic":
        hyd = Config(n=(n, n, n), gamma=1.4, recon="koren", isentropic=True, cfl=0.5)
        prob = Problem("gauss", a=(1.5, 0.02, 1.0, 0.5, 0.1, 1.0, 0.01))
    else:
        hyd = Config(n=(n, n, n), gamma=5 / 3, bc_lo=(1, 2, 1), bc_hi=(2, 1, 2), recon="mc", isentropic=False, cfl=0.5)
        prob = Problem("blast", a=(1, 10, 1, 0.1, 0.2))
    steps = 12
    with Sim(hyd) as s:
        s.reset(prob)
        s.run(steps=steps)
        u1, u2 = s.read_state()
    cfg = AmrConfig(hydro=hyd, ndim=3, nr=n // BS, max_level=0, cap=(n // BS) ** 3, regrid_every=0)
    with AmrSim(cfg) as a:
        a.reset(prob)
        r = a.run(steps=steps)
        assert r.taken == steps
        g1, g2 = a.uniform_level(0)
    u1 = u1.reshape(n, n, n, 4).astype(np.float64)
    g1 = g1.astype(np.float64)
    rel = np.abs(g1[..., 0] - u1[..., 0]).sum() / np.abs(u1[..., 0]).sum()
    assert rel < 1e-6, rel
    assert np.abs(g1[..., 0] - u1[..., 0]).max() / np.abs(u1[..., 0]).max() < 1e-5
    e_rel = np.abs(g2.astype(np.float64)[..., 0] - u2.reshape(n, n, n, 4)[..., 0]).sum() / np.abs(u2[:, 0]).sum()
    assert e_rel < 1e-6, e_rel


def test_unrefined_2d_equals_uniform():
    n = 128
    hyd = Config(n=(n, n, 1), gamma=1.4, recon="minmod", isentropic=True, cfl=0.4)
    prob = Problem("blast", a=(2, 5, 1, 0.5, 0.15))
    with Sim(hyd) as s:
        s.reset(prob)
        s.run(steps=30)
        u1, _ = s.read_state()
    cfg = AmrConfig(hydro=hyd, ndim=2, nr=n // BS, max_level=0, cap=(n // BS) ** 2, regrid_every=0)
    with AmrSim(cfg) as a:
        a.reset(prob)
        a.run(steps=30)
        g1, _ = a.uniform_level(0)
    rel = np.abs(g1[0, ..., 0].astype(np.float64) - u1[:, 0].reshape(n, n)).sum() / np.abs(u1[:, 0]).sum()
    assert rel < 1e-6, rel


@pytest.mark.parametrize("ndim", [2, 3])
def test_conserves_through_remeshes(ndim):
    hyd = Config(gamma=5 / 3, recon="koren", isentropic=True, cfl=0.5)
    cfg = AmrConfig(hydro=hyd, ndim=ndim, nr=4 if ndim == 2 else 2, max_level=2, cap=1200 if ndim == 3 else 400,
                    refine_hi=0.1, refine_lo=0.05, regrid_every=4)
    with AmrSim(cfg) as a:
        a.reset(Problem("blast", a=(1, 10, 1, 0.1, 0.15)))
        def mesh():
            _, lv, co = a.leaves()
            return frozenset((int(x), *map(int, c)) for x, c in zip(lv, co))

        d0 = a.diagnostics()
        meshes = {mesh()}
        for _ in range(20):
            a.run(steps=10)
            meshes.add(mesh())
        d1 = a.diagnostics()
        assert d1.steps == 200
        assert len(meshes) > 1  # the mesh followed the blast
        _, lv, _ = a.leaves()
        assert lv.max() == 2
    assert abs(d1.mass - d0.mass) / d0.mass < 2e-6
    assert abs(d1.e_tot - d0.e_tot) / d0.e_tot < 2e-6
    assert np.isfinite([d1.mass, d1.e_tot, d1.e_kin]).all()


def test_refined_sod_tube_against_exact():
    hyd = Config(gamma=1.4, bc_lo=(1, 0, 0), bc_hi=(1, 0, 0), recon="mc", isentropic=False, cfl=0.4, p_floor=1e-12)
    cfg = AmrConfig(hydro=hyd, ndim=2, nr=2, max_level=2, cap=200, refine_hi=0.1, refine_lo=0.05, regrid_every=4)
    with AmrSim(cfg) as a:
        a.reset(Problem("sod", a=(1, 0, 1, 0.125, 0, 0.1)))
        r = a.run(until=0.1)
        assert r.stopped == "time" and r.t == pytest.approx(0.1, abs=1e-12)
        slots, lv, co = a.leaves()
        u1, _ = a.leaves_state()
        assert lv.max() == 2
    # integrate |rho - exact| over the domain from each leaf's cells
    err = 0.0
    for i in range(len(slots)):
        dx = 1.0 / (2 * BS << lv[i])
        x = (co[i, 0] * BS + np.arange(BS) + 0.5) * dx - 0.5
        ex = exact_riemann((1, 0, 1), (0.125, 0, 0.1), 1.4, x / 0.1)[:, 0]
        rho = u1[i, :, 0].reshape(BS, BS).astype(np.float64)
        err += (np.abs(rho - ex[None, :]).sum()) * dx * dx
    assert err < 0.006, err


def test_sedov_3d_refines_and_conserves():
    hyd = Config(gamma=5 / 3, bc_lo=(1, 1, 1), bc_hi=(1, 1, 1), recon="koren", isentropic=True, cfl=0.5, p_floor=1e-12)
    cfg = AmrConfig(hydro=hyd, ndim=3, nr=2, max_level=3, cap=2500, refine_hi=0.1, refine_lo=0.05, regrid_every=8)
    with AmrSim(cfg) as a:
        a.reset(Problem("sedov", a=(1, 1e-5, 1, 3.5)))
        _, lv, _ = a.leaves()
        assert lv.max() == 3
        d0 = a.diagnostics()
        a.run(steps=40)
        d1 = a.diagnostics()
        _, lv1, _ = a.leaves()
        assert lv1.max() == 3
    assert abs(d1.e_tot - d0.e_tot) / d0.e_tot < 1e-5
    assert abs(d1.mass - d0.mass) / d0.mass < 1e-6
    assert d1.max_mach > 0.5  # a blast wave moving at about the sound speed of the shocked gas


@pytest.mark.parametrize("ndim,recon,isen,bcs", [
    (2, "mc", False, ((2, 1, 0), (1, 0, 0))),
    (2, "koren", True, ((0, 0, 0), (0, 0, 0))),
    (3, "minmod", False, ((2, 0, 1), (1, 2, 0))),
    (3, "koren", True, ((1, 1, 1), (2, 2, 2))),
])
def test_fused_sweep_equals_two_passes(ndim, recon, isen, bcs):
    """The fused block sweep (predict, fluxes and update from the primitives in one pass) against
    the reference's pass structure (a half-step atlas, then the update) on the same refined mesh:
    walls, outflow and periodic faces, coarse-fine faces with fine-flux matching. Both read every
    primitive from the same atlas and do the same arithmetic, so with minmod and MC they agree bit
    for bit; Koren with the isentropic increments (powf) is compiled into two different kernels,
    whose contraction of multiply-adds may differ: a few ulps a step."""
    hyd = Config(gamma=5 / 3, bc_lo=bcs[0], bc_hi=bcs[1], recon=recon, isentropic=isen, cfl=0.4, p_floor=1e-12)
    runs = []
    for two in (False, True):
        cfg = AmrConfig(hydro=hyd, ndim=ndim, nr=2, max_level=2, cap=1200 if ndim == 3 else 200, refine_hi=0.1,
                        refine_lo=0.05, regrid_every=0, two_pass=two)
        with AmrSim(cfg) as a:
            a.reset(Problem("blast", a=(1, 10, 1, 0.1, 0.2)))
            _, lv, _ = a.leaves()
            assert lv.max() == 2 and lv.min() < 2  # coarse-fine faces present
            a.run(steps=20)
            runs.append((a.leaves(), a.leaves_state(), a.diagnostics()))
    ((_, l0, c0), (u0, v0), d0), ((_, l1, c1), (u1, v1), d1) = runs
    assert (l0 == l1).all() and (c0 == c1).all()
    if recon in ("minmod", "mc"):
        assert np.array_equal(u0, u1) and np.array_equal(v0, v1)
    for x, y in ((u0, u1), (v0, v1)):
        x = x.astype(np.float64)
        y = y.astype(np.float64)
        for comp in range(4):
            scale = np.abs(x[..., comp]).sum() + np.abs(x[..., 0]).sum() * 1e-3
            assert np.abs(x[..., comp] - y[..., comp]).sum() / scale < 2e-5, comp
    assert d0.steps == d1.steps == 20
    assert d0.t == pytest.approx(d1.t, rel=1e-5)


@pytest.mark.parametrize("two_pass", [False, True])
def test_folded_checks_equal_explicit_checks(two_pass):
    """The refinement check folded into the next step (its flags from that step's own assemble, the
    step launched ahead of the host's decision and taken again on a new mesh) gives the same meshes
    and states, bit for bit, as an explicit check after every 8th step."""
    hyd = Config(gamma=5 / 3, bc_lo=(1, 1, 1), bc_hi=(1, 1, 1), recon="koren", cfl=0.5, p_floor=1e-12)
    out = []
    for folded in (True, False):
        cfg = AmrConfig(hydro=hyd, ndim=2, nr=4, max_level=2, cap=400, refine_hi=0.1, refine_lo=0.05,
                        regrid_every=8 if folded else 0, two_pass=two_pass)
        with AmrSim(cfg) as a:
            a.reset(Problem("blast", a=(1, 10, 1, 0.1, 0.15)))
            meshes = []
            for _ in range(12):
                if folded:
                    a.step(8)
                else:
                    a.step(8)
                    a.regrid()
                _, lv, co = a.leaves()
                meshes.append(sorted((int(x), *map(int, c)) for x, c in zip(lv, co)))
            a.step(1)  # the folded run's due check happens here
            _, lv, co = a.leaves()
            meshes.append(sorted((int(x), *map(int, c)) for x, c in zip(lv, co)))
            out.append((meshes, a.leaves_state(), a.clock()))
    (ma, (a1, a2), ca), (mb, (b1, b2), cb) = out
    assert len(set(map(tuple, map(tuple, ma)))) > 1  # the mesh changed along the way
    # the explicit check lands one step earlier than the folded one; after the next step both agree
    assert ma[-1] == mb[-1] and ca == cb
    assert np.array_equal(a1, b1) and np.array_equal(a2, b2)
