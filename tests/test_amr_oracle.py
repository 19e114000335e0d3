"""The block-grid oracle (oracle/amr_ref.cpp) pinned on the CPU before it checks the GPU.

- On a mesh with no refinement its step is the uniform-grid oracle's step (oracle/ref_hydro.cpp,
  itself pinned to the reference's own tests/unit/reference.test.ts), to float64 rounding, for
  periodic, outflow and reflecting faces, 2D and 3D: the block machinery (ghost sources, images,
  predictions at the source) adds nothing of its own.
- On refined periodic meshes the fine-flux matching conserves mass, momentum and energy to
  float64 rounding (the property amr/update.wgsl:1-8 states for it).
- Prolonged ghosts average to their coarse cell, and a regrid (prolongation with the kinetic
  energy kept consistent, restriction, copy; amr/regrid.wgsl) conserves the totals.
"""
import math

import numpy as np
import pytest

from oracle.amr import AmrOracle
from oracle.oracle import RefHydro
from shaderous_b200.tree import BlockTree

BS = 16


def leaf_cells(tab, slot, nr, box, ndim):
    """Cell-centre coordinates (CB, 3) of block `slot`, box centred on 0, x fastest."""
    lv = int(tab[slot, 0])
    dx = box / (nr * BS * 2 ** lv)
    c = tab[slot, 1:4]
    i = np.arange(BS)
    if ndim == 3:
        z, y, x = np.meshgrid(i, i, i, indexing="ij")
    else:
        y, x = np.meshgrid(i, i, indexing="ij")
        z = np.zeros_like(x)
    pos = np.stack([(c[0] * BS + x + 0.5) * dx, (c[1] * BS + y + 0.5) * dx,
                    (c[2] * BS + z + 0.5) * dx if ndim == 3 else 0 * x], axis=-1).reshape(-1, 3)
    return pos - (box / 2) * np.array([1, 1, 1 if ndim == 3 else 0])


def smooth_prims(pos):
    """A smooth field with structure on every axis: (rho, vx, vy, vz, p, s)."""
    x, y, z = pos[:, 0], pos[:, 1], pos[:, 2]
    two_pi = 2 * math.pi
    rho = 1.0 + 0.3 * np.sin(two_pi * x) * np.cos(two_pi * y) + 0.1 * np.cos(two_pi * z)
    vx = 0.2 * np.sin(two_pi * y) + 0.05
    vy = -0.15 * np.cos(two_pi * x) * np.sin(two_pi * z)
    vz = 0.1 * np.sin(two_pi * (x + y))
    p = 1.0 + 0.2 * np.cos(two_pi * (x - z))
    s = (x > 0).astype(float)
    return np.stack([rho, vx, vy, vz, p, s], axis=1)


def blast_prims(pos, r=0.15):
    rr = np.sqrt((pos ** 2).sum(axis=1))
    w = np.zeros((len(pos), 6))
    w[:, 0] = 1.0
    w[:, 4] = np.where(rr < r, 10.0, 0.1)
    w[:, 5] = (rr < r).astype(float)
    return w


def to_state(w, gamma):
    """Primitives -> float32 (u1, u2) as the reference's init does (hydro.ts:195-214)."""
    rho = w[:, 0]
    eint = w[:, 4] / (gamma - 1)
    u1 = np.stack([rho, rho * w[:, 1], rho * w[:, 2], rho * w[:, 3]], axis=1)
    u2 = np.stack([eint + 0.5 * rho * (w[:, 1:4] ** 2).sum(axis=1), eint, rho * w[:, 5], 0 * rho], axis=1)
    return u1.astype(np.float32), u2.astype(np.float32)


def mesh(ndim, nr, bc_lo, bc_hi, refine=(), max_level=2, cap=None):
    cap = cap or (400 if ndim == 3 else 200)
    t = BlockTree(ndim, nr, max_level, cap, bc_lo, bc_hi)
    for level, c in refine:
        t.refine(level, c)
    return t


def fill(o, tab, leaves, nr, box, ndim, gamma, field):
    u1s, u2s = [], []
    for s in leaves:
        u1, u2 = to_state(field(leaf_cells(tab, int(s), nr, box, ndim)), gamma)
        u1s.append(u1)
        u2s.append(u2)
    u1, u2 = np.stack(u1s), np.stack(u2s)
    o.set_state(leaves, u1, u2)
    return u1, u2


def totals(o, tab, leaves, nr, box, ndim):
    st = o.state(leaves)
    out = np.zeros(7)
    for i, s in enumerate(leaves):
        dv = (box / (nr * BS * 2 ** int(tab[s, 0]))) ** ndim
        out += st[i][:, [0, 1, 2, 3, 4, 5, 6]].sum(axis=0) * dv
    return out


@pytest.mark.parametrize("ndim,bc,recon,isen", [
    (2, "periodic", "mc", False),
    (2, "walls", "koren", True),
    (3, "periodic", "minmod", False),
    (3, "walls", "vanleer", True),
])
def test_unrefined_block_step_equals_uniform_oracle(ndim, bc, recon, isen):
    nr, box, gamma = 2, 1.0, 1.4
    if bc == "periodic":
        bc_lo, bc_hi = (0, 0, 0), (0, 0, 0)
    else:
        bc_lo, bc_hi = (1, 2, 1), (2, 1, 2)
    t = mesh(ndim, nr, bc_lo, bc_hi, max_level=0, cap=64)
    tab = t.table()
    all_blocks, leaves, _ = t.lists()
    n = nr * BS
    dx0 = box / n
    o = AmrOracle(ndim, nr, t.cap, dx0, gamma, recon=recon, isentropic=isen)
    o.set_table(tab)
    field = smooth_prims if bc == "periodic" else blast_prims
    u1, u2 = fill(o, tab, leaves, nr, box, ndim, gamma, field)
    # the same state as one uniform grid, x fastest
    shape = (n, n, n) if ndim == 3 else (1, n, n)
    g1 = np.zeros(shape + (4,), np.float32)
    g2 = np.zeros(shape + (4,), np.float32)
    for i, s in enumerate(leaves):
        c = tab[s, 1:4] * BS
        if ndim == 3:
            g1[c[2]:c[2] + BS, c[1]:c[1] + BS, c[0]:c[0] + BS] = u1[i].reshape(BS, BS, BS, 4)
            g2[c[2]:c[2] + BS, c[1]:c[1] + BS, c[0]:c[0] + BS] = u2[i].reshape(BS, BS, BS, 4)
        else:
            g1[0, c[1]:c[1] + BS, c[0]:c[0] + BS] = u1[i].reshape(BS, BS, 4)
            g2[0, c[1]:c[1] + BS, c[0]:c[0] + BS] = u2[i].reshape(BS, BS, 4)
    ref = RefHydro(n=(n, n, n if ndim == 3 else 1), dx=dx0, gamma=gamma,
                   bc_lo=bc_lo if ndim == 3 else (bc_lo[0], bc_lo[1], 0),
                   bc_hi=bc_hi if ndim == 3 else (bc_hi[0], bc_hi[1], 0),
                   cfl=0.4, limiter=recon, isentropic=isen, threads=4)
    ref.set_state32(g1.reshape(-1, 4), g2.reshape(-1, 4))
    for _ in range(3):
        rate = o.assemble(all_blocks)
        dt = 0.4 / rate
        ref.step()
        assert abs(ref.dt - dt) <= 1e-13 * dt, (ref.dt, dt)
        o.step(leaves, dt)
    st = o.state(leaves)
    U = ref.U  # (7, ncell)
    for i, s in enumerate(leaves):
        c = tab[s, 1:4] * BS
        if ndim == 3:
            idx = ((np.arange(BS)[:, None, None] + c[2]) * n + (np.arange(BS)[None, :, None] + c[1])) * n \
                + (np.arange(BS)[None, None, :] + c[0])
        else:
            idx = (np.arange(BS)[:, None] + c[1]) * n + (np.arange(BS)[None, :] + c[0])
        want = U[:, idx.reshape(-1)].T  # (CB, 7)
        got = st[i][:, :7]
        np.testing.assert_allclose(got, want, rtol=1e-11, atol=1e-12, err_msg=f"block {s}")


# (root blocks per side, refinements): meshes that keep coarse leaves beside refined ones
REFINED = {
    2: (4, [(0, (0, 0, 0)), (0, (2, 2, 0)), (1, (1, 1, 0))]),
    3: (2, [(0, (0, 0, 0)), (0, (1, 1, 1))]),
}


@pytest.mark.parametrize("ndim", [2, 3])
def test_refined_periodic_step_conserves(ndim):
    nr, refine = REFINED[ndim]
    box, gamma = 1.0, 5 / 3
    t = mesh(ndim, nr, (0, 0, 0), (0, 0, 0), refine=refine)
    tab = t.table()
    all_blocks, leaves, _ = t.lists()
    assert (tab[leaves, 0] > 0).any() and (tab[leaves, 0] == 0).any()
    dx0 = box / (nr * BS)
    o = AmrOracle(ndim, nr, t.cap, dx0, gamma, recon="mc")
    o.set_table(tab)
    fill(o, tab, leaves, nr, box, ndim, gamma, smooth_prims)
    before = totals(o, tab, leaves, nr, box, ndim)
    for _ in range(3):
        rate = o.assemble(all_blocks)
        o.step(leaves, 0.4 / rate)
    after = totals(o, tab, leaves, nr, box, ndim)
    scale = np.array([before[0], before[0], before[0], before[0], before[4], before[5], before[0]])
    np.testing.assert_allclose(after[[0, 1, 2, 3, 4, 6]], before[[0, 1, 2, 3, 4, 6]],
                               rtol=0, atol=1e-13 * scale[[0, 1, 2, 3, 4, 6]].max())


@pytest.mark.parametrize("ndim", [2, 3])
def test_prolonged_ghosts_average_to_their_coarse_cell(ndim):
    nr, box, gamma = 2, 1.0, 1.4
    t = mesh(ndim, nr, (1, 1, 1), (1, 1, 1), refine=[(0, (0, 0, 0))])
    tab = t.table()
    all_blocks, leaves, _ = t.lists()
    dx0 = box / (nr * BS)
    o = AmrOracle(ndim, nr, t.cap, dx0, gamma, recon="mc")
    o.set_table(tab)
    fill(o, tab, leaves, nr, box, ndim, gamma, smooth_prims)
    o.assemble(all_blocks)
    pad = BS + 4
    checked = 0
    for s in leaves:
        w = o.prims(int(s)).reshape((pad,) * ndim + (7,))
        for f in range(2 * ndim):
            if tab[s, 6 + f] != -1:
                continue
            axis, upper = f // 2, f % 2
            cs = int(tab[s, 20 + f])
            st = o.state([cs])[0].reshape((BS,) * ndim + (8,))
            groups = {}
            rng = [range(BS)] * 3
            rng[axis] = range(BS, BS + 2) if upper else range(-2, 0)
            if ndim == 2:
                rng[2] = [0]
            for z in rng[2]:
                for y in rng[1]:
                    for x in rng[0]:
                        tex = w[z + 2, y + 2, x + 2] if ndim == 3 else w[y + 2, x + 2]
                        gf = tab[s, 1:4] * BS + np.array([x, y, z])
                        key = tuple(((gf >> 1) - tab[cs, 1:4] * BS)[:ndim])
                        groups.setdefault(key, []).append((tex[0], tex[0] * tex[1], tex[0] * tex[2]))
            for key, vals in groups.items():
                v = np.array(vals)
                assert len(v) == 2 ** ndim
                coarse = st[key[::-1]]
                np.testing.assert_allclose(v[:, 0].mean(), coarse[0], rtol=1e-13)
                np.testing.assert_allclose(v[:, 1].mean(), coarse[1], rtol=1e-12, atol=1e-13)
                np.testing.assert_allclose(v[:, 2].mean(), coarse[2], rtol=1e-12, atol=1e-13)
                checked += 1
    assert checked > 0


@pytest.mark.parametrize("ndim", [2, 3])
def test_regrid_conserves_totals(ndim):
    nr, refine = REFINED[ndim]
    box, gamma = 1.0, 5 / 3
    t = mesh(ndim, nr, (0, 0, 0), (0, 0, 0), refine=refine)
    tab = t.table()
    all_blocks, leaves, _ = t.lists()
    dx0 = box / (nr * BS)
    o = AmrOracle(ndim, nr, t.cap, dx0, gamma, recon="koren")
    o.set_table(tab)
    fill(o, tab, leaves, nr, box, ndim, gamma, smooth_prims)
    before = totals(o, tab, leaves, nr, box, ndim)
    o.assemble(all_blocks)
    # refine every coarse leaf's first block and merge what can be merged
    ind = np.zeros(t.cap)
    for s in leaves:
        ind[s] = 1.0 if tab[s, 0] == 0 and (tab[s, 1:4] == 0).all() else 0.0
    ind[leaves[tab[leaves, 0] == 0][:1]] = 1.0
    rg = t.adapt(ind, 0.5, 0.25)
    assert rg is not None
    new_tab = t.table()
    _, new_leaves, _ = t.lists()
    kinds = set(rg[new_leaves, 0].tolist())
    assert 2 in kinds  # something was prolonged
    o.regrid(new_tab, rg, new_leaves)
    after = totals(o, new_tab, new_leaves, nr, box, ndim)
    for i in (0, 1, 2, 3, 4, 6):
        assert abs(after[i] - before[i]) <= 1e-13 * max(abs(before[0]), abs(before[4])), (i, after[i], before[i])
