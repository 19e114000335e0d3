"""The refined-mesh block step on the GPU against the float64 block-grid oracle (oracle/amr_ref.cpp,
pinned on the CPU by tests/test_amr_oracle.py), from the same float32 state on the same block table:

- assemble: every texel of every leaf's primitive region, own cells and ghosts (same-level,
  restricted from refined neighbours, prolonged beyond coarser faces, boundary images, edges and
  corners): relative L-inf per variable <= 1e-6 (amr/assemble.wgsl:78-154, amr/cons.wgsl:19-125);
- the step's dt from the leaves' rates: relative 1e-6;
- one step, and several, of the block sweep (fused, and the reference's two passes): relative L1
  per conserved variable <= 1e-5 against the oracle's predict and update with fine-flux matching
  (amr/predict.wgsl:184-221, amr/update.wgsl:207-560), L-inf <= 1e-4;
- the Löhner indicators (amr/flag.wgsl:66-155) within float32 rounding (2e-5 relative plus 1e-6),
  and the
  block tree's decisions from the oracle's indicators equal the ones the GPU run made;
- the regrid fill of the new leaves (amr/regrid.wgsl:41-139): relative L-inf per variable <= 1e-6.
Meshes: 2D and 3D, levels 0-2, with reflecting, outflow and periodic faces.
"""
import numpy as np
import pytest

from oracle.amr import AmrOracle
from shaderous_b200 import Config, Problem
from shaderous_b200.amr import AmrConfig, AmrSim
from shaderous_b200.tree import BlockTree

pytestmark = pytest.mark.gpu

BS = 16
CASES = [
    # (ndim, bc_lo, bc_hi, recon, isentropic, two_pass)
    (2, (2, 1, 0), (1, 2, 0), "mc", False, False),
    (2, (0, 0, 0), (0, 0, 0), "koren", True, True),
    (3, (2, 1, 0), (1, 0, 2), "mc", False, False),
    (3, (0, 2, 1), (0, 2, 1), "minmod", True, True),
]
IDS = ["2d-walls-mc-fused", "2d-periodic-koren-twopass", "3d-mixed-mc-fused", "3d-mixed-minmod-twopass"]


def make(ndim, bc_lo, bc_hi, recon, isen, two_pass):
    hyd = Config(gamma=5 / 3, bc_lo=bc_lo, bc_hi=bc_hi, recon=recon, isentropic=isen, cfl=0.4)
    cfg = AmrConfig(hydro=hyd, ndim=ndim, nr=2, max_level=2, cap=900 if ndim == 3 else 300, refine_hi=0.1,
                    refine_lo=0.05, regrid_every=0, two_pass=two_pass)
    a = AmrSim(cfg)
    a.reset(Problem("blast", a=(1, 10, 1, 0.1, 0.18)))
    return cfg, a


def oracle_for(cfg, tab, recon, isen):
    h = cfg.hydro
    dx0 = cfg.box / (cfg.nr * BS)
    o = AmrOracle(cfg.ndim, cfg.nr, cfg.cap, dx0, h.gamma, recon=recon, isentropic=isen, rho_floor=h.rho_floor,
                  p_floor=h.p_floor, eta_dual=h.eta_dual, shock_thresh=h.shock_thresh, threads=8)
    o.set_table(tab)
    return o


def active_blocks(tab):
    """Every block of the table (leaves and parents), coarsest first."""
    act = np.nonzero(tab[:, 4] & 1)[0]
    return act[np.argsort(tab[act, 0], kind="stable")].astype(np.int32)


def rel_l1(got, want):
    return np.abs(got - want).sum() / max(np.abs(want).sum(), 1e-300)


def check_state(got1, got2, want, l1, linf, tag):
    """got (float32 u1, u2 per leaf) against the oracle's float64 (leaves, cells, 8)."""
    g = np.concatenate([got1, got2], axis=2).astype(np.float64)
    names = ["rho", "mx", "my", "mz", "E", "eint", "rho_s"]
    mom = np.sqrt((want[..., 1:4] ** 2).sum(axis=-1))
    for v, name in enumerate(names):
        if name == "mz" and g.shape[1] == BS * BS:
            continue
        if name == "rho_s" and np.abs(want[..., v]).max() == 0:
            continue
        den = np.abs(mom).sum() if name in ("mx", "my", "mz") else np.abs(want[..., v]).sum()
        e1 = np.abs(g[..., v] - want[..., v]).sum() / den
        scale = np.abs(mom).max() if name in ("mx", "my", "mz") else np.abs(want[..., v]).max()
        einf = np.abs(g[..., v] - want[..., v]).max() / scale
        assert e1 <= l1 and einf <= linf, f"{tag} {name}: rel L1 {e1:.3e}, rel L-inf {einf:.3e}"


@pytest.mark.parametrize("case", CASES, ids=IDS)
def test_assemble_and_steps_match_oracle(case):
    ndim, bc_lo, bc_hi, recon, isen, two_pass = case
    cfg, a = make(*case)
    with a:
        slots, levels, _ = a.leaves()
        assert levels.max() == 2 and levels.min() < 2
        tab = a.table()
        u1, u2 = a.leaves_state()
        o = oracle_for(cfg, tab, recon, isen)
        o.set_state(slots, u1, u2)

        # one step: its assemble's primitives, its dt, its new state
        a.step(1)
        _, dt_gpu, _ = a.clock()
        rate = o.assemble(active_blocks(tab))
        dt_o = cfg.hydro.cfl / rate
        assert abs(dt_gpu - dt_o) <= 1e-6 * dt_o, (dt_gpu, dt_o)
        kinds = {"plain": 0, "coarse": 0}
        for s in slots:
            g = a.prims(int(s)).astype(np.float64)[:, :7]
            w = o.prims(int(s))
            assert np.isfinite(w).all(), f"oracle left texels of block {s} unresolved"
            gm = a.ghost_map(int(s))
            kinds["coarse"] += int((gm[:, 0] == 1).sum())
            kinds["plain"] += int((gm[:, 0] == 0).sum())
            for v in range(7):
                scale = np.abs(w[:, 1:4]).max() if v in (1, 2, 3) else np.abs(w[:, v]).max()
                if scale == 0:
                    assert np.abs(g[:, v]).max() == 0
                    continue
                err = np.abs(g[:, v] - w[:, v]).max() / scale
                assert err <= 1e-6, f"block {s} variable {v}: rel L-inf {err:.3e}"
        assert kinds["coarse"] > 0  # prolonged ghosts were compared
        o.step(slots, dt_gpu)
        g1, g2 = a.leaves_state()
        check_state(g1, g2, o.state(slots), 1e-5, 1e-4, "step 1")

        # several more steps, each side with its own dt
        n = 6 if ndim == 3 else 12
        a.step(n)
        for _ in range(n):
            rate = o.assemble(active_blocks(tab))
            o.step(slots, cfg.hydro.cfl / rate)
        g1, g2 = a.leaves_state()
        check_state(g1, g2, o.state(slots), 1e-5, 1e-4, f"step {n + 1}")


def leaf_positions(cfg, level, c):
    """Cell centres (CB, 3) of the leaf at `level`, block coordinates c; box centred on 0."""
    dx = cfg.box / (cfg.nr * BS * 2 ** level)
    i = np.arange(BS)
    if cfg.ndim == 3:
        z, y, x = np.meshgrid(i, i, i, indexing="ij")
    else:
        y, x = np.meshgrid(i, i, indexing="ij")
        z = np.zeros_like(x)
    pos = np.stack([(c[0] * BS + x + 0.5) * dx, (c[1] * BS + y + 0.5) * dx,
                    (c[2] * BS + z + 0.5) * dx if cfg.ndim == 3 else 0.0 * x], axis=-1).reshape(-1, 3)
    return pos - cfg.box / 2 * np.array([1, 1, 1 if cfg.ndim == 3 else 0])


def tree_like(cfg, tab):
    """A host block tree with the same leaves as `tab` (the same parents split, coarsest first)."""
    t = BlockTree(cfg.ndim, cfg.nr, cfg.max_level, cfg.cap, cfg.hydro.bc_lo, cfg.hydro.bc_hi)
    act = active_blocks(tab)
    for s in act:
        if tab[s, 4] & 2:
            continue
        lv, c = int(tab[s, 0]), tuple(int(x) for x in tab[s, 1:4])
        if any(b[1] == lv and b[2] == c for b in t.leaves()):
            t.refine(lv, c)
    return t


def leaf_set(tab):
    act = active_blocks(tab)
    return sorted((int(tab[s, 0]), *map(int, tab[s, 1:4])) for s in act if tab[s, 4] & 2)


@pytest.mark.parametrize("case", CASES, ids=IDS)
def test_flags_decisions_and_regrid_match_oracle(case):
    ndim, bc_lo, bc_hi, recon, isen, two_pass = case
    cfg, a = make(*case)
    with a:
        # a new state on the blast's mesh: a density jump off the centre, so that leaves at the
        # jump refine and the refined blocks about the centre merge
        slots, levels, coords = a.leaves()
        u1s, u2s = [], []
        for lv, c in zip(levels, coords):
            x = leaf_positions(cfg, int(lv), c)
            w = np.zeros((len(x), 6))
            w[:, 0] = 1.0 + 2.0 * (x[:, 0] > 0.2) + 0.05 * np.sin(6.0 * x[:, 1])
            w[:, 1] = 0.1
            w[:, 4] = 1.0
            w[:, 5] = (x[:, 0] > 0.2).astype(float)
            e = w[:, 4] / (cfg.hydro.gamma - 1)
            r = w[:, 0]
            u1s.append(np.stack([r, r * w[:, 1], 0 * r, 0 * r], axis=1))
            u2s.append(np.stack([e + 0.5 * r * w[:, 1] ** 2, e, r * w[:, 5], 0 * r], axis=1))
        a.set_leaves_state(np.stack(u1s).astype(np.float32), np.stack(u2s).astype(np.float32))
        a.step(2)
        slots, _, _ = a.leaves()
        tab = a.table()
        u1, u2 = a.leaves_state()
        changed = a.regrid()
        assert changed
        flags = a.flags()
        new_tab = a.table()
        new_slots, _, _ = a.leaves()
        rg = a.regrid_table()
        n1, n2 = a.leaves_state()

        o = oracle_for(cfg, tab, recon, isen)
        o.set_state(slots, u1, u2)
        o.assemble(active_blocks(tab))
        ind = o.flags(slots)
        got = flags[slots].astype(np.float64)
        # (the indicator is dimensionless, about 1 at a jump; in smooth gas it is a small
        # difference of float32 values, so the bound has an absolute part far below the
        # thresholds the decisions use)
        err = np.abs(got - ind) - 2e-5 * ind
        assert err.max() <= 1e-6, (err.max(), slots[err.argmax()], got[err.argmax()], ind[err.argmax()])
        # no indicator so close to a threshold that float32 rounding could tip it
        for thr in (cfg.refine_hi, cfg.refine_lo):
            assert (np.abs(ind - thr) > 1e-4 * thr).all()

        # the tree's decisions from the oracle's indicators: the GPU run's new mesh
        t = tree_like(cfg, tab)
        assert leaf_set(t.table()) == leaf_set(tab)
        host_tab = t.table()
        by_pos = {(int(tab[s, 0]), *map(int, tab[s, 1:4])): v for s, v in zip(slots, ind)}
        ind_host = np.zeros(cfg.cap)
        for s in active_blocks(host_tab):
            key = (int(host_tab[s, 0]), *map(int, host_tab[s, 1:4]))
            if key in by_pos:
                ind_host[s] = by_pos[key]
        assert t.adapt(ind_host, cfg.refine_hi, cfg.refine_lo) is not None
        assert leaf_set(t.table()) == leaf_set(new_tab)

        # the new leaves' state
        o.regrid(new_tab, rg, new_slots)
        want = o.state(new_slots)
        g = np.concatenate([n1, n2], axis=2).astype(np.float64)
        kinds = rg[new_slots, 0]
        assert (kinds == 2).any() and (kinds == 1).any()
        for v in range(7):
            scale = np.abs(want[..., 1:4]).max() if v in (1, 2, 3) else np.abs(want[..., v]).max()
            if scale == 0 or (ndim == 2 and v == 3):
                continue
            e = np.abs(g[..., v] - want[..., v]).max() / scale
            assert e <= 1e-6, f"regrid variable {v}: rel L-inf {e:.3e}"
