"""A grid split into z-slabs (SHZ_BC_HALO faces) steps exactly as the whole grid.

One GPU only: (1) the NCCL-driven SlabSim at world size 1 (a periodic grid whose one slab
exchanges with itself); (2) two slab handles in one process, their halos and rate maxima
exchanged by host-ordered device copies between steps (no kernel waits on another), for a walled
grid and a periodic one. Both must equal the single grid bit for bit: a slab reads its stored
ghost planes as the single grid reads its neighbouring planes."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist

from shaderous_b200 import Config, Problem, Sim
from shaderous_b200.dist import HALO, SlabSim, _view

pytestmark = pytest.mark.gpu


def _port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_slabsim_world1_periodic_equals_grid():
    cfg = Config(n=(32, 32, 48), dx=2 * np.pi / 32, gamma=5 / 3, recon="ppm", cfl=0.4)
    prob = Problem("tgv", a=(1.0, 100.0, 1.0))
    with Sim(cfg) as s:
        s.reset(prob)
        s.run(steps=8)
        ref = s.read_state()
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(_port())
    torch.cuda.set_device(0)
    dist.init_process_group("nccl", rank=0, world_size=1, device_id=torch.device("cuda", 0))
    try:
        with SlabSim(cfg) as sl:
            assert sl.halo == (True, True) and sl.prev == 0 and sl.next == 0
            sl.reset(prob)
            sl.step(8)
            sl.sync()
            got = sl.read_state()
            d = sl.diagnostics()
    finally:
        dist.destroy_process_group()
    assert np.array_equal(got[0], ref[0]) and np.array_equal(got[1], ref[1])
    assert d.steps == 8


def _two_slabs(cfg: Config, prob: Problem, steps: int, split: int):
    """The grid as two slab handles [0, split) and [split, nz), stepped with host-ordered
    exchanges; returns the joined state."""
    nz = cfg.n[2]
    periodic = cfg.bc_lo[2] == 0
    lo0 = HALO if periodic else cfg.bc_lo[2]
    hi1 = HALO if periodic else cfg.bc_hi[2]
    c0 = Config(**{**cfg.__dict__, "n": (cfg.n[0], cfg.n[1], split), "bc_lo": (*cfg.bc_lo[:2], lo0),
                   "bc_hi": (*cfg.bc_hi[:2], HALO)})
    c1 = Config(**{**cfg.__dict__, "n": (cfg.n[0], cfg.n[1], nz - split), "bc_lo": (*cfg.bc_lo[:2], HALO),
                   "bc_hi": (*cfg.bc_hi[:2], hi1)})
    dev = torch.device("cuda", 0)
    with Sim(c0) as a, Sim(c1) as b:
        a.reset_slab(cfg, prob, 0)
        b.reset_slab(cfg, prob, split)
        assert a.halo_depth() == b.halo_depth() == (3 if cfg.recon == "ppm" else 2)

        def face(sim, side):
            i1, i2, g1, g2, nb = sim.halo_device(side)
            return [_view(p, nb, device=dev) for p in (i1, i2, g1, g2)]

        for _ in range(steps):
            a.sync()
            b.sync()
            a_hi, b_lo = face(a, 1), face(b, 0)
            a_hi[2].copy_(b_lo[0])  # a's upper ghosts: b's lowest planes
            a_hi[3].copy_(b_lo[1])
            b_lo[2].copy_(a_hi[0])  # b's lower ghosts: a's highest planes
            b_lo[3].copy_(a_hi[1])
            if periodic:
                a_lo, b_hi = face(a, 0), face(b, 1)
                a_lo[2].copy_(b_hi[0])
                a_lo[3].copy_(b_hi[1])
                b_hi[2].copy_(a_lo[0])
                b_hi[3].copy_(a_lo[1])
            ra = _view(a.rate_device(), 4, torch.int32, dev)
            rb = _view(b.rate_device(), 4, torch.int32, dev)
            m = torch.maximum(ra, rb)
            ra.copy_(m)
            rb.copy_(m)
            torch.cuda.synchronize()
            a.step(1)
            b.step(1)
        a.sync()
        b.sync()
        sa, sb = a.read_state(), b.read_state()
    return np.concatenate([sa[0], sb[0]]), np.concatenate([sa[1], sb[1]])


@pytest.mark.parametrize("recon,bcs,prob", [
    ("ppm", ((0, 0, 0), (0, 0, 0)), Problem("tgv", a=(1.0, 100.0, 1.0))),
    ("koren", ((1, 2, 2), (1, 1, 1)), Problem("blast", a=(1.0, 10.0, 1.0, 0.1, 0.25))),
    ("mc", ((0, 0, 1), (0, 0, 2)), Problem("sod", a=(1, 0, 1, 0.125, 0, 0.1), axis=2)),
])
def test_two_slabs_equal_grid(recon, bcs, prob):
    n = 32
    cfg = Config(n=(n, n, 40), dx=(2 * np.pi / n) if prob.kind == "tgv" else 1.0 / n, gamma=1.4, recon=recon,
                 cfl=0.4, bc_lo=bcs[0], bc_hi=bcs[1], p_floor=1e-12)
    with Sim(cfg) as s:
        s.reset(prob)
        s.run(steps=10)
        ref = s.read_state()
    got = _two_slabs(cfg, prob, 10, split=17)
    assert np.array_equal(got[0], ref[0]) and np.array_equal(got[1], ref[1])
