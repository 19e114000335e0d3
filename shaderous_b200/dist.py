"""One uniform grid split into z-slabs, one rank (one GPU) each.

The reference runs a grid on one GPU (docs/architecture.md:695-700); this is the sharded form of
the same step. Each rank's handle holds its slab with SHZ_BC_HALO faces where it meets another
slab (include/shaderous_b200.h): the ghost planes beyond those faces are stored on the device.
Before every step, on the handle's own stream:

1. halo exchange: each halo face's inner planes go to the neighbouring slab's ghost planes of the
   facing side (NCCL send/recv between GPUs; a device copy when a periodic grid has one slab);
2. the rate word becomes its maximum over all slabs (all-reduce, max), so every slab takes the
   same dt;
3. the library's step (clock + fused sweep).

A slab's step reads its ghost planes as the single grid reads its neighbouring planes, so the
split grid's state equals the single grid's bit for bit. The exchange moves 2 x depth x nx x ny
x 32 bytes per slab per step (depth 3 with PPM): 50 MB at 512^2, against a step of ~20 ms.

torch.distributed is the transport (NCCL on GPUs, gloo for the CPU tests of this module's
logic); the arithmetic stays in the library.
"""
from __future__ import annotations

import math
from dataclasses import replace

import torch
import torch.distributed as dist

from .sim import Config, Diagnostics, Problem, Sim

HALO = 3  # SHZ_BC_HALO


def slab_bounds(nz: int, world: int, rank: int) -> tuple[int, int]:
    """Planes [k0, k1) of rank `rank`: nz split as evenly as possible, lower ranks first."""
    base, extra = divmod(nz, world)
    k0 = rank * base + min(rank, extra)
    return k0, k0 + base + (1 if rank < extra else 0)


def slab_faces(bc_lo: int, bc_hi: int, rank: int, world: int) -> tuple[int, int, int | None, int | None]:
    """(lower z code, upper z code, rank below, rank above) of a slab. A periodic grid wraps: the
    lowest slab's neighbour below is the highest. A face on the grid's own boundary keeps the
    grid's code and has no neighbour."""
    if bc_lo == 0:
        return HALO, HALO, (rank - 1) % world, (rank + 1) % world
    lo, prev = (bc_lo, None) if rank == 0 else (HALO, rank - 1)
    hi, nxt = (bc_hi, None) if rank == world - 1 else (HALO, rank + 1)
    return lo, hi, prev, nxt


def exchange_halos(faces: dict, prev: int | None, nxt: int | None, rank: int, group=None) -> None:
    """Fill the ghost planes of each halo face from the neighbouring slab.

    faces[side] = (inner_u1, inner_u2, ghost_u1, ghost_u2) tensors of face side (0 lower, 1 upper).
    The lower face's inner planes become the slab below's upper ghosts, the upper face's inner
    planes the slab above's lower ghosts. Sends go in the order (lower face, upper face) and each
    rank receives in the order its peers send (upper ghosts from above first), so that two sends to
    one peer (a two-slab periodic grid) pair with the right receives.
    """
    if prev == rank and nxt == rank:  # one slab of a periodic grid: its own planes wrap around
        faces[0][2].copy_(faces[1][0])
        faces[0][3].copy_(faces[1][1])
        faces[1][2].copy_(faces[0][0])
        faces[1][3].copy_(faces[0][1])
        return
    ops = []
    if prev is not None:
        ops += [dist.P2POp(dist.isend, faces[0][0], prev, group), dist.P2POp(dist.isend, faces[0][1], prev, group)]
    if nxt is not None:
        ops += [dist.P2POp(dist.isend, faces[1][0], nxt, group), dist.P2POp(dist.isend, faces[1][1], nxt, group)]
    if nxt is not None:
        ops += [dist.P2POp(dist.irecv, faces[1][2], nxt, group), dist.P2POp(dist.irecv, faces[1][3], nxt, group)]
    if prev is not None:
        ops += [dist.P2POp(dist.irecv, faces[0][2], prev, group), dist.P2POp(dist.irecv, faces[0][3], prev, group)]
    if ops:
        for req in dist.batch_isend_irecv(ops):
            req.wait()


class _DeviceArray:
    """A device buffer of the library seen as a 1-D tensor (no copy)."""

    def __init__(self, ptr: int, n: int, typestr: str):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": typestr, "data": (ptr, False), "version": 3,
                                         "strides": None, "stream": None}


def _view(ptr: int, nbytes: int, dtype=torch.float32, device=None) -> torch.Tensor:
    typestr = {torch.float32: "<f4", torch.int32: "<i4"}[dtype]
    return torch.as_tensor(_DeviceArray(ptr, nbytes // 4, typestr), device=device)


class SlabSim:
    """This rank's slab of the grid `cfg` (whose n[2] is the whole grid's), on cuda:<device>."""

    def __init__(self, cfg: Config, group=None, device: int | None = None):
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        if cfg.bc_lo[2] == HALO or cfg.bc_hi[2] == HALO:
            raise ValueError("give the whole grid's own z boundaries; the slab faces are derived")
        nz = int(cfg.n[2])
        self.k0, self.k1 = slab_bounds(nz, self.world, self.rank)
        lo, hi, self.prev, self.next = slab_faces(int(cfg.bc_lo[2]), int(cfg.bc_hi[2]), self.rank, self.world)
        dev = torch.cuda.current_device() if device is None else device
        self.dx = cfg.dx if cfg.dx is not None else 1.0 / cfg.n[0]
        self.cfg = replace(cfg, n=(cfg.n[0], cfg.n[1], self.k1 - self.k0), dx=self.dx,
                           bc_lo=(cfg.bc_lo[0], cfg.bc_lo[1], lo), bc_hi=(cfg.bc_hi[0], cfg.bc_hi[1], hi), device=dev)
        self.grid = replace(cfg, dx=self.dx)
        self.device = torch.device("cuda", dev)
        self.sim = Sim(self.cfg)
        self.stream = torch.cuda.ExternalStream(self.sim.stream_handle(), device=self.device)
        self.halo = (lo == HALO, hi == HALO)

    # -- lifecycle ----------------------------------------------------------------------------
    def destroy(self) -> None:
        self.sim.destroy()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.destroy()

    # -- state --------------------------------------------------------------------------------
    def reset(self, prob: Problem) -> None:
        """This slab's planes of `prob` on the whole grid; the clock goes to 0."""
        self.sim.reset_slab(self.grid, prob, self.k0)

    # -- stepping -----------------------------------------------------------------------------
    def _faces(self) -> dict:
        faces = {}
        for side in (0, 1):
            if self.halo[side]:
                i1, i2, g1, g2, nb = self.sim.halo_device(side)
                faces[side] = tuple(_view(p, nb, device=self.device) for p in (i1, i2, g1, g2))
        return faces

    def step(self, n: int = 1) -> None:
        """n steps, each after its halo exchange and dt all-reduce (enqueued on the handle's
        stream; returns without waiting for the GPU)."""
        with torch.cuda.stream(self.stream):
            for _ in range(n):
                if self.prev is not None or self.next is not None:
                    exchange_halos(self._faces(), self.prev, self.next, self.rank, self.group)
                if self.world > 1:
                    allreduce_rate_word(_view(self.sim.rate_device(), 4, torch.int32, self.device), self.group)
                self.sim.step(1)

    def sync(self) -> None:
        self.sim.sync()

    def clock(self) -> tuple[float, float, int]:
        return self.sim.clock()

    def read_state(self):
        return self.sim.read_state()

    def diagnostics(self) -> Diagnostics:
        """Totals over the whole grid (float64 sums over the slabs; the largest Mach number)."""
        d = self.sim.diagnostics()
        mine = [d.mass, *d.momentum, d.e_kin, d.e_int, d.e_tot, d.floored]
        s = sum_over_ranks(mine, self.group, self.device)
        mach = max_over_ranks(d.max_mach, self.group, self.device)
        return Diagnostics(d.t, d.dt, d.steps, s[0], tuple(s[1:4]), s[4], s[5], s[6], mach, s[7])


_SIGN_BIT = -(2 ** 31)  # an int32 word with only its sign bit set


def allreduce_rate_word(word: torch.Tensor, group=None) -> None:
    """Make a slab's rate word (the float bits of its signal-rate maximum, which the sweep folds
    with an unsigned atomicMax) the unsigned maximum over all ranks, in place.

    Collectives have no unsigned 32-bit MAX, so the word is reduced as int32 with its sign bit
    flipped before and after: that maps unsigned order onto signed order exactly. A NaN rate with
    its sign bit set (0xffc00000) therefore wins over every healthy rank's rate, as it does inside
    one GPU's atomicMax, and the clock of every rank sees it."""
    word.bitwise_xor_(_SIGN_BIT)
    dist.all_reduce(word, op=dist.ReduceOp.MAX, group=group)
    word.bitwise_xor_(_SIGN_BIT)


def sum_over_ranks(values: list[float], group=None, device=None) -> list[float]:
    """Each value's sum over the ranks, correctly rounded (math.fsum of every rank's float64
    value, gathered), so the cross-rank step keeps the compensated totals' accuracy."""
    if not dist.is_initialized() or dist.get_world_size(group) == 1:
        return [float(v) for v in values]
    mine = torch.tensor(values, dtype=torch.float64, device=device)
    world = dist.get_world_size(group)
    every = torch.empty(world * len(values), dtype=torch.float64, device=device)
    dist.all_gather_into_tensor(every, mine, group=group)
    rows = every.view(world, len(values)).cpu().tolist()
    return [math.fsum(r[i] for r in rows) for i in range(len(values))]


def max_over_ranks(x: float, group=None, device=None) -> float:
    """The largest of a value over the ranks (timings are taken as the slowest rank's)."""
    if not dist.is_initialized() or dist.get_world_size(group) == 1:
        return x
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())


def total_cells(cfg: Config) -> int:
    return math.prod(int(v) for v in (list(cfg.n) + [1, 1])[:3])
