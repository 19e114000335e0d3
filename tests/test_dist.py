"""The z-slab decomposition's host logic on CPU (gloo, world sizes 2 and 3): slab bounds, face
codes and neighbours, the halo exchange (periodic and walled grids, two sends to one peer), the
max-over-ranks timing, and a multi-step stencil on exchanged halos equal to the same stencil on
the whole field."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from shaderous_b200.dist import HALO, exchange_halos, max_over_ranks, slab_bounds, slab_faces


def test_slab_bounds_cover_the_grid():
    for nz, world in [(512, 1), (512, 2), (512, 8), (100, 3), (7, 7)]:
        spans = [slab_bounds(nz, world, r) for r in range(world)]
        assert spans[0][0] == 0 and spans[-1][1] == nz
        assert all(a[1] == b[0] for a, b in zip(spans, spans[1:]))
        sizes = [k1 - k0 for k0, k1 in spans]
        assert max(sizes) - min(sizes) <= 1


def test_slab_faces():
    # periodic: halos everywhere, wrapping
    assert slab_faces(0, 0, 0, 4) == (HALO, HALO, 3, 1)
    assert slab_faces(0, 0, 3, 4) == (HALO, HALO, 2, 0)
    assert slab_faces(0, 0, 0, 1) == (HALO, HALO, 0, 0)
    # walls / outflow: the grid's own faces at the ends
    assert slab_faces(2, 1, 0, 3) == (2, HALO, None, 1)
    assert slab_faces(2, 1, 1, 3) == (HALO, HALO, 0, 2)
    assert slab_faces(2, 1, 2, 3) == (HALO, 1, 1, None)
    assert slab_faces(1, 1, 0, 1) == (1, 1, None, None)


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


D = 2  # halo depth in planes
NX = 3  # cells per plane (x*y collapsed) in the toy field


def _stencil(u: np.ndarray, periodic: bool) -> np.ndarray:
    """One step of a 5-plane stencil along z on a whole field (outflow: edge planes repeated)."""
    if periodic:
        p = np.concatenate([u[-D:], u, u[:D]])
    else:
        p = np.concatenate([np.repeat(u[:1], D, 0), u, np.repeat(u[-1:], D, 0)])
    n = u.shape[0]
    return (0.5 * p[D:D + n] + 0.2 * (p[D - 1:D - 1 + n] + p[D + 1:D + 1 + n])
            + 0.05 * (p[D - 2:D - 2 + n] + p[D + 2:D + 2 + n])).astype(np.float32)


def _worker(rank: int, world: int, port: int, periodic: bool, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        nz = 11
        rng = np.random.default_rng(5)
        whole = rng.standard_normal((nz, NX)).astype(np.float32)
        k0, k1 = slab_bounds(nz, world, rank)
        lo, hi, prev, nxt = slab_faces(0 if periodic else 1, 0 if periodic else 1, rank, world)
        # this slab with D stored planes each side (u1 and u2 carry the same field, offset)
        buf1 = torch.zeros((k1 - k0 + 2 * D, NX))
        buf2 = torch.zeros((k1 - k0 + 2 * D, NX))
        buf1[D:D + k1 - k0] = torch.from_numpy(whole[k0:k1])
        buf2[D:D + k1 - k0] = torch.from_numpy(whole[k0:k1]) + 100.0
        ref = whole.copy()
        for step in range(4):
            faces = {}
            if lo == HALO:
                faces[0] = (buf1[D:2 * D], buf2[D:2 * D], buf1[0:D], buf2[0:D])
            if hi == HALO:
                n = k1 - k0
                faces[1] = (buf1[n:n + D], buf2[n:n + D], buf1[n + D:n + 2 * D], buf2[n + D:n + 2 * D])
            exchange_halos(faces, prev, nxt, rank)
            # the grid's own outflow faces: edge planes repeated
            if lo != HALO:
                buf1[0:D] = buf1[D]
                buf2[0:D] = buf2[D]
            if hi != HALO:
                n = k1 - k0
                buf1[n + D:] = buf1[n + D - 1]
                buf2[n + D:] = buf2[n + D - 1]
            # the stencil on the slab with its ghosts, against the whole field
            for buf in (buf1, buf2):
                p = buf.numpy()
                n = k1 - k0
                new = (0.5 * p[D:D + n] + 0.2 * (p[D - 1:D - 1 + n] + p[D + 1:D + 1 + n])
                       + 0.05 * (p[D - 2:D - 2 + n] + p[D + 2:D + 2 + n])).astype(np.float32)
                buf[D:D + n] = torch.from_numpy(new)
            ref = _stencil(ref, periodic)
        ok1 = np.array_equal(buf1[D:D + k1 - k0].numpy(), ref[k0:k1])
        ok2 = np.array_equal(buf2[D:D + k1 - k0].numpy(), _ref_offset(whole, periodic)[k0:k1])
        slow = max_over_ranks(float(rank) + 0.5)
        q.put((rank, ok1, ok2, slow))
    finally:
        dist.destroy_process_group()


def _ref_offset(whole, periodic):
    r = whole.astype(np.float32) + np.float32(100.0)
    for _ in range(4):
        r = _stencil(r, periodic)
    return r


@pytest.mark.parametrize("world,periodic", [(2, True), (2, False), (3, True), (3, False)])
def test_halo_exchange_matches_whole_field(world, periodic):
    ctx = mp.get_context("spawn")
    q = ctx.SimpleQueue()
    mp.start_processes(_worker, args=(world, _free_port(), periodic, q), nprocs=world, start_method="spawn")
    got = sorted(q.get() for _ in range(world))
    for rank, ok1, ok2, slow in got:
        assert ok1 and ok2, (rank, ok1, ok2)
        assert slow == world - 1 + 0.5
