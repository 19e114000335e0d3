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


def _word_worker(rank: int, world: int, port: int, q):
    from shaderous_b200.dist import allreduce_rate_word, sum_over_ranks

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        def bits(x):
            return int(np.array([x], dtype=np.float32).view(np.int32)[0])

        neg_nan = int(np.array([0xFFC00000], dtype=np.uint32).view(np.int32)[0])
        cases = {
            "finite": [bits(3.0), bits(7.5), bits(0.25)],
            "neg_nan": [bits(3.0), neg_nan, bits(1e30)],
            "pos_nan": [bits(np.inf), bits(2.0), 0x7FC00000],
            "inf": [bits(np.inf), bits(2.0), bits(5.0)],
        }
        out = {}
        for name, per_rank in cases.items():
            w = torch.tensor([per_rank[rank]], dtype=torch.int32)
            allreduce_rate_word(w)
            out[name] = int(w.item())
        # correctly rounded sums: one rank's large value and others' small ones that plain
        # float64 addition in rank order would lose
        vals = [[1e16, 1.0, -3.0], [1.0, 1e-3, 2.0], [1.0, 1e-3, 1.0]][rank]
        out["sums"] = sum_over_ranks(vals)
        q.put((rank, out))
    finally:
        dist.destroy_process_group()


def test_rate_word_reduces_as_unsigned_and_sums_are_correctly_rounded():
    """The rate word's maximum over ranks is the unsigned maximum the sweep's atomicMax takes: a
    NaN whose sign bit is set wins over the healthy ranks (so every rank's clock reports NaN);
    the totals' cross-rank sum is math.fsum of the ranks' values."""
    import math

    world = 3
    ctx = mp.get_context("spawn")
    q = ctx.SimpleQueue()
    mp.start_processes(_word_worker, args=(world, _free_port(), q), nprocs=world, start_method="spawn")
    got = dict(q.get() for _ in range(world))
    u = lambda x: int(np.array([x], dtype=np.int32).view(np.uint32)[0])  # noqa: E731
    f = lambda x: float(np.array([x], dtype=np.int32).view(np.float32)[0])  # noqa: E731
    for rank, out in got.items():
        assert f(out["finite"]) == 7.5
        assert u(out["neg_nan"]) == 0xFFC00000, hex(u(out["neg_nan"]))
        assert u(out["pos_nan"]) == 0x7FC00000
        assert f(out["inf"]) == np.inf
        want = [math.fsum([1e16, 1.0, 1.0]), math.fsum([1.0, 1e-3, 1e-3]), 0.0]
        assert out["sums"] == want, (rank, out["sums"], want)
