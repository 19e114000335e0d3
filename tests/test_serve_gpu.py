"""Serving on the GPU: each request's result is the same alone and in a mix of others (bitwise:
the blocks of a request see only their own grid), and the same as the plain uniform-grid step
(within 1e-6 relative L1 of density: both float32, the block passes and the fused sweep differ in
the order of a few roundings). A seeded Poisson stream completes with sane statistics."""
import numpy as np
import pytest

from shaderous_b200 import Config, Problem, Sim
from shaderous_b200.serve import Request, Server, ServerConfig, plain_run_stream, request_stream

pytestmark = pytest.mark.gpu


def _mix():
    return [
        Request(ndim=2, n=64, steps=37, problem=Problem("kh", a=(2, 1, 0.5, 2.5, 0.01, 1e-3), seed=5), gamma=1.4, bc=0),
        Request(ndim=3, n=32, steps=20, problem=Problem("blast", a=(3, 50, 1, 1, 0.15)), gamma=5 / 3, bc=1),
        Request(ndim=2, n=48, steps=55, problem=Problem("sod", a=(4, 0, 20, 1, 0, 1)), gamma=5 / 3, bc=1),
        Request(ndim=3, n=48, steps=9, problem=Problem("sod", a=(2, 0, 5, 1, 0, 1)), gamma=1.4, bc=2),
    ]


def _cfg():
    return ServerConfig(hydro=Config(recon="koren", isentropic=True, cfl=0.4), budget_bytes=2e9, max_grids=16,
                        round_steps=4, keep_states=True)


def test_same_result_alone_and_in_the_mix():
    reqs = _mix()
    together = {}
    with Server(_cfg()) as s:
        ids = [s.submit(r) for r in reqs]
        s.drain()
        for r, i in zip(reqs, ids):
            d = s.result(i)
            assert d.steps == r.steps
            together[i] = s.state(i, r)
    for r, i in zip(reqs, ids):
        with Server(_cfg()) as s:
            j = s.submit(r)
            s.drain()
            a1, a2 = s.state(j, r)
        assert np.array_equal(a1, together[i][0]) and np.array_equal(a2, together[i][1])
        # the plain uniform-grid step on the same request
        c = Config(n=(r.n, r.n, r.n if r.ndim == 3 else 1), dx=1.0 / r.n, gamma=r.gamma, recon="koren", isentropic=True,
                   cfl=0.4, bc_lo=tuple(r.bc if a < r.ndim else 0 for a in range(3)),
                   bc_hi=tuple(r.bc if a < r.ndim else 0 for a in range(3)))
        with Sim(c) as p:
            p.reset(r.problem)
            p.run(steps=r.steps)
            u1, _ = p.read_state()
        rel = np.abs(a1[:, 0].astype(np.float64) - u1[:, 0]).sum() / np.abs(u1[:, 0]).sum()
        assert rel < 1e-6, (r, rel)


def test_stream_completes_with_stats():
    reqs = request_stream(24, seed=7, rate=200.0, sizes2=(32, 128), sizes3=(16, 48), steps=(10, 60))
    with Server(ServerConfig(budget_bytes=2e9, max_grids=32, round_steps=4)) as s:
        st = s.run_stream(reqs)
    assert st["completed"] == 24
    assert 0 < st["p50_s"] <= st["p99_s"] <= st["makespan_s"] + 1e-9
    assert st["zone_updates"] == sum(r.cells * r.steps for r in reqs)
    assert st["max_concurrent"] > 1  # requests overlapped on the device
    plain = plain_run_stream(ServerConfig(), reqs)
    assert plain["completed"] == 24 and plain["zone_updates"] == st["zone_updates"]


def test_refuses_bad_requests():
    from shaderous_b200 import ShaderousError

    with Server(ServerConfig(budget_bytes=1e8, max_grids=4)) as s:
        with pytest.raises(ShaderousError):
            s.submit(Request(ndim=3, n=40, steps=5, problem=Problem("blast", a=(1, 10, 1, 1, 0.1))))
        with pytest.raises(ShaderousError):
            s.submit(Request(ndim=3, n=512, steps=5, problem=Problem("blast", a=(1, 10, 1, 1, 0.1))))


def test_large_requests_run_as_uniform_grids_with_the_plain_steps_bits():
    """With direct_large (the default), requests of at least 2^18 (2D) or 2^21 (3D) cells run as
    uniform grids on streams of their own, their steps enqueued in the same rounds as the batched
    blocks of the small requests; each large result equals the plain uniform-grid step's bit for
    bit, and the small ones are unchanged by the mix."""
    big = [
        Request(ndim=3, n=128, steps=21, problem=Problem("blast", a=(3, 50, 1, 1, 0.15)), gamma=5 / 3, bc=1),
        Request(ndim=2, n=512, steps=33, problem=Problem("kh", a=(2, 1, 0.5, 2.5, 0.01, 1e-3), seed=9), gamma=1.4,
                bc=0),
    ]
    small = _mix()[:2]
    reqs = big + small
    with Server(_cfg()) as s:
        ids = [s.submit(r) for r in reqs]
        s.drain()
        got = {i: s.state(i, r) for r, i in zip(reqs, ids)}
        for r, i in zip(reqs, ids):
            assert s.result(i).steps == r.steps
    for r, i in zip(big, ids[:2]):
        c = Config(n=(r.n, r.n, r.n if r.ndim == 3 else 1), dx=1.0 / r.n, gamma=r.gamma, recon="koren", isentropic=True,
                   cfl=0.4, bc_lo=tuple(r.bc if a < r.ndim else 0 for a in range(3)),
                   bc_hi=tuple(r.bc if a < r.ndim else 0 for a in range(3)))
        with Sim(c) as p:
            p.reset(r.problem)
            p.run(steps=r.steps)
            u1, u2 = p.read_state()
        assert np.array_equal(got[i][0], u1) and np.array_equal(got[i][1], u2), r
    with Server(_cfg()) as s:
        for r, i in zip(small, ids[2:]):
            j = s.submit(r)
            s.drain()
            a1, a2 = s.state(j, r)
            assert np.array_equal(a1, got[i][0]) and np.array_equal(a2, got[i][1])
