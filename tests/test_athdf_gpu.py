"""Snapshots and restarts of runs on the GPU (src/io/capture.ts capture and restartFrom): a run
written to an .athdf file and read back starts a new run whose state is the first's to float32
rounding of the primitives (the file holds primitives: momentum and energy are formed again from
them, as the reference's restart does), on a uniform grid, on blocks (the mesh rebuilt where the
file is finer), and from a uniform file onto blocks at a finer root (levels shifted)."""
import numpy as np
import pytest

from shaderous_b200 import Config, Problem, Sim
from shaderous_b200.amr import AmrConfig, AmrSim
from shaderous_b200.athdf import capture, read_athdf, restart, write_athdf

pytestmark = pytest.mark.gpu

META = {"program": "shaderous", "build": "b200", "query": "problem=kh&dim=2"}


def close_state(a, b):
    """Equal density; momentum and energies within the roundings of going through primitives."""
    (u1a, u2a), (u1b, u2b) = a, b
    assert np.array_equal(u1a[..., 0], u1b[..., 0])
    np.testing.assert_allclose(u1b[..., 1:4], u1a[..., 1:4], rtol=3e-7, atol=1e-12)
    np.testing.assert_allclose(u2b[..., 0:3], u2a[..., 0:3], rtol=2e-6, atol=1e-12)


def test_uniform_run_restarts_from_its_file(tmp_path):
    cfg = Config(n=(96, 64, 1), gamma=1.4, recon="mc", isentropic=False, cfl=0.4)
    path = tmp_path / "kh.athdf"
    with Sim(cfg) as a:
        a.reset(Problem("kh", a=(2, 1, 0.5, 2.5, 0.01, 1e-3), seed=5))
        a.run(steps=30)
        write_athdf(capture(a, META), path)
        t, _, steps = a.clock()
        back = read_athdf(path)
        assert back.meta == {"format": 2, **META}
        assert (back.steps, back.time) == (steps, float(np.float32(t)))
        assert back.root_size == [96, 64, 1] and back.lo == [float(np.float32(v)) for v in (-0.5, -1 / 3, -0.5)]
        with Sim(cfg) as b:
            restart(b, back)
            tb, _, sb = b.clock()
            assert (sb, tb) == (30, float(np.float32(t)))
            close_state(a.read_state(), b.read_state())
            a.run(steps=40)
            b.run(steps=40)
            ra, rb = a.read_state()[0][:, 0], b.read_state()[0][:, 0]
            assert np.abs(ra - rb).sum() / np.abs(ra).sum() < 1e-5
            assert abs(a.diagnostics().mass - b.diagnostics().mass) < 1e-6 * a.diagnostics().mass


def by_block(sim):
    _, lv, co = sim.leaves()
    u1, u2 = sim.leaves_state()
    return {(int(l), *map(int, c)): (u1[i], u2[i]) for i, (l, c) in enumerate(zip(lv, co))}


def test_blocks_restart_on_the_mesh_they_were_saved_on():
    hyd = Config(gamma=5 / 3, bc_lo=(1, 1, 1), bc_hi=(1, 1, 1), recon="koren", isentropic=True, cfl=0.5, p_floor=1e-12)
    cfg = AmrConfig(hydro=hyd, ndim=3, nr=2, max_level=2, cap=1200, refine_hi=0.1, refine_lo=0.05, regrid_every=8)
    with AmrSim(cfg) as a:
        a.reset(Problem("sedov", a=(1, 1e-5, 1, 3.5)))
        a.run(steps=20)
        back = read_athdf(write_athdf(capture(a), gzip=1))
        assert back.root_size == [32, 32, 32] and back.block_size == [16, 16, 16]
        assert back.levels.max() == 2 and len(set(back.levels.tolist())) > 1
        ka = by_block(a)
        with AmrSim(cfg) as b:
            restart(b, back)
            kb = by_block(b)
            assert sorted(ka) == sorted(kb)
            for k in ka:
                close_state(ka[k], kb[k])
            assert b.clock()[2] == 20
            m0 = b.diagnostics().mass
            b.run(steps=16)
            assert abs(b.diagnostics().mass - m0) < 1e-6 * m0


def test_uniform_file_onto_blocks_at_a_finer_root():
    """A 128^2 uniform run's file restarts a run on blocks whose root is 32^2: the file is two
    levels finer everywhere, so every block is refined to level 2 and takes the file's cells."""
    hyd = Config(n=(128, 128, 1), gamma=1.4, recon="mc", isentropic=False, cfl=0.4)
    with Sim(hyd) as u:
        u.reset(Problem("kh", a=(2, 1, 0.5, 2.5, 0.01, 1e-3), seed=9))
        u.run(steps=10)
        snap = read_athdf(write_athdf(capture(u)))
        uni = u.read_state()
    cfg = AmrConfig(hydro=Config(gamma=1.4, recon="mc", isentropic=False, cfl=0.4), ndim=2, nr=2, max_level=2, cap=100,
                    regrid_every=0)
    with AmrSim(cfg) as a:
        restart(a, snap)
        _, lv, _ = a.leaves()
        assert len(lv) == 64 and set(lv.tolist()) == {2}
        g1, g2 = a.uniform_level(2)
        close_state((uni[0].reshape(1, 128, 128, 4), uni[1].reshape(1, 128, 128, 4)), (g1, g2))
        a.run(steps=5)
        assert np.isfinite(a.diagnostics().e_tot)


def test_a_file_that_does_not_cover_the_domain_is_refused():
    hyd = Config(gamma=1.4, recon="mc", isentropic=False)
    cfg = AmrConfig(hydro=hyd, ndim=2, nr=2, max_level=1, cap=40, regrid_every=0)
    with Sim(Config(n=(32, 32, 1), gamma=1.4)) as u:
        u.reset(Problem("kh", a=(2, 1, 0.5, 2.5, 0.01, 0.0)))
        snap = capture(u)
    # keep one quarter of the blocks of a 2 x 2 mesh made from it
    snap.root_size, snap.block_size = [32, 32, 1], [16, 16, 1]
    snap.levels = np.zeros(1, np.int32)
    snap.locations = np.zeros((1, 3), np.int32)
    snap.data = {k: v[:256] for k, v in snap.data.items()}
    from shaderous_b200.sim import ShaderousError

    with AmrSim(cfg) as a, pytest.raises(ShaderousError, match="does not cover"):
        restart(a, snap)
