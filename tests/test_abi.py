"""CPU checks of the boundary: the library loads without a GPU, exports every symbol the headers
declare, refuses bad configurations, and its host-side initial conditions are deterministic."""
import ctypes as C
import math
import re
from pathlib import Path

import numpy as np
import pytest

from shaderous_b200 import Config, Problem, problem_prims, prims_to_state
from shaderous_b200 import _abi

ROOT = Path(__file__).resolve().parent.parent


def declared_functions():
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        for m in re.finditer(r"^[A-Za-z_][\w\s\*]*?\b(shz_\w+)\s*\(", text, flags=re.M):
            names.add(m.group(1))
    return names


def test_library_loads_and_exports_every_declared_symbol():
    lib = _abi.load()
    names = declared_functions()
    assert len(names) >= 18
    for name in names:
        assert hasattr(lib, name), name
    # and the ctypes table covers the same set
    assert {n for n, _, _ in _abi.SIGNATURES} >= names


def test_version_and_defaults():
    lib = _abi.load()
    assert b"sm_100a" in lib.shz_version()
    c = _abi.shz_config()
    assert lib.shz_config_default(C.byref(c), 64, 32, 1, 1 / 64) == 0
    assert (c.cfl, c.rho_floor, c.p_floor, c.eta_dual, c.shock_thresh) == (0.8, 1e-10, 1e-14, 1e-3, 0.5)
    assert c.recon == 3 and c.riemann == 0 and c.isentropic == 1 and c.signal_dims == 3
    assert math.isinf(c.t_end)


def test_problem_prims_deterministic_and_slab_independent():
    cfg = Config(n=(32, 16, 8), gamma=1.4)
    prob = Problem("kh", a=(2, 1, 0.5, 2.5, 0.01, 1e-3), seed=7)
    full = problem_prims(cfg, prob)
    parts = np.concatenate([problem_prims(cfg, prob, 0, 3), problem_prims(cfg, prob, 3, 8)])
    assert np.array_equal(full, parts)
    assert np.array_equal(full, problem_prims(cfg, prob))
    other = problem_prims(cfg, Problem("kh", a=(2, 1, 0.5, 2.5, 0.01, 1e-3), seed=8))
    assert not np.array_equal(full, other)
    # the noise has the stated sigma: vy - mode
    nx = 32
    x = (np.arange(nx) + 0.5) / nx
    mode = 0.01 * np.sin(4 * np.pi * x)
    vy = full[:, 2].reshape(8, 16, 32) - mode
    assert abs(vy.std() - 1e-3) < 2e-4


def test_sedov_deposit_matches_region_rule():
    """src/setup/parts/region.ts:199-215: E spread over the cells whose centres lie within r."""
    n = 32
    cfg = Config(n=(n, n, n), gamma=5 / 3)
    p = problem_prims(cfg, Problem("sedov", a=(1, 1e-5, 1.0, 3.5)))
    eint = p[:, 4] / (5 / 3 - 1)
    hot = p[:, 4] > 1e-5 * 2
    dx = 1 / n
    # total internal energy of the deposit is E = 1
    assert eint[hot].sum() * dx ** 3 == pytest.approx(1.0, rel=1e-12)
    # the count: half-integer lattice points within 3.5
    c = np.arange(-4, 4) + 0.5
    X, Y, Z = np.meshgrid(c, c, c)
    assert hot.sum() == int((np.sqrt(X * X + Y * Y + Z * Z) < 3.5).sum())


def test_tgv_and_sod_inits():
    n = 16
    cfg = Config(n=(n, n, n), dx=2 * math.pi / n)
    p = problem_prims(cfg, Problem("tgv", a=(1, 100, 1)))
    X = (np.arange(n) + 0.5) * 2 * math.pi / n
    vx = p[:, 1].reshape(n, n, n)
    expect = np.sin(X)[None, None, :] * np.cos(X)[None, :, None] * np.cos(X)[:, None, None]
    assert np.allclose(vx, expect, atol=1e-14)
    assert np.all(p[:, 3] == 0) and np.all(p[:, 4] == 100)
    cfg1 = Config(n=(512, 1, 1), gamma=1.4)
    s = problem_prims(cfg1, Problem("sod", a=(1, 0, 1, 0.125, 0, 0.1)))
    assert np.all(s[:256, 0] == 1) and np.all(s[256:, 0] == 0.125)
    u1, u2 = prims_to_state(s, 1.4)
    assert u1.dtype == np.float32 and u2[0, 0] == np.float32(1 / 0.4)


def test_refuses_bad_configs_without_gpu():
    lib = _abi.load()
    for cfg in [Config(n=(1, 8, 8)), Config(n=(64, 1, 1), bc_lo=(1, 2, 0)), Config(n=(2, 2, 2), recon="ppm"),
                Config(n=(8, 1, 1), gamma=1.0), Config(n=(8, 1, 1), bc_lo=(5, 0, 0))]:
        c = cfg.to_c()
        h = C.c_void_p()
        rc = lib.shz_create(C.byref(c), C.byref(h))
        assert rc in (_abi.SHZ_E_CONFIG, _abi.SHZ_E_NODEV)
        if rc == _abi.SHZ_E_CONFIG:
            assert b"refused" in lib.shz_last_error(None)


def test_reference_arm_tgv_init_equals_the_library_init():
    """bench.py's reference arm builds the Taylor-Green init with numpy alone; it is the library's
    init of the same grid (both float64 at the cell centres)."""
    import bench

    n = 12
    cfg = Config(n=(n, n, n), dx=2 * math.pi / n, gamma=5 / 3)
    want = problem_prims(cfg, Problem("tgv", a=(1.0, 100.0, 1.0)))
    got = bench.tgv_prims(n)
    np.testing.assert_allclose(got, np.asarray(want).reshape(-1, 6), rtol=0, atol=1e-14)
