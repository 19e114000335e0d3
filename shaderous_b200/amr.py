"""Python host mirror of the reference's adaptive-grid simulation (AmrSim, src/amr/amr_sim.ts) over
the C ABI: the same run/step/diagnostics surface as :class:`shaderous_b200.Sim`, plus the mesh
(leaves, block table, refinement indicators) for checks."""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass

import numpy as np

from . import _abi
from ._abi import load
from .sim import Config, Diagnostics, Problem, RunResult, ShaderousError


@dataclass
class AmrConfig:
    """shz_amr_config: physics from `hydro`, the mesh from the rest."""

    hydro: Config
    ndim: int = 3
    nr: int = 2
    max_level: int = 2
    cap: int = 512
    box: float = 1.0
    refine_hi: float = 0.1
    refine_lo: float = 0.05
    regrid_every: int = 8
    two_pass: bool = False  # predict into a half-step atlas, then update (the reference's passes)
    time_bins: int = 0  # per-block timesteps: cycles of 2^time_bins substeps (0: one timestep)
    time_bins_always: bool = False  # never pause the cycles when they save too little

    def to_c(self) -> _abi.shz_amr_config:
        c = _abi.shz_amr_config()
        c.hydro = self.hydro.to_c()
        c.ndim, c.nr, c.max_level, c.cap = self.ndim, self.nr, self.max_level, self.cap
        c.box, c.refine_hi, c.refine_lo, c.regrid_every = self.box, self.refine_hi, self.refine_lo, self.regrid_every
        c.two_pass = 1 if self.two_pass else 0
        c.time_bins = int(self.time_bins)
        c.time_bins_always = 1 if self.time_bins_always else 0
        return c

    @property
    def cells_per_block(self) -> int:
        return 16 ** self.ndim


class AmrSim:
    def __init__(self, cfg: AmrConfig):
        self._lib = load()
        self.cfg = cfg
        h = C.c_void_p()
        rc = self._lib.shz_amr_create(C.byref(cfg.to_c()), C.byref(h))
        if rc != 0:
            raise ShaderousError(rc, self._lib.shz_amr_error(None).decode())
        self._h = h

    def _ok(self, rc):
        if rc != 0:
            raise ShaderousError(rc, self._lib.shz_amr_error(self._h).decode())

    def destroy(self):
        if self._h:
            self._lib.shz_amr_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.destroy()

    def reset(self, prob: Problem):
        self._ok(self._lib.shz_amr_reset_problem(self._h, C.byref(prob.to_c())))

    def step(self, n: int = 1):
        self._ok(self._lib.shz_amr_step(self._h, int(n)))

    def run(self, steps=None, until=None, timeout_ms=None) -> RunResult:
        if steps is None and until is None:
            raise ValueError("run() needs `steps`, `until`, or both")
        o = _abi.shz_run_opts(int(steps) if steps is not None else -1, float(until) if until is not None else math.nan,
                              float(timeout_ms) if timeout_ms else 0.0)
        r = _abi.shz_run_result()
        self._ok(self._lib.shz_amr_run(self._h, C.byref(o), C.byref(r)))
        return RunResult(r.t, r.dt, r.steps, r.taken, r.seconds, _abi.STOPPED.get(r.stopped, "?"), r.last_dt)

    def regrid(self) -> bool:
        ch = C.c_int32()
        self._ok(self._lib.shz_amr_regrid(self._h, C.byref(ch)))
        return bool(ch.value)

    def clock(self):
        t, dt, st = C.c_double(), C.c_double(), C.c_int64()
        self._ok(self._lib.shz_amr_clock(self._h, C.byref(t), C.byref(dt), C.byref(st)))
        return t.value, dt.value, st.value

    def diagnostics(self) -> Diagnostics:
        d = _abi.shz_diag()
        self._ok(self._lib.shz_amr_diagnostics(self._h, C.byref(d)))
        return Diagnostics(d.t, d.dt, d.steps, d.mass, tuple(d.momentum), d.e_kin, d.e_int, d.e_tot, d.max_mach, d.floored)

    def diagnostics_ext(self):
        from .sim import DiagnosticsExt

        d = _abi.shz_diag_ext()
        self._ok(self._lib.shz_amr_diagnostics_ext(self._h, C.byref(d)))
        return DiagnosticsExt.from_c(d)

    def leaves(self):
        """(slots, levels, coords (n, 3)) of the leaves, coarsest first."""
        cap = self.cfg.cap
        n = C.c_int32()
        s = np.zeros(cap, np.int32)
        lv = np.zeros(cap, np.int32)
        co = np.zeros((cap, 3), np.int32)
        self._ok(self._lib.shz_amr_leaves(self._h, C.byref(n), s.ctypes.data, lv.ctypes.data, co.ctypes.data))
        k = n.value
        return s[:k].copy(), lv[:k].copy(), co[:k].copy()

    def table(self) -> np.ndarray:
        t = np.zeros((self.cfg.cap, 32), np.int32)
        self._ok(self._lib.shz_amr_table(self._h, t.ctypes.data))
        return t

    def leaves_state(self):
        """(u1, u2) of shape (n_leaves, cells_per_block, 4), leaves coarsest first."""
        n = len(self.leaves()[0])
        cb = self.cfg.cells_per_block
        u1 = np.zeros((n, cb, 4), np.float32)
        u2 = np.zeros((n, cb, 4), np.float32)
        self._ok(self._lib.shz_amr_get_leaves_state(self._h, u1.ctypes.data, u2.ctypes.data))
        return u1, u2

    def flags(self) -> np.ndarray:
        f = np.zeros(self.cfg.cap, np.float32)
        self._ok(self._lib.shz_amr_flags(self._h, f.ctypes.data))
        return f

    def ghost_map(self, slot: int) -> np.ndarray:
        wn = 20 ** self.cfg.ndim
        out = np.zeros((wn, 5), np.int32)
        self._ok(self._lib.shz_amr_ghost_map(self._h, int(slot), out.ctypes.data))
        return out

    def prims(self, slot: int) -> np.ndarray:
        """Block `slot`'s primitive region as the last assemble left it: (20^ndim, 8) floats per
        texel, x fastest: rho, vx, vy, vz, p, s, cs, 0."""
        wn = 20 ** self.cfg.ndim
        w1 = np.zeros((wn, 4), np.float32)
        w2 = np.zeros((wn, 4), np.float32)
        self._ok(self._lib.shz_amr_prims(self._h, int(slot), w1.ctypes.data, w2.ctypes.data))
        return np.concatenate([w1, w2], axis=1)

    def regrid_table(self) -> np.ndarray:
        """The last re-mesh's regrid table (cap x 12 ints: kind, source, octant, _, children)."""
        t = np.zeros((self.cfg.cap, 12), np.int32)
        self._ok(self._lib.shz_amr_regrid_table(self._h, t.ctypes.data))
        return t

    def profile(self, n: int) -> dict:
        r = _abi.shz_profile_result()
        self._ok(self._lib.shz_amr_profile(self._h, int(n), C.byref(r)))
        return {"steps": r.steps, "total_ms": r.total_ms, "launches": r.launches}

    @property
    def kernel_launches(self) -> int:
        return int(self._lib.shz_amr_kernel_launches(self._h))

    def bins(self):
        """The last cycle's bin table (cap + 1 ints: the substep, then each slot's bin) and the
        blocks' own rates per unit cell size it was formed from (AmrSim.readBins)."""
        b = np.zeros(self.cfg.cap + 1, np.int32)
        r = np.zeros(self.cfg.cap, np.float32)
        self._ok(self._lib.shz_amr_bins(self._h, b.ctypes.data, r.ctypes.data))
        return b, r

    def bin_work(self) -> dict:
        """Cycles taken, block updates made and what single steps would have made (AmrSim.binWork),
        and the single steps left before the cycles resume."""
        cy, up, si, pa = C.c_int64(), C.c_int64(), C.c_int64(), C.c_int32()
        self._ok(self._lib.shz_amr_bin_work(self._h, C.byref(cy), C.byref(up), C.byref(si), C.byref(pa)))
        return {"cycles": cy.value, "updates": up.value, "single": si.value, "paused": pa.value}

    def reset_mesh(self, levels, coords, root_size, block_size, lo, hi, shift: int = 0):
        """Rebuild the mesh from a snapshot's leaves as a restart does (shz_amr_reset_mesh): the
        leaves' state is zero and the clock 0 until set_leaves_state and set_clock."""
        lv = np.ascontiguousarray(levels, np.int32)
        co = np.ascontiguousarray(coords, np.int32).reshape(-1, 3)
        m = _abi.shz_mesh_spec()
        m.n = len(lv)
        m.levels, m.coords = lv.ctypes.data, co.ctypes.data
        m.root_size[:] = [int(v) for v in root_size]
        m.block_size[:] = [int(v) for v in block_size]
        m.lo[:] = [float(v) for v in lo]
        m.hi[:] = [float(v) for v in hi]
        m.shift = int(shift)
        self._ok(self._lib.shz_amr_reset_mesh(self._h, C.byref(m)))

    def set_leaves_state(self, u1: np.ndarray, u2: np.ndarray):
        """Replace every leaf's state: arrays shaped as leaves_state() gives them."""
        n = len(self.leaves()[0])
        cb = self.cfg.cells_per_block
        u1 = np.ascontiguousarray(u1, np.float32).reshape(n, cb, 4)
        u2 = np.ascontiguousarray(u2, np.float32).reshape(n, cb, 4)
        self._ok(self._lib.shz_amr_set_leaves_state(self._h, u1.ctypes.data, u2.ctypes.data))

    def set_clock(self, t: float, steps: int = 0):
        self._ok(self._lib.shz_amr_set_clock(self._h, float(t), int(steps)))

    def uniform_level(self, level: int = 0):
        """Leaves all at one level assembled into a uniform (nz, ny, nx, 4) pair of arrays."""
        s, lv, co = self.leaves()
        assert np.all(lv == level), "the mesh is not uniform at that level"
        u1, u2 = self.leaves_state()
        nb = self.cfg.nr << level
        nd = self.cfg.ndim
        n = nb * 16
        shape = (n, n, n, 4) if nd == 3 else (1, n, n, 4)
        g1 = np.zeros(shape, np.float32)
        g2 = np.zeros(shape, np.float32)
        for i in range(len(s)):
            x0, y0, z0 = co[i] * 16
            if nd == 3:
                g1[z0:z0 + 16, y0:y0 + 16, x0:x0 + 16] = u1[i].reshape(16, 16, 16, 4)
                g2[z0:z0 + 16, y0:y0 + 16, x0:x0 + 16] = u2[i].reshape(16, 16, 16, 4)
            else:
                g1[0, y0:y0 + 16, x0:x0 + 16] = u1[i].reshape(16, 16, 4)
                g2[0, y0:y0 + 16, x0:x0 + 16] = u2[i].reshape(16, 16, 4)
        return g1, g2
