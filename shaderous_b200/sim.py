"""Python host mirror of the reference's simulation API over the C ABI.

The reference's TypeScript callers hold a ``Simulation`` (src/sim.ts:465-628) and drive it with
``run({steps, until, timeoutMs}) -> RunResult`` (src/ui/api.ts:188-210, 538). :class:`Sim` has the
same operations with the same argument meaning and the same refusals, so host code and tests
read like the reference's: ``step``, ``run``, ``read_state``/``set_state``, ``diagnostics``,
``reset``, ``destroy``.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field

import numpy as np

from . import _abi
from ._abi import load


class ShaderousError(RuntimeError):
    """A non-zero status from the C ABI, with the library's message."""

    def __init__(self, code: int, message: str):
        super().__init__(f"[{code}] {message}")
        self.code = code


@dataclass
class RunResult:
    """As RunResult (src/ui/api.ts:199-210)."""

    t: float
    dt: float
    steps: int
    taken: int
    seconds: float
    stopped: str
    last_dt: float


@dataclass
class Diagnostics:
    """Conservation totals in float64, as Diagnostics (src/sim.ts:1810-1862)."""

    t: float
    dt: float
    steps: int
    mass: float
    momentum: tuple
    e_kin: float
    e_int: float
    e_tot: float
    max_mach: float
    floored: float


@dataclass
class DiagnosticsExt:
    """The totals and the reference's other Diagnostics channels (src/sim.ts:1810-1862): ranges
    as [min, max] of density, temperature, scalar, pressure and speed (FIELDS order), the centre
    of mass from the box centre; gravity, Jeans and burning channels (zero on this path)."""

    totals: Diagnostics
    ranges: dict
    com: tuple
    e_grav: float
    jeans_unresolved: float
    nuclear_heating: float

    @staticmethod
    def from_c(d) -> "DiagnosticsExt":
        b = d.base
        tot = Diagnostics(b.t, b.dt, b.steps, b.mass, tuple(b.momentum), b.e_kin, b.e_int, b.e_tot, b.max_mach, b.floored)
        names = ("rho", "temperature", "scalar", "pressure", "speed")
        return DiagnosticsExt(tot, {k: (d.range[i][0], d.range[i][1]) for i, k in enumerate(names)}, tuple(d.com),
                              d.e_grav, d.jeans_unresolved, d.nuclear_heating)


@dataclass
class Config:
    """The hot-path subset of SimConfig (src/sim.ts:48-265), defaults from configFor (:645-742)."""

    n: tuple = (64, 1, 1)
    dx: float | None = None  # default: 1 / n[0] (the reference's box of 1)
    gamma: float = 5.0 / 3.0
    bc_lo: tuple = (0, 0, 0)
    bc_hi: tuple = (0, 0, 0)
    cfl: float = 0.8
    rho_floor: float = 1e-10
    p_floor: float = 1e-14
    eta_dual: float = 1e-3
    shock_thresh: float = 0.5
    riemann: str = "hllc"
    recon: str = "koren"
    isentropic: bool = True
    signal_dims: int = 3
    t_end: float = math.inf
    dt_max: float = math.inf
    device: int = 0

    def to_c(self) -> _abi.shz_config:
        c = _abi.shz_config()
        nx, ny, nz = (list(self.n) + [1, 1])[:3]
        c.n[:] = [int(nx), int(ny), int(nz)]
        c.dx = float(self.dx if self.dx is not None else 1.0 / nx)
        c.gamma = float(self.gamma)
        c.bc_lo[:] = [int(b) for b in self.bc_lo]
        c.bc_hi[:] = [int(b) for b in self.bc_hi]
        c.cfl = float(self.cfl)
        c.rho_floor = float(self.rho_floor)
        c.p_floor = float(self.p_floor)
        c.eta_dual = float(self.eta_dual)
        c.shock_thresh = float(self.shock_thresh)
        c.riemann = _abi.RIEMANN[self.riemann]
        c.recon = _abi.RECON[self.recon]
        c.isentropic = 1 if self.isentropic else 0
        c.signal_dims = int(self.signal_dims)
        c.t_end = float(self.t_end)
        c.dt_max = float(self.dt_max)
        c.device = int(self.device)
        return c

    @property
    def ncell(self) -> int:
        nx, ny, nz = (list(self.n) + [1, 1])[:3]
        return int(nx) * int(ny) * int(nz)


@dataclass
class Problem:
    """A built-in initial condition (include/shaderous_b200.h SHZ_PROB_*)."""

    kind: str
    a: tuple = ()
    axis: int = 0
    seed: int = 0

    def to_c(self) -> _abi.shz_problem:
        p = _abi.shz_problem()
        p.kind = _abi.PROBLEM[self.kind]
        p.axis = int(self.axis)
        p.seed = int(self.seed) & 0xFFFFFFFFFFFFFFFF
        vals = list(self.a) + [0.0] * (8 - len(self.a))
        p.a[:] = [float(v) for v in vals[:8]]
        return p


def _check(lib, handle, rc: int):
    if rc != 0:
        msg = lib.shz_last_error(handle)
        raise ShaderousError(rc, msg.decode() if msg else "unknown error")


def problem_prims(cfg: Config, prob: Problem, k0: int = 0, k1: int | None = None) -> np.ndarray:
    """Float64 primitives (rho, vx, vy, vz, p, s) of planes k0..k1-1: the numbers the library
    rounds to float32 in ``Sim.reset``. Host code only; no device is needed."""
    lib = load()
    c = cfg.to_c()
    nx, ny, nz = c.n[0], c.n[1], c.n[2]
    k1 = nz if k1 is None else k1
    out = np.empty(((k1 - k0) * ny * nx, 6), dtype=np.float64)
    _check(lib, None, lib.shz_problem_prims(C.byref(c), C.byref(prob.to_c()), k0, k1, out.ctypes.data))
    return out


def prims_to_state(prims: np.ndarray, gamma: float) -> tuple[np.ndarray, np.ndarray]:
    """Conserved float32 (u1, u2) from float64 primitives, rounded once (src/sim.ts:2704-2848)."""
    rho, vx, vy, vz, p, s = (prims[:, i] for i in range(6))
    eint = p / (gamma - 1)
    u1 = np.stack([rho, rho * vx, rho * vy, rho * vz], axis=1).astype(np.float32)
    u2 = np.stack([eint + 0.5 * rho * (vx * vx + vy * vy + vz * vz), eint, rho * s, np.zeros_like(rho)], axis=1).astype(np.float32)
    return u1, u2


class Sim:
    """One uniform grid on the device: the reference's ``Simulation`` for a uniform grid."""

    def __init__(self, cfg: Config):
        self._lib = load()
        self.cfg = cfg
        self._c = cfg.to_c()
        h = C.c_void_p()
        _check(self._lib, None, self._lib.shz_create(C.byref(self._c), C.byref(h)))
        self._h = h
        self.ncell = cfg.ncell

    # -- lifecycle ----------------------------------------------------------------------------
    def destroy(self) -> None:
        if self._h:
            self._lib.shz_destroy(self._h)
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

    def _ok(self, rc: int):
        _check(self._lib, self._h, rc)

    # -- state --------------------------------------------------------------------------------
    def reset(self, prob: Problem) -> None:
        """Load a built-in problem; the clock goes to 0 (Sim.reset, src/sim.ts:2704)."""
        self._ok(self._lib.shz_reset_problem(self._h, C.byref(prob.to_c())))

    def set_state(self, u1: np.ndarray, u2: np.ndarray) -> None:
        """Replace the state (Simulation.setState): float32 (ncell, 4) arrays, x fastest."""
        u1 = np.ascontiguousarray(u1, dtype=np.float32).reshape(-1, 4)
        u2 = np.ascontiguousarray(u2, dtype=np.float32).reshape(-1, 4)
        self._ok(self._lib.shz_set_state(self._h, u1.ctypes.data, u2.ctypes.data, u1.shape[0]))

    def read_state(self) -> tuple[np.ndarray, np.ndarray]:
        """Fresh host copies of (u1, u2), shape (ncell, 4) (Simulation.readState, src/sim.ts:3790)."""
        u1 = np.empty((self.ncell, 4), dtype=np.float32)
        u2 = np.empty((self.ncell, 4), dtype=np.float32)
        self._ok(self._lib.shz_get_state(self._h, u1.ctypes.data, u2.ctypes.data, self.ncell))
        return u1, u2

    # -- stepping -----------------------------------------------------------------------------
    def step(self, n: int = 1) -> None:
        """Enqueue n steps (encodeSteps + submit); returns at once."""
        self._ok(self._lib.shz_step(self._h, int(n)))

    def sync(self) -> None:
        self._ok(self._lib.shz_sync(self._h))

    def run(self, steps: int | None = None, until: float | None = None, timeout_ms: float | None = None) -> RunResult:
        """As run() (src/ui/api.ts:538): needs `steps`, `until`, or both."""
        if steps is None and until is None:
            raise ValueError("run() needs `steps`, `until`, or both")
        if steps is not None and not steps >= 0:
            raise ValueError("`steps` must be a number of steps, 0 or more")
        o = _abi.shz_run_opts(int(steps) if steps is not None else -1, float(until) if until is not None else math.nan,
                              float(timeout_ms) if timeout_ms else 0.0)
        r = _abi.shz_run_result()
        self._ok(self._lib.shz_run(self._h, C.byref(o), C.byref(r)))
        return RunResult(r.t, r.dt, r.steps, r.taken, r.seconds, _abi.STOPPED.get(r.stopped, "?"), r.last_dt)

    def clock(self) -> tuple[float, float, int]:
        t, dt, st = C.c_double(), C.c_double(), C.c_int64()
        self._ok(self._lib.shz_clock(self._h, C.byref(t), C.byref(dt), C.byref(st)))
        return t.value, dt.value, st.value

    def set_clock(self, t: float, steps: int = 0) -> None:
        self._ok(self._lib.shz_set_clock(self._h, float(t), int(steps)))

    def set_t_end(self, t_end: float) -> None:
        self._ok(self._lib.shz_set_t_end(self._h, float(t_end)))

    def diagnostics(self) -> Diagnostics:
        d = _abi.shz_diag()
        self._ok(self._lib.shz_diagnostics(self._h, C.byref(d)))
        return Diagnostics(d.t, d.dt, d.steps, d.mass, tuple(d.momentum), d.e_kin, d.e_int, d.e_tot, d.max_mach, d.floored)

    def diagnostics_ext(self) -> DiagnosticsExt:
        d = _abi.shz_diag_ext()
        self._ok(self._lib.shz_diagnostics_ext(self._h, C.byref(d)))
        return DiagnosticsExt.from_c(d)

    def state_device(self) -> tuple[int, int]:
        a, b = C.c_void_p(), C.c_void_p()
        self._ok(self._lib.shz_state_device(self._h, C.byref(a), C.byref(b)))
        return a.value, b.value

    # -- slabs of a grid split along z (SHZ_BC_HALO faces) -----------------------------------------
    def reset_slab(self, grid: Config, prob: Problem, k0: int) -> None:
        """Load planes k0.. of `prob` sampled on the whole grid `grid`; the clock goes to 0."""
        self._ok(self._lib.shz_reset_problem_slab(self._h, C.byref(grid.to_c()), C.byref(prob.to_c()), int(k0)))

    def halo_depth(self) -> int:
        d = C.c_int32()
        self._ok(self._lib.shz_halo_depth(self._h, C.byref(d)))
        return d.value

    def halo_device(self, side: int) -> tuple[int, int, int, int, int]:
        """(inner u1, inner u2, ghost u1, ghost u2, bytes) of z face `side` of the current state."""
        p = [C.c_void_p() for _ in range(4)]
        b = C.c_size_t()
        self._ok(self._lib.shz_halo_device(self._h, int(side), *[C.byref(x) for x in p], C.byref(b)))
        return p[0].value, p[1].value, p[2].value, p[3].value, b.value

    def rate_device(self) -> int:
        p = C.c_void_p()
        self._ok(self._lib.shz_rate_device(self._h, C.byref(p)))
        return p.value

    def stream_handle(self) -> int:
        p = C.c_void_p()
        self._ok(self._lib.shz_stream(self._h, C.byref(p)))
        return p.value or 0

    def profile(self, n: int) -> dict:
        """Device time of n steps and of their sweeps alone, by CUDA events on the handle's
        stream (the reference's Sim.profile, src/sim.ts:3541)."""
        r = _abi.shz_profile_result()
        self._ok(self._lib.shz_profile(self._h, int(n), C.byref(r)))
        return {"steps": r.steps, "total_ms": r.total_ms, "sweep_ms": r.sweep_ms, "launches": r.launches}

    @property
    def kernel_launches(self) -> int:
        return int(self._lib.shz_kernel_launches(self._h))
