"""ORACLE — test infrastructure only (tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
leg). ctypes wrapper of ``oracle/liboracle.so``, the float64 C++ restatement of the reference's
CPU scheme ``src/reference/hydro.ts`` (``RefHydro``) and its exact Riemann solver
``src/reference/riemann_exact.ts`` (see ``oracle/ref_hydro.cpp``).
"""
from __future__ import annotations

import ctypes as C
import math
from pathlib import Path

import numpy as np

LIB_PATH = Path(__file__).resolve().parent / "liboracle.so"

RECON = {"minmod": 0, "mc": 1, "vanleer": 2, "koren": 3, "ppm": 4}
RIEMANN = {"hllc": 0, "hll": 1}


class orc_config(C.Structure):
    _fields_ = [
        ("n", C.c_int32 * 3),
        ("dx", C.c_double),
        ("gamma", C.c_double),
        ("bc_lo", C.c_int32 * 3),
        ("bc_hi", C.c_int32 * 3),
        ("cfl", C.c_double),
        ("rho_floor", C.c_double),
        ("p_floor", C.c_double),
        ("eta_dual", C.c_double),
        ("shock_thresh", C.c_double),
        ("riemann", C.c_int32),
        ("recon", C.c_int32),
        ("isentropic", C.c_int32),
        ("signal_dims", C.c_int32),
    ]


_lib = None


def load():
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise OSError(f"{LIB_PATH} is not built: run `python -m shaderous_b200.build`")
        lib = C.CDLL(str(LIB_PATH))
        lib.orc_create.restype = C.c_void_p
        lib.orc_create.argtypes = [C.POINTER(orc_config)]
        lib.orc_destroy.argtypes = [C.c_void_p]
        lib.orc_set_threads.argtypes = [C.c_void_p, C.c_int]
        lib.orc_init_prims.argtypes = [C.c_void_p, C.c_void_p]
        lib.orc_set_conserved.argtypes = [C.c_void_p, C.c_void_p]
        lib.orc_get_conserved.argtypes = [C.c_void_p, C.c_void_p]
        lib.orc_step.restype = C.c_double
        lib.orc_step.argtypes = [C.c_void_p, C.c_double]
        lib.orc_run.argtypes = [C.c_void_p, C.c_double, C.c_int64]
        lib.orc_time.restype = C.c_double
        lib.orc_time.argtypes = [C.c_void_p]
        lib.orc_dt.restype = C.c_double
        lib.orc_dt.argtypes = [C.c_void_p]
        lib.orc_steps.restype = C.c_int64
        lib.orc_steps.argtypes = [C.c_void_p]
        lib.orc_set_clock.argtypes = [C.c_void_p, C.c_double, C.c_int64]
        lib.orc_limiter.restype = C.c_double
        lib.orc_limiter.argtypes = [C.c_int, C.c_double, C.c_double, C.c_double]
        lib.orc_ppm_edges.argtypes = [C.c_double] * 5 + [C.POINTER(C.c_double), C.POINTER(C.c_double)]
        lib.orc_exact_riemann.argtypes = [C.c_double] * 7 + [C.c_void_p, C.c_int64, C.c_void_p]
        _lib = lib
    return _lib


def limiter(kind: str, a: float, b: float, scale: float = 0.0) -> float:
    """hydro.ts:30-46 LIMITERS[kind](a, b, scale)."""
    return load().orc_limiter(RECON[kind], a, b, scale)


def ppm_edges(a2m: float, am: float, a: float, ap: float, a2p: float) -> tuple[float, float]:
    """The parabola's lower and upper edge values of the middle cell of five (Colella & Woodward
    1984, eqs. 1.6, 1.8 and 1.10): the oracle's PPM, which has no reference counterpart."""
    lo, hi = C.c_double(), C.c_double()
    load().orc_ppm_edges(a2m, am, a, ap, a2p, C.byref(lo), C.byref(hi))
    return lo.value, hi.value


def exact_riemann(left, right, gamma: float, xi) -> np.ndarray:
    """riemann_exact.ts exactRiemann(L, R, gamma)(xi) for each xi: rows (rho, u, p)."""
    xi = np.ascontiguousarray(np.atleast_1d(xi), dtype=np.float64)
    out = np.empty((xi.size, 3), dtype=np.float64)
    load().orc_exact_riemann(left[0], left[1], left[2], right[0], right[1], right[2], gamma, xi.ctypes.data, xi.size,
                             out.ctypes.data)
    return out


class RefHydro:
    """hydro.ts RefHydro: float64 state U (7, ncell) = rho, mx, my, mz, E, e_int, rho s."""

    def __init__(self, n=(128, 1, 1), dx=None, gamma=1.4, bc_lo=(1, 0, 0), bc_hi=(1, 0, 0), cfl=0.8, rho_floor=1e-10,
                 p_floor=1e-12, eta_dual=1e-3, shock_thresh=0.5, riemann="hllc", limiter="mc", isentropic=False,
                 signal_dims=3, threads=1):
        self._lib = load()
        n = (list(n) + [1, 1])[:3]
        c = orc_config()
        c.n[:] = [int(v) for v in n]
        c.dx = float(dx if dx is not None else 1.0 / n[0])
        c.gamma = float(gamma)
        c.bc_lo[:] = [int(b) for b in bc_lo]
        c.bc_hi[:] = [int(b) for b in bc_hi]
        c.cfl, c.rho_floor, c.p_floor = float(cfl), float(rho_floor), float(p_floor)
        c.eta_dual, c.shock_thresh = float(eta_dual), float(shock_thresh)
        c.riemann = RIEMANN[riemann]
        c.recon = RECON[limiter]
        c.isentropic = 1 if isentropic else 0
        c.signal_dims = int(signal_dims)
        self.cfg = c
        self.n = tuple(n)
        self.ncell = n[0] * n[1] * n[2]
        self._h = self._lib.orc_create(C.byref(c))
        self._lib.orc_set_threads(self._h, int(threads))

    def __del__(self):
        if getattr(self, "_h", None):
            self._lib.orc_destroy(self._h)
            self._h = None

    def set_threads(self, n: int):
        self._lib.orc_set_threads(self._h, int(n))

    def init_prims(self, prims: np.ndarray):
        """hydro.ts:195-214 init from (ncell, 6) primitives (rho, vx, vy, vz, p, s)."""
        prims = np.ascontiguousarray(prims, dtype=np.float64).reshape(self.ncell, 6)
        self._lib.orc_init_prims(self._h, prims.ctypes.data)

    def init(self, fn):
        """hydro.ts init(fn): fn(x, y, z) -> (rho, vx, vy, vz, p, s) at cell centres, box centred on 0."""
        nx, ny, nz = self.n
        dx = self.cfg.dx
        out = np.empty((self.ncell, 6))
        o = 0
        for k in range(nz):
            for j in range(ny):
                for i in range(nx):
                    out[o] = fn((i + 0.5 - nx / 2) * dx, (j + 0.5 - ny / 2) * dx, (k + 0.5 - nz / 2) * dx)
                    o += 1
        self.init_prims(out)

    @property
    def U(self) -> np.ndarray:
        u = np.empty((7, self.ncell), dtype=np.float64)
        self._lib.orc_get_conserved(self._h, u.ctypes.data)
        return u

    @U.setter
    def U(self, u: np.ndarray):
        u = np.ascontiguousarray(u, dtype=np.float64).reshape(7, self.ncell)
        self._lib.orc_set_conserved(self._h, u.ctypes.data)

    def set_state32(self, u1: np.ndarray, u2: np.ndarray):
        """Load the float32 GPU layout (u1 = rho, m; u2 = E, e_int, rho s, solid) as float64."""
        u = np.empty((7, self.ncell))
        u[0:4] = np.asarray(u1, dtype=np.float64).reshape(-1, 4).T
        u[4:7] = np.asarray(u2, dtype=np.float64).reshape(-1, 4).T[0:3]
        self.U = u

    def step(self, t_end: float = math.inf) -> float:
        return self._lib.orc_step(self._h, t_end)

    def run(self, t_end: float, max_steps: int = 100000):
        self._lib.orc_run(self._h, t_end, max_steps)

    @property
    def t(self) -> float:
        return self._lib.orc_time(self._h)

    @property
    def dt(self) -> float:
        return self._lib.orc_dt(self._h)

    @property
    def steps(self) -> int:
        return self._lib.orc_steps(self._h)

    def set_clock(self, t: float, steps: int = 0):
        self._lib.orc_set_clock(self._h, t, steps)
