"""ORACLE — test infrastructure only (tests/). ctypes wrapper of the block-grid oracle in
``oracle/liboracle.so`` (``oracle/amr_ref.cpp``): a float64 restatement of one step of the
reference's block grid (src/amr: assemble, predict, update with fine-flux matching, the Löhner
flag and the regrid fill) on a block table and a state the caller gives.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from .oracle import RECON, RIEMANN, load

BS = 16
BT_STRIDE = 32
RG_STRIDE = 12


class oamr_params(C.Structure):
    _fields_ = [
        ("ndim", C.c_int32),
        ("nr", C.c_int32),
        ("cap", C.c_int32),
        ("dx0", C.c_double),
        ("gamma", C.c_double),
        ("rho_floor", C.c_double),
        ("p_floor", C.c_double),
        ("eta_dual", C.c_double),
        ("shock_thresh", C.c_double),
        ("riemann", C.c_int32),
        ("recon", C.c_int32),
        ("isentropic", C.c_int32),
        ("signal_dims", C.c_int32),
    ]


_bound = False


def _lib():
    global _bound
    lib = load()
    if not _bound:
        P = C.c_void_p
        lib.oamr_create.restype = P
        lib.oamr_create.argtypes = [C.POINTER(oamr_params)]
        lib.oamr_destroy.argtypes = [P]
        lib.oamr_set_threads.argtypes = [P, C.c_int]
        lib.oamr_set_table.argtypes = [P, P]
        lib.oamr_set_state.argtypes = [P, C.c_int32, P, P, P]
        lib.oamr_get_state.argtypes = [P, C.c_int32, P, P]
        lib.oamr_assemble.restype = C.c_double
        lib.oamr_assemble.argtypes = [P, C.c_int32, P]
        lib.oamr_get_prims.argtypes = [P, C.c_int32, P]
        lib.oamr_step.argtypes = [P, C.c_int32, P, C.c_double]
        lib.oamr_get_halfsteps.argtypes = [P, C.c_int32, P]
        lib.oamr_flags.argtypes = [P, C.c_int32, P, P]
        lib.oamr_regrid.argtypes = [P, P, P, C.c_int32, P]
        _bound = True
    return lib


def _i32(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.int32)


class AmrOracle:
    """The block grid of one run: `table` (cap x 32 ints, the reference's BlockTree table) and the
    leaves' state, in float64. Slots index blocks as the table does."""

    def __init__(self, ndim: int, nr: int, cap: int, dx0: float, gamma: float, recon: str = "mc",
                 isentropic: bool = False, riemann: str = "hllc", rho_floor: float = 1e-10, p_floor: float = 1e-12,
                 eta_dual: float = 1e-3, shock_thresh: float = 0.5, signal_dims: int = 3, threads: int = 4):
        self._l = _lib()
        p = oamr_params(ndim, nr, cap, dx0, gamma, rho_floor, p_floor, eta_dual, shock_thresh, RIEMANN[riemann],
                        RECON[recon], 1 if isentropic else 0, signal_dims)
        self.ndim, self.cap = ndim, cap
        self.cells = BS ** ndim
        self.texels = (BS + 4) ** ndim
        self.half_texels = (BS + 2) ** ndim
        self._h = self._l.oamr_create(C.byref(p))
        if not self._h:
            raise ValueError("the block-grid oracle refused its parameters")
        self._l.oamr_set_threads(self._h, int(threads))

    def __del__(self):
        if getattr(self, "_h", None):
            self._l.oamr_destroy(self._h)
            self._h = None

    def set_table(self, table: np.ndarray) -> None:
        t = _i32(table).reshape(-1)
        assert t.size == self.cap * BT_STRIDE
        self._table = t
        self._l.oamr_set_table(self._h, t.ctypes.data)

    def set_state(self, slots, u1: np.ndarray, u2: np.ndarray) -> None:
        """u1, u2: float32 (len(slots) x 16^ndim x 4), the blocks in the order of `slots`."""
        s = _i32(slots)
        a = np.ascontiguousarray(u1, np.float32).reshape(s.size * self.cells, 4)
        b = np.ascontiguousarray(u2, np.float32).reshape(s.size * self.cells, 4)
        self._l.oamr_set_state(self._h, s.size, s.ctypes.data, a.ctypes.data, b.ctypes.data)

    def state(self, slots) -> np.ndarray:
        """float64 (len(slots), 16^ndim, 8): u1 then u2 per cell."""
        s = _i32(slots)
        out = np.empty((s.size, self.cells, 8))
        self._l.oamr_get_state(self._h, s.size, s.ctypes.data, out.ctypes.data)
        return out

    def assemble(self, blocks) -> float:
        """Primitives of every listed block; returns the leaves' largest rate per unit cell size."""
        s = _i32(blocks)
        return float(self._l.oamr_assemble(self._h, s.size, s.ctypes.data))

    def prims(self, slot: int) -> np.ndarray:
        """(20^ndim, 7): rho, vx, vy, vz, p, s, cs per texel, x fastest; NaN where unwritten."""
        out = np.empty((self.texels, 7))
        self._l.oamr_get_prims(self._h, int(slot), out.ctypes.data)
        return out

    def step(self, leaves, dt: float) -> None:
        s = _i32(leaves)
        self._l.oamr_step(self._h, s.size, s.ctypes.data, float(dt))

    def halfsteps(self, slot: int) -> np.ndarray:
        out = np.empty((self.half_texels, 8))
        self._l.oamr_get_halfsteps(self._h, int(slot), out.ctypes.data)
        return out

    def flags(self, leaves) -> np.ndarray:
        s = _i32(leaves)
        out = np.empty(s.size)
        self._l.oamr_flags(self._h, s.size, s.ctypes.data, out.ctypes.data)
        return out

    def regrid(self, new_table: np.ndarray, rg: np.ndarray, new_leaves) -> None:
        t = _i32(new_table).reshape(-1)
        r = _i32(rg).reshape(-1)
        s = _i32(new_leaves)
        assert t.size == self.cap * BT_STRIDE and r.size == self.cap * RG_STRIDE
        self._l.oamr_regrid(self._h, t.ctypes.data, r.ctypes.data, s.size, s.ctypes.data)
        self._table = t
