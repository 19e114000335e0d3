"""Python view of the host block tree (the reference's BlockTree, src/amr/tree.ts) over the C ABI.

The tree itself is C++ (``csrc/amr_tree.cpp``); this wrapper exposes the calls the reference's
own tree tests make (tests/unit/tree.test.ts), with tables as numpy arrays.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._abi import load

BS = 16
BT_STRIDE = 32
RG_STRIDE = 12
NB_COARSE = -1
FLAG_ACTIVE, FLAG_LEAF = 1, 2
RG_NONE, RG_COPY, RG_PROLONG, RG_RESTRICT = 0, 1, 2, 3
ADAPT_REFINE, ADAPT_EVICT, ADAPT_MERGE = 0, 1, 2
MAX_AMR_LEVELS = 7


class TreeError(RuntimeError):
    pass


def _i3(v):
    v = list(v) + [0, 0, 0]
    return (C.c_int32 * 3)(*[int(x) for x in v[:3]])


class BlockTree:
    def __init__(self, ndim: int, nr: int, max_level: int, cap: int, bc_lo=(0, 0, 0), bc_hi=(0, 0, 0), edge_balance=False):
        self._lib = load()
        self.ndim, self.nr, self.max_level, self.cap = ndim, nr, max_level, cap
        self.nface = 2 * ndim
        h = C.c_void_p()
        self._ok(self._lib.shz_tree_create(ndim, nr, max_level, cap, _i3(bc_lo), _i3(bc_hi), 1 if edge_balance else 0,
                                           C.byref(h)))
        self._h = h
        self._bc = (tuple(bc_lo), tuple(bc_hi))

    def _ok(self, rc):
        if rc != 0:
            raise TreeError(self._lib.shz_tree_error().decode())

    def __del__(self):
        if getattr(self, "_h", None):
            self._lib.shz_tree_destroy(self._h)
            self._h = None

    # -- re-meshing ----------------------------------------------------------------------------
    def adapt(self, indicator_by_slot, hi: float, lo: float):
        """adapt((b) => ind[b.slot], hi, lo): regrid table (cap, 12) or None if nothing changed."""
        ind = np.ascontiguousarray(np.asarray(indicator_by_slot, dtype=np.float64))
        assert ind.size >= self.cap
        rg = np.zeros((self.cap, RG_STRIDE), dtype=np.int32)
        ch = C.c_int32()
        self._ok(self._lib.shz_tree_adapt(self._h, ind.ctypes.data, hi, lo, rg.ctypes.data, C.byref(ch)))
        return rg if ch.value else None

    @property
    def last_steps(self):
        n = C.c_int32()
        self._ok(self._lib.shz_tree_last_steps(self._h, None, 0, C.byref(n)))
        buf = np.zeros(max(n.value, 1), dtype=np.int32)
        self._ok(self._lib.shz_tree_last_steps(self._h, buf.ctypes.data, buf.size, C.byref(n)))
        w = 2 + self.ndim
        return [list(map(int, buf[i:i + w])) for i in range(0, n.value, w)]

    def replay(self, steps):
        flat = np.asarray([v for s in steps for v in s], dtype=np.int32)
        rg = np.zeros((self.cap, RG_STRIDE), dtype=np.int32)
        ch = C.c_int32()
        self._ok(self._lib.shz_tree_replay(self._h, flat.ctypes.data if flat.size else None, flat.size, rg.ctypes.data,
                                           C.byref(ch)))
        return rg if ch.value else None

    def refine(self, level: int, c) -> int:
        n = C.c_int32()
        self._ok(self._lib.shz_tree_refine(self._h, level, _i3(c), C.byref(n)))
        return n.value

    def neighbor(self, level: int, c, f: int):
        """('same'|'coarse', slot) or ('bc', type)."""
        k, v = C.c_int32(), C.c_int32()
        self._ok(self._lib.shz_tree_neighbor(self._h, level, _i3(c), f, C.byref(k), C.byref(v)))
        return (("same", "coarse", "bc")[k.value], v.value)

    # -- tables ----------------------------------------------------------------------------------
    def table(self) -> np.ndarray:
        t = np.zeros((self.cap, BT_STRIDE), dtype=np.int32)
        self._ok(self._lib.shz_tree_table(self._h, t.ctypes.data))
        return t

    def lists(self):
        a = np.zeros(self.cap, dtype=np.int32)
        lv = np.zeros(self.cap, dtype=np.int32)
        per = np.zeros(self.max_level + 1, dtype=np.int32)
        na, nl = C.c_int32(), C.c_int32()
        self._ok(self._lib.shz_tree_lists(self._h, a.ctypes.data, lv.ctypes.data, per.ctypes.data, C.byref(na),
                                          C.byref(nl)))
        return a[:na.value].copy(), lv[:nl.value].copy(), per

    def index_grid(self) -> np.ndarray:
        n = self._lib.shz_tree_index_grid_size(self._h)
        g = np.zeros(n, dtype=np.uint32)
        self._ok(self._lib.shz_tree_index_grid(self._h, g.ctypes.data))
        return g

    def index_grid_boxes(self):
        """indexGrid(boxes): the grid and the boxes (origin, size) that changed since the last call."""
        n = self._lib.shz_tree_index_grid_size(self._h)
        g = np.zeros(n, dtype=np.uint32)
        cap = 4096
        bx = np.zeros((cap, 6), dtype=np.int32)
        k = C.c_int32()
        self._ok(self._lib.shz_tree_index_grid_boxes(self._h, g.ctypes.data, bx.ctypes.data, cap, C.byref(k)))
        assert k.value <= cap
        return g, [(tuple(map(int, b[:3])), tuple(map(int, b[3:]))) for b in bx[:k.value]]

    def set_bc(self, bc_lo, bc_hi):
        """The bcLo / bcHi setters: boundary types of a built tree (tree.ts:193-199)."""
        self._ok(self._lib.shz_tree_set_bc(self._h, _i3(bc_lo), _i3(bc_hi)))
        self._bc = (tuple(bc_lo), tuple(bc_hi))

    def stats(self) -> dict:
        v = [C.c_int32() for _ in range(5)]
        self._ok(self._lib.shz_tree_stats(self._h, *[C.byref(x) for x in v]))
        return dict(zip(["blocks", "free", "leaves", "deepest", "high_slot"], [x.value for x in v]))

    # -- convenience -------------------------------------------------------------------------------
    def leaves(self):
        """(slot, level, c) of every leaf, coarsest first."""
        t = self.table()
        _, lv, _ = self.lists()
        return [(int(s), int(t[s, 0]), tuple(int(x) for x in t[s, 1:4])) for s in lv]
