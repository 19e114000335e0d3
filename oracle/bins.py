"""ORACLE — test infrastructure only (tests/). A numpy restatement of the reference's per-block
timestep bins over a block table (32 ints per slot, the reference's BlockTree.table layout:
word 0 level, 4 flags with bit 2 = leaf, 6..11 face neighbours, 12..19 children, 20..25 the
coarser leaf beyond a face whose entry is -1):

- ``bins_init``   src/amr/bins_init.wgsl:17-35, the first guess of each block's bin;
- ``bins_relax``  src/amr/bins_relax.wgsl:24-61, one sweep (DILATE for the first), face
  neighbours only (EDGES off: hydro without a magnetic field);
- ``cycle_bins``  the sequence src/amr/amr_sim.ts:1556-1570 (setBins) runs: init, one dilation
  sweep, then (K + levels + 2) | 1 relaxation sweeps;
- ``substep_lists`` src/amr/bins_lists.wgsl:52-78 with ``faster_neighbor`` :27-51, the blocks a
  substep assembles (LA), predicts (LL) and updates (LU), deposits included.

Floor of the logarithm in bins_init: taken as the largest k with 2^k <= dtb / dt (the
mathematical definition; float32 divisions rounded to nearest as IEEE 754 defines them).
"""
from __future__ import annotations

import numpy as np

BTS = 32


def _leaf(bt: np.ndarray, slot: int) -> bool:
    return (int(bt[slot, 4]) & 2) != 0


def bins_init(bt: np.ndarray, blocks, rates: np.ndarray, dt: float, cfl: float, kmax: int, out: np.ndarray) -> None:
    """bins_init.wgsl: k = clamp(floor(log2(dtb / dt)), 0, KMAX), dtb = cfl / max(rate, 1e-30) in
    float32, for leaves while the clock moves; KMAX otherwise."""
    dt32 = np.float32(dt)
    for slot in blocks:
        k = kmax
        if _leaf(bt, slot) and dt32 > 0:
            dtb = np.float32(np.float32(cfl) / max(np.float32(rates[slot]), np.float32(1e-30)))
            x = np.float32(dtb / dt32)
            k = 0
            while k < kmax and x >= np.float32(2 << k):
                k += 1
        out[1 + slot] = k


def bins_relax(bt: np.ndarray, blocks, ndim: int, kmax: int, dilate: bool, kin: np.ndarray, kout: np.ndarray) -> None:
    """bins_relax.wgsl: a parent takes its fastest child; a leaf is at most one bin slower than a
    same-level face neighbour (none slower in the dilation sweep) and no slower than a coarser one."""
    for slot in blocks:
        k = int(kin[1 + slot])
        if not _leaf(bt, slot):
            k = kmax
            for ch in range(8):
                c = int(bt[slot, 12 + ch])
                if c >= 0:
                    k = min(k, int(kin[1 + c]))
        else:
            for f in range(2 * ndim):
                nb = int(bt[slot, 6 + f])
                if nb >= 0 and nb != slot:
                    k = min(k, int(kin[1 + nb]) + (0 if dilate else 1))
                elif nb == -1:
                    k = min(k, int(kin[1 + int(bt[slot, 20 + f])]))
        kout[1 + slot] = k


def cycle_bins(bt: np.ndarray, blocks, ndim: int, levels: int, rates: np.ndarray, dt: float, cfl: float,
               kmax: int) -> np.ndarray:
    """The bins of a cycle (amr_sim.ts setBins): init into A, dilate A -> B, then an odd number of
    relaxation sweeps alternating B -> A, A -> B, so that the result lands in A."""
    cap = bt.shape[0]
    a = np.zeros(cap + 1, np.int64)
    b = np.zeros(cap + 1, np.int64)
    bins_init(bt, blocks, rates, dt, cfl, kmax, a)
    bins_relax(bt, blocks, ndim, kmax, True, a, b)
    sweeps = (kmax + levels + 2) | 1
    for i in range(sweeps):
        if i % 2 == 0:
            bins_relax(bt, blocks, ndim, kmax, False, b, a)
        else:
            bins_relax(bt, blocks, ndim, kmax, False, a, b)
    return a


def faster_neighbor(bt: np.ndarray, kb: np.ndarray, slot: int, ndim: int) -> bool:
    """bins_lists.wgsl faster_neighbor: a face neighbour leaf, or a child of a refined same-level
    neighbour on the shared face, in a faster bin."""
    k = int(kb[1 + slot])
    for f in range(2 * ndim):
        nb = int(bt[slot, 6 + f])
        if nb < 0 or nb == slot:
            continue
        if _leaf(bt, nb):
            if int(kb[1 + nb]) < k:
                return True
            continue
        axis, want = f >> 1, 1 - (f & 1)
        for ch in range(8):
            if ((ch >> axis) & 1) != want:
                continue
            c = int(bt[nb, 12 + ch])
            if c >= 0 and _leaf(bt, c) and int(kb[1 + c]) < k:
                return True
    return False


def substep_lists(bt: np.ndarray, blocks, kb: np.ndarray, s: int, ndim: int):
    """bins_lists.wgsl for substep s: (LA, LL, LU) as sets of slots."""
    la, ll, lu = set(), set(), set()
    for slot in blocks:
        k = int(kb[1 + slot])
        phase = s & ((1 << k) - 1)
        on = phase == 0
        leaf = _leaf(bt, slot)
        if on:
            la.add(slot)
        if on and leaf:
            ll.add(slot)
        half = k > 0 and phase == (1 << (k - 1))
        deposit = leaf and not on and half and faster_neighbor(bt, kb, slot, ndim)
        if leaf and (on or deposit):
            lu.add(slot)
    return la, ll, lu


def cycle_updates(bt: np.ndarray, blocks, kb: np.ndarray, kmax: int, ndim: int) -> int:
    """Block updates of one cycle: every leaf on its first substep, then the substeps' LU lists."""
    leaves = [s for s in blocks if _leaf(bt, s)]
    n = len(leaves)
    for s in range(1, 1 << kmax):
        n += len(substep_lists(bt, blocks, kb, s, ndim)[2])
    return n
