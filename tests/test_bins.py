"""The per-block timesteps' bin rules (src/amr/bins_relax.wgsl:1-9, bins_lists.wgsl:1-8), checked on
the oracle's restatement over refined trees built by the host block tree: after a cycle's sweeps
face neighbours are at most one bin apart, no leaf is slower than a coarser neighbour, a parent is
its fastest child, and every leaf half way through its step beside a faster one takes a deposit."""
import numpy as np
import pytest

from oracle import bins as ob
from shaderous_b200.tree import BlockTree

LEAF = 2


def refined_tree(ndim):
    t = BlockTree(ndim, 4 if ndim == 2 else 2, 3, 2000, (1, 1, 1), (1, 1, 1))
    # a refined corner region three levels deep, so that bins differ by level and by rate
    t.refine(0, (0, 0, 0))
    t.refine(1, (0, 0, 0))
    t.refine(1, (1, 0, 0))
    t.refine(2, (1, 1, 0))
    t.refine(2, (0, 0, 0))
    t.refine(3 - 1, (1, 0, 0))
    return t


def used(tab):
    return [s for s in range(tab.shape[0]) if tab[s, 4] & 1]


def rates_for(tab, blocks, seed):
    rng = np.random.default_rng(seed)
    r = np.zeros(tab.shape[0], np.float32)
    for s in blocks:
        if tab[s, 4] & LEAF:
            # a rate per unit cell size: finer blocks and a few hot spots are faster
            r[s] = np.float32((1 << int(tab[s, 0])) * (1.0 + 9.0 * rng.random() ** 4))
    return r


@pytest.mark.parametrize("ndim,seed,K", [(2, 1, 3), (2, 2, 3), (3, 3, 3), (2, 4, 1), (2, 5, 5), (3, 6, 2), (3, 7, 5)])
def test_relaxed_bins_obey_the_rules(ndim, seed, K):
    t = refined_tree(ndim)
    tab = t.table()
    blocks = used(tab)
    levels, cfl = 3, 0.8
    r = rates_for(tab, blocks, seed)
    dt = cfl / float(r.max())
    kb = ob.cycle_bins(tab, blocks, ndim, levels, r, dt, cfl, K)
    first = np.zeros_like(kb)
    ob.bins_init(tab, blocks, r, dt, cfl, K, first)
    leaves = [s for s in blocks if tab[s, 4] & LEAF]
    assert len(set(int(kb[1 + s]) for s in leaves)) >= min(3, K + 1), "the case exercises several bins"
    for s in blocks:
        k = int(kb[1 + s])
        assert 0 <= k <= K
        if not tab[s, 4] & LEAF:
            kids = [int(c) for c in tab[s, 12:20] if c >= 0]
            assert k == min(int(kb[1 + c]) for c in kids)
            continue
        assert k <= first[1 + s]  # relaxation only ever speeds a block up
        for f in range(2 * ndim):
            nb = int(tab[s, 6 + f])
            if nb >= 0 and nb != s:
                assert k <= kb[1 + nb] + 1
                if tab[nb, 4] & LEAF:
                    assert abs(k - int(kb[1 + nb])) <= 1
            elif nb == -1:
                assert k <= kb[1 + int(tab[s, 20 + f])]
    # deposits: a leaf with a faster same-level leaf neighbour is updated at its own midpoint
    for s in leaves:
        k = int(kb[1 + s])
        if k == 0:
            continue
        fast = any(int(tab[s, 6 + f]) >= 0 and tab[int(tab[s, 6 + f]), 4] & LEAF and
                   kb[1 + int(tab[s, 6 + f])] < k for f in range(2 * ndim))
        _, _, lu = ob.substep_lists(tab, blocks, kb, 1 << (k - 1), ndim)
        assert (s in lu) == ob.faster_neighbor(tab, kb, s, ndim)
        if fast:
            assert s in lu
    upd = ob.cycle_updates(tab, blocks, kb, K, ndim)
    assert len(leaves) < upd < len(leaves) << K


def test_first_guess_is_the_floor_of_the_logarithm():
    t = BlockTree(2, 2, 0, 8, (0, 0, 0), (0, 0, 0))
    tab = t.table()
    blocks = used(tab)
    cfl, dt = np.float32(0.5), 0.5 / 8.0
    # dtb / dt = 8 / rate: rates 8, 4.0001, 4, 1 give 1, 1.99998, 2, 8 -> bins 0, 0, 1, 3
    r = np.zeros(tab.shape[0], np.float32)
    for s, v in zip(blocks, (8.0, 4.0001, 4.0, 1.0)):
        r[s] = v
    out = np.zeros(tab.shape[0] + 1, np.int64)
    ob.bins_init(tab, blocks, r, dt, float(cfl), 5, out)
    assert [int(out[1 + s]) for s in blocks] == [0, 0, 1, 3]
    ob.bins_init(tab, blocks, r, dt, float(cfl), 2, out)
    assert [int(out[1 + s]) for s in blocks] == [0, 0, 1, 2]
    ob.bins_init(tab, blocks, r, 0.0, float(cfl), 2, out)  # a held clock: the slowest bin
    assert [int(out[1 + s]) for s in blocks] == [2, 2, 2, 2]
