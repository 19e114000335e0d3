"""The host block tree against the reference's own tree tests, tests/unit/tree.test.ts, case by
case (same trees, budgets and thresholds). The reference ships no golden tables; its pins are
these properties plus the concrete slots and codes the individual cases assert.

Every case is ported, including the index-grid boxes that changed between reads and a change of
boundaries after the tree was built.
"""
import math

import numpy as np
import pytest

from shaderous_b200.tree import (BT_STRIDE, FLAG_LEAF, MAX_AMR_LEVELS, NB_COARSE, RG_COPY, RG_PROLONG, RG_RESTRICT,
                                 BlockTree, TreeError)

PERIODIC = (0, 0, 0)
OUTFLOW = (1, 1, 1)


def blocks(t):
    """slot -> (level, c, parent, children) from the block table."""
    tab = t.table()
    out = {}
    for s in range(t.cap):
        if tab[s, 4] & 1:
            ch = [int(x) for x in tab[s, 12:12 + (1 << t.ndim)] if x >= 0]
            out[s] = (int(tab[s, 0]), tuple(int(x) for x in tab[s, 1:4]), int(tab[s, 5]), ch)
    return out


def slot_of(t, level, c):
    for s, (lv, cc, _, _) in blocks(t).items():
        if lv == level and cc[:t.ndim] == tuple(c)[:t.ndim]:
            return s
    return None


def balanced(t):
    """Every leaf's face neighbours lie at most one level away; children know their parent."""
    bl = blocks(t)
    for s, (lv, c, par, ch) in bl.items():
        if not ch:
            for f in range(t.nface):
                t.neighbor(lv, c, f)  # raises if a region is two levels coarser
        for x in ch:
            assert bl[x][2] == s


def covers(t):
    """The leaves tile the domain exactly once."""
    g = t.index_grid()
    m = t.nr << t.max_level
    assert g.size == m ** t.ndim
    counts = np.bincount(g.astype(np.int64), minlength=t.cap)
    for s, (lv, c, par, ch) in blocks(t).items():
        if not ch:
            assert counts[s] == (1 << (t.max_level - lv)) ** t.ndim


def indicator(t, fn):
    """Per-slot indicator array from fn(level, c), evaluated leaf by leaf coarsest first (the
    order adapt() asks its indicator in)."""
    ind = np.zeros(t.cap)
    for slot, lv, c in t.leaves():
        ind[slot] = fn(lv, c)
    return ind


def test_nests_to_deepest_level():
    assert MAX_AMR_LEVELS == 7
    for ndim, nr in [(2, 2), (3, 1)]:
        L = MAX_AMR_LEVELS
        t = BlockTree(ndim, nr, L, 4000, OUTFLOW, OUTFLOW)
        p = [0.3, 0.6, 0.45]

        def f(level, c):
            size = 1 / (nr << level)
            for i in range(ndim):
                if p[i] < c[i] * size or p[i] >= (c[i] + 1) * size:
                    return 0.0
            return 1.0

        for _ in range(L + 2):
            t.adapt(indicator(t, f), 0.6, 0.2)
        assert t.stats()["deepest"] == L
        balanced(t)
        covers(t)


def test_replays_a_remesh_slot_for_slot():
    for ndim, cap, edge in [(2, 100, False), (2, 400, True), (3, 300, True)]:
        make = lambda: BlockTree(ndim, 2, 4 if ndim == 2 else 3, cap, PERIODIC, PERIODIC, edge)
        a, b = make(), make()
        seed = [12345]

        def rand():
            seed[0] = (seed[0] * 1103515245 + 12345) % 2 ** 32
            return seed[0] / 2 ** 32

        evictions = 0
        for rnd in range(25):
            p = [0.3 + 0.02 * rnd, 0.5, 0.5]

            def f(level, c):
                size = 1 / (2 << level)
                d2 = 0.0
                for i in range(ndim):
                    lo = c[i] * size
                    d2 += max(0.0, lo - p[i], p[i] - lo - size) ** 2
                return math.exp(-d2 / 0.003) + 0.3 * rand()

            ops_a = a.adapt(indicator(a, f), 0.6, 0.2)
            steps = a.last_steps
            evictions += sum(1 for s in steps if s[0] == 1)
            ops_b = b.replay(steps)
            assert (ops_a is None) == (ops_b is None)
            if ops_a is not None:
                assert np.array_equal(ops_a, ops_b)
            assert b.last_steps == steps
            assert np.array_equal(a.table(), b.table())
        assert a.stats()["blocks"] > (40 if ndim == 2 else 60)
        if cap == 100:
            assert evictions > 0
        balanced(b)
    t = BlockTree(2, 2, 3, 100, PERIODIC, PERIODIC)
    with pytest.raises(TreeError, match="does not have"):
        t.replay([[0, 3, 5, 5]])


def test_tables_equal_for_equal_remeshes():
    for ndim, bc in [(2, PERIODIC), (2, (1, 2, 0)), (3, PERIODIC), (3, OUTFLOW)]:
        make = lambda: BlockTree(ndim, 2, 4 if ndim == 2 else 3, 3000, bc, bc)
        a, b = make(), make()
        seed = [7]

        def rnd():
            seed[0] = (seed[0] * 16807) % 2147483647
            return seed[0] / 2147483647

        for _ in range(10):
            ind = np.array([rnd() * 1.2 for _ in range(3000)])
            a.adapt(ind, 0.8, 0.3)
            b.adapt(ind, 0.8, 0.3)
            a.table()
            a.index_grid()
        assert np.array_equal(a.table(), b.table())
        assert np.array_equal(a.index_grid(), b.index_grid())
        covers(a)
        # A change of boundaries reaches the table read after it: b2 takes the same re-meshes under
        # the old boundaries and is switched only before its table is read.
        flipped = tuple(0 if x else 1 for x in bc)
        a.set_bc(flipped, bc)
        b2 = make()
        seed2 = [7]

        def rnd2():
            seed2[0] = (seed2[0] * 16807) % 2147483647
            return seed2[0] / 2147483647

        for _ in range(10):
            ind = np.array([rnd2() * 1.2 for _ in range(3000)])
            b2.set_bc(bc, bc)
            b2.adapt(ind, 0.8, 0.3)
        b2.set_bc(flipped, bc)
        assert np.array_equal(a.table(), b2.table())
        # and the boundary codes in it are the new ones (-1 - type at a lower face of the domain)
        t = a.table()
        for s, lv, c in a.leaves():
            for axis in range(ndim):
                if c[axis] == 0 and flipped[axis] != 0:
                    assert t[s, 6 + 2 * axis] == -1 - flipped[axis]


def test_reports_the_index_grid_boxes_that_changed():
    """A copy updated only inside the reported boxes, as the GPU texture is, stays equal; and not
    every re-mesh re-sends the whole grid (tree.test.ts 'reports the index-grid boxes that
    changed')."""
    for ndim in (2, 3):
        t = BlockTree(ndim, 2, 4 if ndim == 2 else 3, 3000, PERIODIC, PERIODIC)
        m = t.nr << t.max_level
        mz = m if ndim == 3 else 1
        copy = np.zeros((mz, m, m), np.uint32)
        seed = [11]

        def rnd():
            seed[0] = (seed[0] * 16807) % 2147483647
            return seed[0] / 2147483647

        partial = 0
        for rnd_i in range(12):
            if rnd_i:
                ind = np.array([rnd() * 1.2 for _ in range(3000)])
                t.adapt(ind, 0.8, 0.3)
            g, boxes = t.index_grid_boxes()
            g3 = g.reshape(mz, m, m)
            cells = 0
            for o, sz in boxes:
                cells += sz[0] * sz[1] * sz[2]
                # each box packed on its own, as gridBox packs it, then written at its origin
                data = g3[o[2]:o[2] + sz[2], o[1]:o[1] + sz[1], o[0]:o[0] + sz[0]].copy()
                assert data.size == sz[0] * sz[1] * sz[2]
                copy[o[2]:o[2] + sz[2], o[1]:o[1] + sz[1], o[0]:o[0] + sz[0]] = data
            if rnd_i and cells < g.size:
                partial += 1
            assert np.array_equal(copy.reshape(-1), g)
            assert np.array_equal(g, t.index_grid())
        assert partial > 0  # not every re-mesh re-sends the whole grid


def test_starts_as_uniform_root_grid():
    t = BlockTree(3, 2, 2, 64, PERIODIC, PERIODIC)
    assert t.stats()["blocks"] == 8 and t.stats()["leaves"] == 8
    covers(t)
    kind, slot = t.neighbor(0, (0, 0, 0), 0)
    assert kind == "same"
    assert blocks(t)[slot][1] == (1, 0, 0)  # wrapped


def test_reports_physical_boundaries():
    t = BlockTree(2, 2, 1, 16, OUTFLOW, (2, 3, 0))
    s = slot_of(t, 0, (1, 1))
    assert t.neighbor(0, (1, 1), 0)[0] == "same"
    assert t.neighbor(0, (1, 1), 1) == ("bc", 2)
    assert t.neighbor(0, (1, 1), 3) == ("bc", 3)
    tab = t.table()
    assert tab[s, 6 + 1] == -3
    assert tab[s, 6 + 3] == -4
    assert tab[s, 6 + 4] == s  # 2D: its own neighbour in z


def test_refines_keeping_balance():
    t = BlockTree(2, 4, 3, 400, OUTFLOW, OUTFLOW)
    lv, c = 0, (1, 1)
    for _ in range(3):
        assert t.refine(lv, c) > 0
        c = (2 * c[0] + 1, 2 * c[1] + 1)  # child 3 (x = 1, y = 1)
        lv += 1
        balanced(t)
        covers(t)
    assert t.stats()["deepest"] == 3
    s = slot_of(t, 0, (2, 1))
    assert blocks(t)[s][3]  # the block next to the level-1 parent had to split


def test_refuses_past_deepest_level_or_budget():
    t = BlockTree(3, 1, 1, 9, PERIODIC, PERIODIC)
    assert t.refine(0, (0, 0, 0)) == 1
    assert t.stats()["free"] == 0
    assert t.refine(1, (0, 0, 0)) == 0
    u = BlockTree(3, 2, 2, 12, PERIODIC, PERIODIC)
    assert u.refine(0, (0, 0, 0)) == 0
    assert u.stats()["blocks"] == 8


def test_records_coarse_neighbours_and_children():
    t = BlockTree(2, 2, 1, 16, OUTFLOW, OUTFLOW)
    p = slot_of(t, 0, (0, 0))
    t.refine(0, (0, 0))
    tab = t.table()
    kids = blocks(t)[p][3]
    ch = kids[1]  # x = 1, y = 0: its +x neighbour is the coarse block (1, 0)
    assert tab[ch, 0] == 1
    assert tab[ch, 4] & FLAG_LEAF == FLAG_LEAF
    assert tab[ch, 5] == p
    assert tab[ch, 6 + 1] == NB_COARSE
    assert tab[ch, 20 + 1] == slot_of(t, 0, (1, 0))
    assert tab[ch, 6 + 0] == kids[0]
    assert tab[p, 4] & FLAG_LEAF == 0
    assert list(tab[p, 12:16]) == kids
    assert tab[slot_of(t, 0, (1, 0)), 6 + 0] == p


def test_adapt_splits_merges_and_says_how_to_fill():
    t = BlockTree(2, 4, 2, 200, PERIODIC, PERIODIC)
    target = slot_of(t, 0, (2, 2))
    ind = np.zeros(200)
    ind[target] = 1
    ops = t.adapt(ind, 0.5, 0.1)
    assert ops is not None
    balanced(t)
    covers(t)
    kids = blocks(t)[target][3]
    for ch in kids:
        assert ops[ch, 0] == RG_PROLONG
    assert ops[kids[2], 1] == target and ops[kids[2], 2] == 2
    assert ops[slot_of(t, 0, (0, 0)), 0] == RG_COPY
    assert ops[target, 0] == 0  # parents hold no data
    ops = t.adapt(np.zeros(200), 0.5, 0.1)
    assert not blocks(t)[target][3]
    assert ops[target, 0] == RG_RESTRICT and list(ops[target, 4:8]) == kids
    assert t.stats()["blocks"] == 16
    assert t.adapt(np.zeros(200), 0.5, 0.1) is None


def test_no_merge_next_to_flagged_or_against_balance():
    t = BlockTree(2, 4, 2, 400, PERIODIC, PERIODIC)
    a = slot_of(t, 0, (1, 1))
    t.refine(0, (1, 1))
    a3 = blocks(t)[a][3][3]
    t.refine(1, blocks(t)[a3][1][:2])
    balanced(t)
    deep = blocks(t)[a3][3]
    ind = np.zeros(400)
    ind[deep] = 1
    t.adapt(ind, 2, 0.1)
    balanced(t)
    covers(t)
    assert blocks(t)[a][3]
    assert blocks(t)[a3][3]


def test_makes_room_by_merging_least_flagged():
    def make():
        t = BlockTree(2, 4, 1, 20, OUTFLOW, OUTFLOW)
        a = slot_of(t, 0, (0, 0))
        t.refine(0, (0, 0))
        assert t.stats()["free"] == 0
        return t, a, slot_of(t, 0, (3, 3))

    t, a, b = make()
    old = blocks(t)[a][3]
    ind = np.full(20, 0.3)
    ind[b] = 2
    ops = t.adapt(ind, 0.5, 0.1)
    assert not blocks(t)[a][3]
    assert blocks(t)[b][3]
    assert ops[a, 0] == RG_RESTRICT and list(ops[a, 4:8]) == old
    assert sorted(blocks(t)[b][3]) == sorted(old)
    for ch in blocks(t)[b][3]:
        assert ops[ch, 0] == RG_PROLONG and ops[ch, 1] == b
    balanced(t)
    covers(t)

    t, a, b = make()
    ind = np.full(20, 0.3)
    ind[b] = 2
    ind[blocks(t)[a][3]] = 3
    t.adapt(ind, 0.5, 0.1)
    assert blocks(t)[a][3]
    assert not blocks(t)[b][3]


def test_fills_every_new_block_from_old_data():
    seed = [7]

    def rand():
        seed[0] = (seed[0] * 1103515245 + 12345) % 2147483648
        return seed[0] / 2147483648

    for ndim, cap in [(2, 60), (3, 120)]:
        t = BlockTree(ndim, 4, 3, cap, OUTFLOW, OUTFLOW)
        for _ in range(60):
            leaves = {s for s, _, _ in t.leaves()}
            cx, cy = rand() * 4, rand() * 4

            def f(level, c):
                s = 1 / (1 << level)
                d = math.hypot((c[0] + 0.5) * s - cx, (c[1] + 0.5) * s - cy)
                return 2 / (0.3 + d) + rand()

            ops = t.adapt(indicator(t, f), 1.5, 0.5)
            balanced(t)
            covers(t)
            if ops is None:
                continue
            for s, _, _ in t.leaves():
                if ops[s, 0] in (RG_PROLONG, RG_COPY):
                    assert int(ops[s, 1]) in leaves
                if ops[s, 0] == RG_RESTRICT:
                    for ch in ops[s, 4:4 + (1 << ndim)]:
                        assert int(ch) in leaves


def test_lists_coarsest_first():
    t = BlockTree(3, 2, 1, 64, PERIODIC, PERIODIC)
    t.refine(0, (1, 1, 1))
    a, lv, per = t.lists()
    assert len(a) == 16 and len(lv) == 15
    tab = t.table()
    levels = [int(tab[s, 0]) for s in a]
    assert levels == sorted(levels)
    assert list(per) == [8, 8]


def _at_offset(t, by, lv, c, d):
    cc = list(c)
    for a in range(t.ndim):
        if not d[a]:
            continue
        n = t.nr << lv
        v = cc[a] + d[a]
        if v < 0 or v >= n:
            return None  # these trees are periodic or outflow; outflow is closed
        cc[a] = v
    for l in range(lv, -1, -1):
        s = lv - l
        q = by.get((l, tuple(x >> s for x in cc[:t.ndim])))
        if q is not None:
            return q
    return None


def _worst(t, periodic):
    bl = blocks(t)
    by = {(v[0], v[1][:t.ndim]): s for s, v in bl.items()}
    diag = []
    for a in range(t.ndim):
        for b in range(a + 1, t.ndim):
            for sa in (-1, 1):
                for sb in (-1, 1):
                    d = [0, 0, 0]
                    d[a], d[b] = sa, sb
                    diag.append(d)
    w = 0
    for s, (lv, c, _, ch) in bl.items():
        if ch:
            continue
        for d in diag:
            cc = list(c)
            if periodic:
                n = t.nr << lv
                cc = [(cc[i] + d[i]) % n if i < t.ndim else cc[i] for i in range(3)]
                q = _at_offset(t, by, lv, cc, [0, 0, 0])
            else:
                q = _at_offset(t, by, lv, c, d)
            if q is not None and not bl[q][3]:
                w = max(w, lv - bl[q][0])
    return w


def test_edge_balance_within_one_level():
    for ndim, bc in [(2, PERIODIC), (2, OUTFLOW), (3, PERIODIC), (3, OUTFLOW)]:
        t = BlockTree(ndim, 2, 4 if ndim == 2 else 3, 4000, bc, bc, True)
        seed = [3]

        def rnd():
            seed[0] = (seed[0] * 16807) % 2147483647
            return seed[0] / 2147483647

        for _ in range(12):
            ind = np.array([rnd() * 1.2 for _ in range(4000)])
            t.adapt(ind, 0.85, 0.3)
            balanced(t)
            covers(t)
            assert _worst(t, bc == PERIODIC) <= 1


def test_edge_balance_is_needed():
    for ndim in (2, 3):
        res = []
        for edge in (False, True):
            t = BlockTree(ndim, 2, 3, 4000, PERIODIC, PERIODIC, edge)
            lv, c = 0, (0, 0, 0)
            for _ in range(3):
                t.refine(lv, c)
                lv, c = lv + 1, tuple(2 * x for x in c)
            res.append(_worst(t, True))
        assert res == [2, 1]
