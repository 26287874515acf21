"""The level-order numbering behind the simulation step's octree build, checked
on the host against the oracle's reference-numbered octree.

The step's build (lo_span_kernel, lo_tile_scan_kernel, lo_rank_kernel and
lo_upsweep_kernel in csrc/build.cu) never builds the reference's radix tree:
it numbers the octree's cells straight from the sorted unique keys with
closed formulas.  This file restates those formulas in numpy -- the common
levels delta of neighbouring keys, the leaf level lambda, the cells a group
starts and ends, each cell's level-order index, parent and first child, its
depth-first preorder index, and the count-free last-arrival test of the
upward pass -- and checks them against the octree the oracle builds in the
reference's own stages (leaf groups, Karras tree, plan, materialisation):
same cells at every level, same parents, same preorder.  The GPU tests
(tests/test_gpu_level_order.py) then hold the kernels to the reference-
numbered build bit for bit; this one pins the arithmetic they rely on.
"""
import numpy as np
import pytest

KEY_BITS = 30
LEVELS = KEY_BITS // 3
ARRIVED = 1 << 31


def _prefix(key, level):
    return int(key) >> (KEY_BITS - 3 * level)


def _common_levels(a, b):
    c = 0
    for level in range(1, LEVELS + 1):
        if _prefix(a, level) != _prefix(b, level):
            break
        c = level
    return c


def _level_order(uniq):
    """Cells per level, parents, first children and preorder indices from the
    sorted unique keys alone (the formulas of lo_span / lo_rank)."""
    g_count = len(uniq)
    delta = [-1] + [_common_levels(uniq[g - 1], uniq[g]) for g in range(1, g_count)] + [-1]
    lam = [1 + max(0, delta[g], delta[g + 1]) for g in range(g_count)]
    started = [range(delta[g] + 1, lam[g] + 1) for g in range(g_count)]
    per_level = np.zeros(LEVELS + 3, np.int64)
    for g in range(g_count):
        for level in started[g]:
            per_level[level] += 1
    base = np.concatenate([[0], np.cumsum(per_level)])
    m = int(base[LEVELS + 1])
    # S(g): cells added by the groups >= g (group g ends its cells at levels (delta_{g+1}, lambda_g])
    ends = [lam[g] - delta[g + 1] for g in range(g_count)]
    s_from = np.concatenate([np.cumsum(ends[::-1])[::-1], [0]])
    cell_prefix = np.zeros(m, np.int64)
    cell_level = np.zeros(m, np.int64)
    parent = np.full(m, -1, np.int64)
    first_child = np.zeros(m, np.int64)
    preorder = np.full(m, -1, np.int64)
    excl = np.zeros(LEVELS + 3, np.int64)  # cells started per level by the groups before g
    for g in range(g_count):
        for level in started[g]:
            b = int(base[level] + excl[level])
            cell_prefix[b] = _prefix(uniq[g], level)
            cell_level[b] = level
            first_child[b] = base[level + 1] + excl[level + 1]
            if level > 0:
                # g's own cell one level up, or (one below the common levels)
                # the last cell started before g at level delta_g
                parent[b] = base[level - 1] + excl[level - 1] - (1 if level - 1 == delta[g] else 0)
        for level in range(delta[g + 1] + 1, lam[g] + 1):
            # the cell at this level whose last group is g
            b = int(base[level] + excl[level] + (1 if level in started[g] else 0) - 1)
            preorder[b] = s_from[g] - lam[g] + level - 1
        for level in started[g]:
            excl[level] += 1
    return dict(m=m, base=base, prefix=cell_prefix, level=cell_level, parent=parent,
                first_child=first_child, preorder=preorder, lam=lam)


def _oracle_preorder(oc):
    """Depth-first preorder of the oracle's octree, children visited octant 7 -> 0."""
    m = oc["nNodes"]
    kids = oc["children"].reshape(m, 8)
    order = np.full(m, -1, np.int64)
    stack, nxt = [0], 0
    while stack:
        node = stack.pop()
        order[node] = nxt
        nxt += 1
        ch = [int(c) for c in kids[node] if c >= 0]
        ch.sort(key=lambda c: int(oc["prefix"][c]))  # ascending octant; the stack pops the last first
        stack.extend(ch)
    return order


def _keys(case, rng):
    if case == "uniform":
        return rng.integers(0, 1 << KEY_BITS, 3000)
    if case == "clustered":
        centres = rng.integers(0, 1 << KEY_BITS, 12)
        return np.concatenate([c ^ rng.integers(0, 1 << rng.integers(3, 18), 300) for c in centres])
    if case == "duplicates":
        pts = rng.integers(0, 1 << KEY_BITS, 40)
        return pts[rng.integers(0, 40, 2000)]
    if case == "deep_pairs":
        base = rng.integers(0, 1 << (KEY_BITS - 1), 200) << 1
        return np.concatenate([base, base | 1])
    if case == "single":
        return np.array([12345])
    raise KeyError(case)


@pytest.mark.parametrize("case", ["uniform", "clustered", "duplicates", "deep_pairs", "single"])
def test_level_order_numbering_matches_reference_octree(oracle, case):
    rng = np.random.default_rng(np.random.Philox(17))
    keys = np.sort(_keys(case, rng).astype(np.uint32) & np.uint32((1 << KEY_BITS) - 1))
    ref = oracle.octree_from_keys(keys)
    oc = ref["octree"]
    uniq = [int(k) for k in ref["groups"][0]]
    lo = _level_order(uniq)
    m = oc["nNodes"]
    assert lo["m"] == m
    # the same cells at every level; level-order index = rank of the prefix in its level
    shift = KEY_BITS - 3 * oc["level"].astype(np.int64)
    ref_prefix = oc["prefix"].astype(np.int64) >> shift
    key_of = {(int(l), int(p)): i for i, (l, p) in enumerate(zip(oc["level"], ref_prefix))}
    to_lo = np.full(m, -1, np.int64)
    for b in range(m):
        node = key_of[(int(lo["level"][b]), int(lo["prefix"][b]))]
        to_lo[node] = b
    assert (to_lo >= 0).all()
    for level in range(LEVELS + 1):
        cells = lo["prefix"][lo["base"][level]:lo["base"][level + 1]]
        assert (np.diff(cells) > 0).all()  # each level in ascending key order
    # parents, first children and child counts
    ref_parent = oc["parent"]
    for node in range(m):
        b = to_lo[node]
        want = -1 if ref_parent[node] < 0 else to_lo[ref_parent[node]]
        assert lo["parent"][b] == want
    kids = oc["children"].reshape(m, 8)
    for node in range(m):
        b = to_lo[node]
        ch = sorted(to_lo[c] for c in kids[node] if c >= 0)
        level = lo["level"][b]
        nxt = lo["first_child"][b + 1] if b + 1 < lo["base"][level + 1] else lo["base"][level + 2]
        assert ch == list(range(lo["first_child"][b], nxt))
    # preorder (children octant 7 -> 0), as the walks' records are laid out
    pre = _oracle_preorder(oc)
    assert (lo["preorder"][to_lo] == pre).all()
    # every group's leaf sits at level lambda and holds the group's particles
    for g, key in enumerate(uniq):
        node = key_of[(lo["lam"][g], _prefix(key, lo["lam"][g]))]
        assert oc["particleCount"][node] > 0


def test_count_free_last_arrival():
    """Child c of the cells [c0, c1) adds 1, plus c if first, plus 2^31 - (c + 1)
    if last: the 32-bit counter reaches 2^31 exactly at the last arrival, in
    any arrival order, and never exceeds it."""
    rng = np.random.default_rng(np.random.Philox(5))
    for _ in range(5000):
        c0 = int(rng.integers(0, 1 << 30))
        nk = int(rng.integers(1, 9))
        order = rng.permutation(nk) + c0
        total = 0
        for i, c in enumerate(order):
            add = 1 + (c if c == c0 else 0) + (ARRIVED - (c + 1) if c == c0 + nk - 1 else 0)
            total = (total + add) & 0xFFFFFFFF
            assert total <= ARRIVED
            assert (total == ARRIVED) == (i == nk - 1)
