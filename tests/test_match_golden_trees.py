"""The reference's path-table golden trees (apps/xb/test/device/path_table_test.cu:80-272)
restated as matching cases.

Each tree is grown there by ExpandTwoNodes(v, w, x): an unmatched edge v-w and
the matched edge w-x.  Here the same trees become graphs with those matched
edges as the initial matching, plus the blossom edges the reference test
contracts (FindAndAddBlossomImplicit(a, b) -> edge a-b) and, for tree 1, the
edge 6-7 its AddAugmentingPath(6, 7) flips.  Tree 1's flip result is pinned
exactly (the reference test's EXPECT_EQs; that maximum matching is unique).
Trees 2-5 have one exposed vertex, so their matching is already maximum;
each is also run with a pendant exposed vertex on an inner vertex of a
blossom, which forces an augmenting path around the blossom.  The
reference's root distances belong to its path-table layout, which this
engine does not keep (its forest stores pred / blossom base instead)."""
import numpy as np
import pytest

from oracle import oracle as O

from test_match_oracle import _csr

TREES = {
    1: (8, [(0, 1, 2), (0, 3, 4), (4, 5, 6)], [(6, 7)]),
    2: (19, [(0, 1, 2), (2, 3, 4), (2, 5, 6), (4, 7, 8), (8, 9, 10), (8, 11, 12), (6, 13, 14), (6, 15, 16),
             (16, 17, 18)], [(10, 12), (14, 18), (11, 17)]),
    3: (5, [(0, 1, 2), (2, 3, 4)], [(0, 4)]),
    4: (7, [(0, 1, 2), (2, 3, 4), (2, 5, 6)], [(4, 6)]),
    5: (7, [(0, 1, 2), (2, 3, 4), (0, 5, 6)], [(4, 6)]),
}
# an inner vertex of a blossom of each tree, for the pendant variant
PENDANT_AT = {2: 9, 3: 3, 4: 5, 5: 3}
# tree 1 after AddAugmentingPath(6, 7): the reference test's expectations
GOLDEN_1 = {0: 3, 3: 0, 1: 2, 2: 1, 4: 5, 5: 4, 6: 7, 7: 6}


def tree_case(t, pendant=False):
    n, expands, extra = TREES[t]
    pairs, mate = [], None
    pairs += [(v, w) for v, w, _ in expands] + [(w, x) for _, w, x in expands] + list(extra)
    if pendant:
        pairs.append((PENDANT_AT[t], n))
        n += 1
    mate = np.full(n, -1, np.int32)
    for _, w, x in expands:
        mate[w], mate[x] = x, w
    ro, ci = _csr(n, pairs)
    return n, ro, ci, mate


def _check_golden_1(mate):
    for v, m in GOLDEN_1.items():
        assert mate[v] == m, (v, mate[v], m)


def test_oracle_tree1_golden():
    n, ro, ci, mate = tree_case(1)
    size, out = O.max_match(ro, ci, init=mate)
    assert size == 4
    _check_golden_1(out)


@pytest.mark.parametrize("t", [2, 3, 4, 5])
@pytest.mark.parametrize("pendant", [False, True])
def test_oracle_blossom_trees(t, pendant):
    n, ro, ci, mate = tree_case(t, pendant)
    start = int((mate >= 0).sum()) // 2
    size, out = O.max_match(ro, ci, init=mate)
    assert O.check_matching(ro, ci, out) == 0
    assert size == start + (1 if pendant else 0)


@pytest.mark.gpu
def test_gpu_tree1_golden(ctx):
    n, ro, ci, mate = tree_case(1)
    g = ctx.upload_arrays(ro, ci)
    out, st = ctx.max_match(g, init=mate)
    g.close()
    assert st["reached"] == 4
    _check_golden_1(out)


@pytest.mark.gpu
@pytest.mark.parametrize("t", [2, 3, 4, 5])
@pytest.mark.parametrize("pendant", [False, True])
def test_gpu_blossom_trees(ctx, t, pendant):
    n, ro, ci, mate = tree_case(t, pendant)
    g = ctx.upload_arrays(ro, ci)
    out, st = ctx.max_match(g, init=mate)
    g.close()
    assert O.check_matching(ro, ci, out) == 0
    want, oracle_mate = O.max_match(ro, ci, init=mate)
    assert st["reached"] == want
    if not pendant:  # no augmenting path: the matching is returned as given
        np.testing.assert_array_equal(out, mate)
