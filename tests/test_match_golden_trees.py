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
blossom, which forces an augmenting path around the blossom.

The same trees also pin the alternating mode (xb_traverse with
XB_MODE_ALTERNATING): grown from the exposed vertex 0 over the tree edges
alone, each outer vertex x of ExpandTwoNodes(v, w, x) is labeled at the level
equal to the reference's root_distance[x] (the EXPECT_EQs at
path_table_test.cu:93-96, 149-156, 192-194, 224-227, 257-260), w at that
level minus one, with parent[w] = v, parent[x] = w and owner 0."""
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


# root_distance expectations of the reference test, per tree
ROOT_DISTANCE = {
    1: {0: 0, 2: 2, 4: 2, 6: 4},
    2: {0: 0, 2: 2, 4: 4, 6: 4, 8: 6, 10: 8, 12: 8, 18: 8},
    3: {0: 0, 2: 2, 4: 4},
    4: {0: 0, 2: 2, 4: 4, 6: 4},
    5: {0: 0, 2: 2, 4: 4, 6: 2},
}


def tree_only_case(t):
    """The tree of ExpandTwoNodes calls alone: edges v-w and w-x, matching
    w-x, vertex 0 the exposed root."""
    n, expands, _ = TREES[t]
    pairs = [(v, w) for v, w, _ in expands] + [(w, x) for _, w, x in expands]
    mate = np.full(n, -1, np.int32)
    for _, w, x in expands:
        mate[w], mate[x] = x, w
    ro, ci = _csr(n, pairs)
    return n, ro, ci, mate


def _check_root_distances(t, level, parent, owner):
    for x, d in ROOT_DISTANCE[t].items():
        assert level[x] == d, (t, x, level[x], d)
    for v, w, x in TREES[t][1]:
        assert level[w] == level[v] + 1 and level[x] == level[w] + 1, (t, v, w, x)
        assert parent[w] == v and parent[x] == w, (t, v, w, x)
        assert owner[w] == 0 and owner[x] == 0
    assert level[0] == 0 and parent[0] == 0 and owner[0] == 0


@pytest.mark.parametrize("t", [1, 2, 3, 4, 5])
def test_oracle_alternating_forest_root_distances(t):
    n, ro, ci, mate = tree_only_case(t)
    level, parent, owner, _ = O.alt_forest(ro, ci, mate)
    _check_root_distances(t, level, parent, owner)


@pytest.mark.gpu
@pytest.mark.parametrize("t", [1, 2, 3, 4, 5])
def test_gpu_alternating_forest_root_distances(ctx, t):
    n, ro, ci, mate = tree_only_case(t)
    g = ctx.upload_arrays(ro, ci)
    level, parent, owner, _ = ctx.alternating_forest(g, mate)
    g.close()
    _check_root_distances(t, level, parent, owner)
    lv_o, pr_o, ow_o, _ = O.alt_forest(ro, ci, mate)
    np.testing.assert_array_equal(level, lv_o)
    np.testing.assert_array_equal(parent, pr_o)
    np.testing.assert_array_equal(owner, ow_o)


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
