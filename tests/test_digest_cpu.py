"""The serving digest (xb_row_digest) on the CPU side: its row hash is the
restated splitmix64 finalizer of each (vertex, level, parent) entry, summed
mod 2^64, and it notices a parent moved from one vertex to another (which the
sums of levels and parents alone would not)."""
import numpy as np

import xbtrav
from oracle import oracle as O

MASK = (1 << 64) - 1


def _entry_hash_py(v: int, level: int, parent: int) -> int:
    z = (v * 0x9E3779B97F4A7C15) & MASK
    z ^= ((level & 0xFFFFFFFF) << 32) | (parent & 0xFFFFFFFF)
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & MASK
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & MASK
    return z ^ (z >> 31)


def test_entry_hash_matches_the_integer_restatement():
    rng = np.random.default_rng(3)
    v = rng.integers(0, 1 << 33, 200)
    lv = rng.integers(0, 1 << 20, 200).astype(np.int32)
    pr = rng.integers(-1, 1 << 31, 200).astype(np.int64).astype(np.int32)
    got = O.row_entry_hash(v, lv, pr)
    for i in range(200):
        assert int(got[i]) == _entry_hash_py(int(v[i]), int(lv[i]), int(pr[i]))


def test_digest_sees_a_parent_swap_that_sums_miss():
    ro, ci = xbtrav.HostCSR.rmat(10, 8, seed=17).arrays()
    src = xbtrav.select_sources_csr(ro, 18, 4)
    lv, pr, _, _ = O.msbfs(ro, ci, src)
    base = O.row_digests(lv, pr)
    row = 0
    # two vertices at one level with different parents: swap their parents
    L = lv[row]
    for d in range(2, int(L.max()) + 1):
        at = np.nonzero(L == d)[0]
        pairs = [(a, b) for a in at[:50] for b in at[:50] if a < b and pr[row, a] != pr[row, b]]
        if pairs:
            a, b = pairs[0]
            break
    else:
        raise AssertionError("no swappable pair in the fixture")
    mut = pr.copy()
    mut[row, a], mut[row, b] = pr[row, b], pr[row, a]
    after = O.row_digests(lv, mut)
    assert after[row, 0] == base[row, 0] and after[row, 1] == base[row, 1] and after[row, 3] == base[row, 3]
    assert after[row, 2] != base[row, 2]
    # the old parent sum would not have changed
    m = L >= 0
    assert pr[row][m].astype(np.int64).sum() == mut[row][m].astype(np.int64).sum()
    np.testing.assert_array_equal(after[1:], base[1:])
