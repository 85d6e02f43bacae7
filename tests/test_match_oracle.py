"""The maximum-matching restatement (oracle_max_match, Edmonds' blossom
algorithm) pinned three ways on the CPU: exhaustive search on small graphs,
scipy's bipartite matching on bipartite graphs, and the reference's own CPU
matching engine (apps/xb/src/xblsm_cpu/par_pro_pernode.cu, compiled into
oracle/_ref) on R-MAT, uniform and blossom-rich graphs."""
import functools

import numpy as np
import pytest

import xbtrav
from oracle import oracle as O


def _csr(n, pairs):
    """Symmetric sorted CSR without self-loops or duplicates."""
    s = set()
    for a, b in pairs:
        if a != b:
            s.add((a, b))
            s.add((b, a))
    deg = np.zeros(n + 1, np.int64)
    e = sorted(s)
    for a, _ in e:
        deg[a + 1] += 1
    return np.cumsum(deg), np.array([b for _, b in e], np.int32)


def _exhaustive(n, ro, ci):
    adj = [set(ci[ro[v]:ro[v + 1]].tolist()) for v in range(n)]

    @functools.lru_cache(maxsize=None)
    def best(mask):
        if mask == 0:
            return 0
        v = (mask & -mask).bit_length() - 1
        rest = mask & ~(1 << v)
        r = best(rest)
        for u in adj[v]:
            if rest >> u & 1:
                r = max(r, 1 + best(rest & ~(1 << u)))
        return r

    return best((1 << n) - 1)


def _random_pairs(rng, n, p):
    return [(a, b) for a in range(n) for b in range(a + 1, n) if rng.random() < p]


@pytest.mark.parametrize("seed", range(40))
def test_oracle_equals_exhaustive(seed):
    rng = np.random.default_rng(seed)
    n = int(rng.integers(2, 13))
    ro, ci = _csr(n, _random_pairs(rng, n, float(rng.uniform(0.15, 0.7))))
    size, mate = O.max_match(ro, ci)
    assert O.check_matching(ro, ci, mate) == 0
    assert size == _exhaustive(n, ro, ci)


NAMED = {
    # odd cycles, nested blossoms, a blossom hanging off a path, Petersen (perfect)
    "triangle+pendant": (4, [(0, 1), (1, 2), (2, 0), (2, 3)]),
    "pentagon+tails": (9, [(0, 1), (1, 2), (2, 3), (3, 4), (4, 0), (0, 5), (2, 6), (6, 7), (3, 8)]),
    "flower": (11, [(0, 1), (1, 2), (2, 0), (2, 3), (3, 4), (4, 2), (4, 5), (5, 6), (6, 4),
                    (0, 7), (7, 8), (6, 9), (9, 10)]),
    "petersen": (10, [(0, 1), (1, 2), (2, 3), (3, 4), (4, 0), (0, 5), (1, 6), (2, 7), (3, 8), (4, 9),
                      (5, 7), (7, 9), (9, 6), (6, 8), (8, 5)]),
    "path7": (7, [(i, i + 1) for i in range(6)]),
}


@pytest.mark.parametrize("name", sorted(NAMED))
def test_named_graphs(name):
    n, pairs = NAMED[name]
    ro, ci = _csr(n, pairs)
    for init in (None, "greedy-bad"):
        start = None
        if init:  # a poor maximal start that forces augmentations through blossoms
            start = np.full(n, -1, np.int32)
            for a, b in pairs[::-1]:
                if start[a] < 0 and start[b] < 0:
                    start[a], start[b] = b, a
        size, mate = O.max_match(ro, ci, init=start)
        assert O.check_matching(ro, ci, mate) == 0
        assert size == _exhaustive(n, ro, ci)


def test_bipartite_equals_scipy():
    from scipy.sparse import csr_matrix
    from scipy.sparse.csgraph import maximum_bipartite_matching

    rng = np.random.default_rng(5)
    for _ in range(10):
        a, b = int(rng.integers(50, 400)), int(rng.integers(50, 400))
        k = int(rng.integers(a, 4 * a))
        pairs = {(int(x), int(y)) for x, y in zip(rng.integers(0, a, k), rng.integers(0, b, k))}
        bip = csr_matrix((np.ones(len(pairs)), ([p[0] for p in pairs], [p[1] for p in pairs])), shape=(a, b))
        want = int((maximum_bipartite_matching(bip, perm_type="column") >= 0).sum())
        ro, ci = _csr(a + b, [(x, a + y) for x, y in pairs])
        size, mate = O.max_match(ro, ci)
        assert O.check_matching(ro, ci, mate) == 0
        assert size == want


@pytest.mark.skipif(not O.ref_match_available(), reason="reference matching engine not built")
@pytest.mark.parametrize("graph", ["rmat10", "rmat12", "rmat14_ef4", "er", "dense300"])
def test_oracle_size_equals_reference(graph):
    if graph.startswith("rmat"):
        scale = int(graph[4:6])
        h = xbtrav.HostCSR.rmat(scale, 4 if "ef4" in graph else 16, seed=17)
        ro, ci = h.arrays()
        h.close()
    elif graph == "er":
        h = xbtrav.HostCSR.er(20000, 16000, seed=17)
        ro, ci = h.arrays()
        h.close()
    else:  # dense random graph: many odd cycles
        rng = np.random.default_rng(17)
        ro, ci = _csr(301, _random_pairs(rng, 301, 0.02))
    size, mate = O.max_match(ro, ci)
    rsize, rmate = O.ref_max_match(ro, ci, threads=4)
    assert O.check_matching(ro, ci, mate) == 0 and O.check_matching(ro, ci, rmate) == 0
    assert size == rsize
