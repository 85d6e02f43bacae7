"""The multi-source SSSP restatement (oracle_msssp) against the reference's
Ligra MultiSSSP (apps/ligra/apps/MultiSSSP.C compiled into oracle/_ref) and
against a textbook Dijkstra on small graphs; CPU only."""
import heapq

import numpy as np
import pytest

import xbtrav
from oracle import oracle as O

INF = np.float32(np.finfo(np.float32).max / 4)


def _dijkstra(ro, ci, w, sources):
    n = len(ro) - 1
    d = np.full(n, np.inf)
    pq = []
    for s in set(int(x) for x in sources):
        d[s] = 0.0
        pq.append((0.0, s))
    heapq.heapify(pq)
    while pq:
        du, u = heapq.heappop(pq)
        if du > d[u]:
            continue
        for e in range(ro[u], ro[u + 1]):
            v = ci[e]
            if du + w[e] < d[v]:
                d[v] = du + w[e]
                heapq.heappush(pq, (d[v], v))
    return np.where(np.isinf(d), INF, d).astype(np.float32)


def _graph(kind, seed):
    if kind == "rmat":
        h = xbtrav.HostCSR.rmat(10, 8, seed=seed)
    else:
        h = xbtrav.HostCSR.er(3000, 2000, seed=seed)  # sparse: many unreached vertices
    ro, ci = h.arrays()
    h.close()
    return ro, ci


@pytest.mark.parametrize("kind", ["rmat", "er"])
@pytest.mark.parametrize("wrange", [(1, 100), (1, 1), (0, 3)])
def test_oracle_equals_dijkstra(kind, wrange):
    ro, ci = _graph(kind, 11)
    w = xbtrav.symmetric_weights(ro, ci, 5, *wrange)
    src = xbtrav.select_sources_csr(ro, 3, 7)
    np.testing.assert_array_equal(O.msssp(ro, ci, w, src), _dijkstra(ro, ci, w, src))


@pytest.mark.skipif(not O.ligra_msssp_available(), reason="reference Ligra MultiSSSP not built")
@pytest.mark.parametrize("kind", ["rmat", "er"])
@pytest.mark.parametrize("wrange", [(1, 100), (1, 10), (0, 0)])
@pytest.mark.parametrize("k", [1, 17])
def test_oracle_equals_reference(kind, wrange, k):
    ro, ci = _graph(kind, 29)
    w = xbtrav.symmetric_weights(ro, ci, 9, *wrange)
    src = xbtrav.select_sources_csr(ro, 4, k)
    np.testing.assert_array_equal(O.msssp(ro, ci, w, src), O.ligra_msssp(ro, ci, w, src))


@pytest.mark.skipif(not O.ligra_msssp_available(), reason="reference Ligra MultiSSSP not built")
def test_negative_weight_marks_everything():
    # an undirected edge of negative weight is a negative cycle: both give -FLT_MAX/4 everywhere
    ro = np.array([0, 1, 3, 4, 4], np.int64)
    ci = np.array([1, 0, 2, 1], np.int32)
    w = np.array([2, 2, -1, -1], np.int32)
    src = np.array([0], np.int32)
    want = np.full(4, -INF, np.float32)
    np.testing.assert_array_equal(O.msssp(ro, ci, w, src), want)
    np.testing.assert_array_equal(O.ligra_msssp(ro, ci, w, src), want)


def test_duplicate_sources_and_symmetry():
    ro, ci = _graph("rmat", 3)
    w = xbtrav.symmetric_weights(ro, ci, 1, 1, 50)
    # weights agree on both directions of every edge
    u = np.repeat(np.arange(len(ro) - 1), np.diff(ro))
    fwd = dict(zip(zip(u.tolist(), ci.tolist()), w.tolist()))
    assert all(fwd[(b, a)] == x for (a, b), x in fwd.items())
    src = np.array([5, 5, 9, 5], np.int32)
    np.testing.assert_array_equal(O.msssp(ro, ci, w, src), O.msssp(ro, ci, w, np.array([9, 5], np.int32)))
