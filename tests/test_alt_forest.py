"""xb_traverse in XB_MODE_ALTERNATING (the alternating forest of a matching,
the expansion of the reference's alternating mode): the oracle's rule on
hand-checked cases and structural properties (CPU), and the CUDA result
bit-exact against it (GPU)."""
import numpy as np
import pytest

import xbtrav
from oracle import oracle as O

from test_match_oracle import _csr, _random_pairs


def _greedy(n, ro, ci, order):
    mate = np.full(n, -1, np.int32)
    for v in order:
        if mate[v] >= 0:
            continue
        for w in ci[ro[v]:ro[v + 1]]:
            if mate[w] < 0 and w != v:
                mate[v], mate[w] = w, v
                break
    return mate


def _check_structure(ro, ci, mate, lv, pr, ow):
    n = len(ro) - 1
    for v in range(n):
        if lv[v] < 0:
            assert pr[v] == -1 and ow[v] == -1
            continue
        if lv[v] == 0:
            assert mate[v] < 0 and pr[v] == v and ow[v] == v
        elif lv[v] % 2 == 1:  # inner: parent is an adjacent outer vertex one level up
            p = pr[v]
            assert lv[p] == lv[v] - 1 and p in set(ci[ro[v]:ro[v + 1]].tolist()) and ow[v] == ow[p]
            assert lv[mate[v]] == lv[v] + 1 and pr[mate[v]] == v
        else:  # outer: parent is its mate
            assert pr[v] == mate[v] and lv[mate[v]] == lv[v] - 1 and ow[v] == ow[mate[v]]
    # complete: no outer vertex has an unlabeled matched neighbour
    for v in range(n):
        if lv[v] >= 0 and lv[v] % 2 == 0:
            for w in ci[ro[v]:ro[v + 1]]:
                assert not (lv[w] < 0 and mate[w] >= 0)


def test_oracle_hand_cases():
    # path 0 - 1 = 2 - 3 = 4 (= matched), 0 exposed
    ro, ci = _csr(5, [(0, 1), (1, 2), (2, 3), (3, 4)])
    mate = np.array([-1, 2, 1, 4, 3], np.int32)
    lv, pr, ow, rounds = O.alt_forest(ro, ci, mate)
    assert lv.tolist() == [0, 1, 2, 3, 4] and pr.tolist() == [0, 0, 1, 2, 3] and ow.tolist() == [0] * 5
    assert rounds == 3
    # triangle 0-1-2 with 1 = 2 matched: both ends qualify; the smaller id is inner
    ro, ci = _csr(3, [(0, 1), (1, 2), (0, 2)])
    lv, pr, ow, _ = O.alt_forest(ro, ci, np.array([-1, 2, 1], np.int32))
    assert lv.tolist() == [0, 1, 2] and pr.tolist() == [0, 0, 1]
    # two roots compete for one pair: the smaller root claims it
    ro, ci = _csr(4, [(0, 2), (1, 3), (2, 3)])
    lv, pr, ow, _ = O.alt_forest(ro, ci, np.array([-1, -1, 3, 2], np.int32))
    assert lv.tolist() == [0, 0, 1, 2] and pr.tolist() == [0, 1, 0, 2] and ow.tolist() == [0, 1, 0, 0]


@pytest.mark.parametrize("seed", range(12))
def test_oracle_structure(seed):
    rng = np.random.default_rng(300 + seed)
    n = int(rng.integers(5, 300))
    ro, ci = _csr(n, _random_pairs(rng, n, float(rng.uniform(0.01, 0.2))))
    mate = _greedy(n, ro, ci, rng.permutation(n))
    lv, pr, ow, _ = O.alt_forest(ro, ci, mate)
    _check_structure(ro, ci, mate, lv, pr, ow)


def _gpu_case(ctx, ro, ci, mate):
    g = ctx.upload_arrays(ro, ci)
    lv, pr, ow, st = ctx.alternating_forest(g, mate)
    g.close()
    wl, wp, wo, rounds = O.alt_forest(ro, ci, mate)
    np.testing.assert_array_equal(lv, wl)
    np.testing.assert_array_equal(pr, wp)
    np.testing.assert_array_equal(ow, wo)
    assert st["levels"] == rounds and st["reached"] == int((wl >= 0).sum())


@pytest.mark.gpu
@pytest.mark.parametrize("seed", range(12))
def test_gpu_random_graphs(ctx, seed):
    rng = np.random.default_rng(500 + seed)
    n = int(rng.integers(5, 400))
    ro, ci = _csr(n, _random_pairs(rng, n, float(rng.uniform(0.01, 0.2))))
    _gpu_case(ctx, ro, ci, _greedy(n, ro, ci, rng.permutation(n)))


@pytest.mark.gpu
@pytest.mark.parametrize("scale,ef", [(14, 8), (16, 16)])
def test_gpu_rmat(ctx, scale, ef):
    h = xbtrav.HostCSR.rmat(scale, ef, seed=77)
    ro, ci = h.arrays()
    h.close()
    n = len(ro) - 1
    rng = np.random.default_rng(scale)
    _gpu_case(ctx, ro, ci, _greedy(n, ro, ci, rng.permutation(n)))  # a maximal matching
    g = ctx.upload_arrays(ro, ci)
    mate, _ = ctx.max_match(g)  # a maximum matching: the forest is Hungarian (no outer-outer edges across trees)
    g.close()
    _gpu_case(ctx, ro, ci, mate)


@pytest.mark.gpu
def test_gpu_device_buffers_and_errors(ctx):
    import torch

    ro, ci = _csr(5, [(0, 1), (1, 2), (2, 3), (3, 4)])
    g = ctx.upload_arrays(ro, ci)
    lv, pr, ow, _ = ctx.alternating_forest(g, torch.tensor([-1, 2, 1, 4, 3], dtype=torch.int32, device="cuda"))
    assert lv.cpu().tolist() == [0, 1, 2, 3, 4] and pr.cpu().tolist() == [0, 0, 1, 2, 3]
    with pytest.raises(xbtrav.XbError):
        ctx.alternating_forest(g, np.array([-1, 3, -1, 1, -1], np.int32))  # 1-3 is not an edge
    with pytest.raises(xbtrav.XbError):
        ctx.alternating_forest(g, np.array([-1, 2, -1, -1, -1], np.int32))  # not symmetric
    g.close()
