"""Parity of the CUDA multi-source SSSP (xb_multi_sssp through the C ABI)
with the CPU oracle, which equals the reference's Ligra MultiSSSP
(tests/test_msssp_oracle.py).  Bar: distances bit-exact (float32)."""
import numpy as np
import pytest

import xbtrav
from oracle import oracle as O

pytestmark = pytest.mark.gpu

INF = np.float32(np.finfo(np.float32).max / 4)


def _csr(kind, scale_or_n, ef_or_m, seed):
    h = (xbtrav.HostCSR.rmat(scale_or_n, ef_or_m, seed=seed) if kind == "rmat"
         else xbtrav.HostCSR.er(scale_or_n, ef_or_m, seed=seed))
    ro, ci = h.arrays()
    h.close()
    return ro, ci


@pytest.mark.parametrize("graph", [("rmat", 12, 16), ("rmat", 14, 8), ("er", 20000, 15000)])
@pytest.mark.parametrize("wrange", [(1, 100), (1, 1), (0, 5)])
@pytest.mark.parametrize("k", [1, 64, 1000])
def test_distances_match_oracle(ctx, graph, wrange, k):
    ro, ci = _csr(*graph, seed=77)
    w = xbtrav.symmetric_weights(ro, ci, 13, *wrange)
    src = xbtrav.select_sources_csr(ro, 21, k)
    g = ctx.upload_arrays(ro, ci)
    g.set_weights(w)
    d, st = ctx.multi_sssp(g, src)
    np.testing.assert_array_equal(d, O.msssp(ro, ci, w, src))
    assert st["levels"] >= 1 and st["edges_scanned"] > 0
    g.close()


def test_device_buffers_and_duplicates(ctx):
    import torch

    ro, ci = _csr("rmat", 13, 16, seed=5)
    w = xbtrav.symmetric_weights(ro, ci, 2, 1, 30)
    src = np.array([3, 3, 17, 3, 900], np.int32)
    g = ctx.upload_arrays(ro, ci)
    g.set_weights(w)
    d, _ = ctx.multi_sssp(g, torch.from_numpy(src).cuda(), out="device")
    np.testing.assert_array_equal(d.cpu().numpy(), O.msssp(ro, ci, w, src))
    g.close()


def test_negative_cycle(ctx):
    ro = np.array([0, 1, 3, 4, 4], np.int64)
    ci = np.array([1, 0, 2, 1], np.int32)
    w = np.array([2, 2, -1, -1], np.int32)
    g = ctx.upload_arrays(ro, ci)
    g.set_weights(w)
    d, st = ctx.multi_sssp(g, np.array([0], np.int32))
    np.testing.assert_array_equal(d, np.full(4, -INF, np.float32))
    assert st["levels"] == 4
    g.close()


def test_unit_weights_equal_bfs_levels(ctx):
    # size-independent property at a full bench size: with every weight 1 the
    # distance is the smallest level over the sources of the traversal tables
    ro, ci = _csr("rmat", 18, 16, seed=101)
    src = xbtrav.select_sources_csr(ro, 8, 128)
    g = ctx.upload_arrays(ro, ci)
    r = ctx.traverse(g, src)
    g.set_weights(np.ones(g.m, np.int32))
    d, _ = ctx.multi_sssp(g, src)
    lv = np.where(r.level < 0, np.iinfo(np.int32).max, r.level).min(axis=0)
    want = np.where(lv == np.iinfo(np.int32).max, INF, lv.astype(np.float32))
    np.testing.assert_array_equal(d, want)
    # the traversal afterwards still sees a clean workspace
    r2 = ctx.traverse(g, src)
    np.testing.assert_array_equal(r2.level, r.level)
    np.testing.assert_array_equal(r2.parent, r.parent)
    g.close()


def test_errors(ctx):
    ro, ci = _csr("rmat", 8, 4, seed=1)
    g = ctx.upload_arrays(ro, ci)
    with pytest.raises(xbtrav.XbError):
        ctx.multi_sssp(g, np.array([0], np.int32))  # no weights yet
    with pytest.raises(ValueError):
        g.set_weights(np.ones(g.m + 1, np.int32))
    g.set_weights(np.ones(g.m, np.int32))
    with pytest.raises(xbtrav.XbError):
        ctx.multi_sssp(g, np.array([g.n], np.int32))
    with pytest.raises(xbtrav.XbError):
        ctx.multi_sssp(g, np.array([], np.int32))
    g.close()


def test_edgeless_sources_and_small_graphs(ctx):
    # isolated sources (no edges) next to a path 1-2-3; and a one-vertex graph
    ro = np.array([0, 0, 1, 3, 4, 4], np.int64)
    ci = np.array([2, 1, 3, 2], np.int32)
    w = np.array([4, 4, 7, 7], np.int32)
    g = ctx.upload_arrays(ro, ci)
    g.set_weights(w)
    for src in ([0], [4, 0], [0, 1], [3]):
        s = np.array(src, np.int32)
        d, _ = ctx.multi_sssp(g, s)
        np.testing.assert_array_equal(d, O.msssp(ro, ci, w, s))
    g.close()
    g1 = ctx.upload_arrays(np.array([0, 0], np.int64), np.zeros(0, np.int32))
    g1.set_weights(np.zeros(0, np.int32))
    d, st = ctx.multi_sssp(g1, np.array([0], np.int32))
    np.testing.assert_array_equal(d, np.zeros(1, np.float32))
    assert st["levels"] == 1
    g1.close()
