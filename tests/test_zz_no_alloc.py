"""xb_traverse_noalloc: the traversal entry point for callers that may not
allocate device memory (a plugin whose host owns the GPU's memory through its
own pool, or a latency-critical path that forbids cudaMalloc/cudaFree and
their device synchronisation).  It keeps its working state in a fixed array
compiled into the library, so it must give the same tables as xb_traverse
call after call, although every call reuses what the previous one left in
that array.

This file is collected last on purpose: it runs after every other test, and
also passes when run alone in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

import xbtrav

pytestmark = pytest.mark.gpu

MAX_N = 131072  # XB_NOALLOC_MAX_VERTICES


def _noalloc():
    f = xbtrav.lib().xb_traverse_noalloc
    f.restype = C.c_int32
    f.argtypes = [C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p,
                  C.POINTER(xbtrav.XbStats)]
    return f


def _call(ro_d, ci_d, src_d, level_d, parent_d, n, k, stats=None, stream=None):
    """One call through the C ABI; stream is a torch.cuda.Stream (None: the
    legacy default stream)."""
    import torch

    torch.cuda.synchronize()
    st = stats if stats is not None else xbtrav.XbStats()
    handle = C.c_void_p(stream.cuda_stream) if stream is not None else None
    rc = _noalloc()(n, ro_d.data_ptr(), ci_d.data_ptr() if ci_d.numel() else None, src_d.data_ptr(), k,
                    level_d.data_ptr(), parent_d.data_ptr(), handle, C.byref(st))
    torch.cuda.synchronize()
    return rc, st


def _device_inputs(ro, ci, src):
    import torch

    dev = torch.device("cuda", 0)
    n, k = len(ro) - 1, len(src)
    return (torch.from_numpy(ro.astype(np.int32)).to(dev), torch.from_numpy(ci.astype(np.int32)).to(dev),
            torch.from_numpy(np.ascontiguousarray(src, np.int32)).to(dev),
            torch.full((k, n), -7, dtype=torch.int32, device=dev),
            torch.full((k, n), -7, dtype=torch.int32, device=dev))


def _csr_from_edges(n, edges):
    """Symmetric, sorted, duplicate-free CSR of an undirected edge list."""
    a = np.array(edges, np.int64)
    u = np.concatenate([a[:, 0], a[:, 1]])
    v = np.concatenate([a[:, 1], a[:, 0]])
    key = np.unique(u * n + v)
    u, v = key // n, key % n
    ro = np.zeros(n + 1, np.int64)
    np.add.at(ro, u + 1, 1)
    return np.cumsum(ro), v.astype(np.int32)


def test_noalloc_matches_xb_traverse_two_calls_in_a_row():
    import torch

    ctx = xbtrav.Context(0)
    ctx.set_tuning(word_bits=64, words=1, pull_alpha=4.0, heavy_degree=2048, timing=0)
    # two different graphs and source sets: the second call must not see the first's leftovers
    cases = []
    for scale, ef, seed, k in ((14, 16, 41, 100), (12, 8, 42, 70)):
        csr = xbtrav.HostCSR.rmat(scale, ef, seed=seed)
        ro, ci = csr.arrays()
        src = xbtrav.select_sources_csr(ro, seed + 1, k)
        g = ctx.upload(csr)
        ref = ctx.traverse(g, src)  # existing entry point
        g.close()
        cases.append((ro, ci, src, ref))
    for ro, ci, src, ref in cases + cases[:1]:
        n, k = len(ro) - 1, len(src)
        dev = torch.device("cuda", 0)
        ro_d = torch.from_numpy(ro.astype(np.int32)).to(dev)
        ci_d = torch.from_numpy(ci).to(dev)
        src_d = torch.from_numpy(src).to(dev)
        lv_d = torch.full((k, n), -7, dtype=torch.int32, device=dev)
        pr_d = torch.full((k, n), -7, dtype=torch.int32, device=dev)
        rc, st = _call(ro_d, ci_d, src_d, lv_d, pr_d, n, k)
        assert rc == xbtrav.XB_OK, xbtrav.lib().xb_last_error()
        np.testing.assert_array_equal(lv_d.cpu().numpy(), ref.level)
        np.testing.assert_array_equal(pr_d.cpu().numpy(), ref.parent)
        assert st.edges_traversed == ref.stats["edges_traversed"]
    ctx.close()


def test_noalloc_rejects_graphs_above_its_capacity_and_bad_ids():
    import torch

    dev = torch.device("cuda", 0)
    n = MAX_N + 1
    ro_d = torch.zeros(n + 1, dtype=torch.int32, device=dev)
    ci_d = torch.zeros(1, dtype=torch.int32, device=dev)
    src_d = torch.zeros(1, dtype=torch.int32, device=dev)
    out = torch.zeros(1, dtype=torch.int32, device=dev)
    rc, _ = _call(ro_d, ci_d, src_d, out, out, n, 1)
    assert rc == xbtrav.XB_ERR_CAPACITY
    assert b"131072" in xbtrav.lib().xb_last_error()
    # a source id outside the graph is reported, not traversed
    ro = torch.tensor([0, 1, 2], dtype=torch.int32, device=dev)
    ci = torch.tensor([1, 0], dtype=torch.int32, device=dev)
    bad = torch.tensor([5], dtype=torch.int32, device=dev)
    tab = torch.zeros(2, dtype=torch.int32, device=dev)
    rc, _ = _call(ro, ci, bad, tab, tab, 2, 1)
    assert rc == xbtrav.XB_ERR_ARG


def test_noalloc_at_its_maximum_size_on_a_side_stream_matches_the_oracle():
    """A graph of exactly XB_NOALLOC_MAX_VERTICES vertices (R-MAT scale 17),
    called on a stream of the caller's, checked against the CPU oracle
    directly; a second call with other sources follows on the same array."""
    import torch

    from oracle import oracle

    csr = xbtrav.HostCSR.rmat(17, 8, seed=77)
    ro, ci = csr.arrays()
    assert len(ro) - 1 == MAX_N
    stream = torch.cuda.Stream()
    for seed, k in ((78, 130), (79, 64)):
        src = xbtrav.select_sources_csr(ro, seed, k)
        ro_d, ci_d, src_d, lv_d, pr_d = _device_inputs(ro, ci, src)
        rc, st = _call(ro_d, ci_d, src_d, lv_d, pr_d, MAX_N, k, stream=stream)
        assert rc == xbtrav.XB_OK, xbtrav.lib().xb_last_error()
        lv, pr, edges, _ = oracle.msbfs(ro, ci, src)
        np.testing.assert_array_equal(lv_d.cpu().numpy(), lv)
        np.testing.assert_array_equal(pr_d.cpu().numpy(), pr)
        assert st.edges_traversed == edges


def test_noalloc_deep_traversal_uses_every_level_plane():
    """A long path with chords (depth in the thousands, so level planes 3 and
    up are cleared and decoded) and a few branches: bit-exact against the
    oracle and against xb_traverse, with the deep call between two shallow ones
    so the planes it leaves behind must not leak into the next call."""
    from oracle import oracle

    n = 6000
    edges = [(i, i + 1) for i in range(n - 1)]
    edges += [(i, i + 7) for i in range(0, n - 7, 997)]  # sparse chords
    edges += [(3, 4000), (2500, 5999)]
    ro, ci = _csr_from_edges(n, edges)
    src = np.array([0, 5999, 3000, 17, 4321], np.int32)
    shallow = xbtrav.HostCSR.rmat(12, 8, seed=5)
    sro, sci = shallow.arrays()
    ssrc = xbtrav.select_sources_csr(sro, 6, 64)
    for ro_, ci_, src_ in ((sro, sci, ssrc), (ro, ci, src), (sro, sci, ssrc)):
        nn, k = len(ro_) - 1, len(src_)
        ro_d, ci_d, src_d, lv_d, pr_d = _device_inputs(ro_, ci_, src_)
        rc, st = _call(ro_d, ci_d, src_d, lv_d, pr_d, nn, k)
        assert rc == xbtrav.XB_OK, xbtrav.lib().xb_last_error()
        lv, pr, _, _ = oracle.msbfs(ro_, ci_, src_)
        np.testing.assert_array_equal(lv_d.cpu().numpy(), lv)
        np.testing.assert_array_equal(pr_d.cpu().numpy(), pr)
    ro_d, ci_d, src_d, lv_d, pr_d = _device_inputs(ro, ci, src)
    rc, st = _call(ro_d, ci_d, src_d, lv_d, pr_d, n, len(src))
    assert rc == xbtrav.XB_OK
    assert st.levels > 1024  # planes 0..10 at least
    ctx = xbtrav.Context(0)
    g = ctx.upload(xbtrav.HostCSR.from_arrays(ro, ci))
    ref = ctx.traverse(g, src)
    np.testing.assert_array_equal(lv_d.cpu().numpy(), ref.level)
    np.testing.assert_array_equal(pr_d.cpu().numpy(), ref.parent)
    g.close()
    ctx.close()


def test_noalloc_allocates_no_device_memory():
    """After a first call (set-up), further calls on a new graph leave the
    device's free memory unchanged."""
    import torch

    csr = xbtrav.HostCSR.rmat(13, 8, seed=91)
    ro, ci = csr.arrays()
    src = xbtrav.select_sources_csr(ro, 92, 100)
    ro_d, ci_d, src_d, lv_d, pr_d = _device_inputs(ro, ci, src)
    rc, _ = _call(ro_d, ci_d, src_d, lv_d, pr_d, len(ro) - 1, len(src))
    assert rc == xbtrav.XB_OK
    csr2 = xbtrav.HostCSR.rmat(14, 4, seed=93)
    ro2, ci2 = csr2.arrays()
    src2 = xbtrav.select_sources_csr(ro2, 94, 70)
    ins = _device_inputs(ro2, ci2, src2)
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(2):
        rc, _ = _call(*ins, len(ro2) - 1, len(src2))
        assert rc == xbtrav.XB_OK
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0
