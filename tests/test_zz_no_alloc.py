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


def _call(ro_d, ci_d, src_d, level_d, parent_d, n, k, stats=None):
    import torch

    torch.cuda.synchronize()
    st = stats if stats is not None else xbtrav.XbStats()
    rc = _noalloc()(n, ro_d.data_ptr(), ci_d.data_ptr() if ci_d.numel() else None, src_d.data_ptr(), k,
                    level_d.data_ptr(), parent_d.data_ptr(), None, C.byref(st))
    torch.cuda.synchronize()
    return rc, st


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
