"""Parity of the batched path (xb_traverse_batched: one CUDA-graph launch per
batch, device-side level loop, sources of several queries sharing words,
passes over concurrent chains) with the CPU oracle and with the plain path.

Bar: levels and parents bit-exact under the min-id rule for every query,
whatever the packing of its sources into words and whichever chain ran them.
"""
import numpy as np
import pytest

import xbtrav
from oracle import oracle as O

pytestmark = pytest.mark.gpu

LAYOUTS = [
    dict(word_bits=64, words=1),
    dict(word_bits=32, words=1),
    dict(word_bits=64, words=2),
    dict(word_bits=32, words=4),
    dict(word_bits=64, words=4),  # the default layout (256 sources per pass)
]


def _tune(ctx, **kw):
    base = dict(word_bits=64, words=1, pull_alpha=64.0, heavy_degree=256, timing=0, chains=2, tile=0, push_beta=0.0)
    base.update(kw)
    ctx.set_tuning(**base)


def _host(t):
    return t.cpu().numpy() if hasattr(t, "cpu") else np.asarray(t)


def _check(ro, ci, src, res):
    lv, pr, edges, reached = O.msbfs(ro, ci, src, rule=O.RULE_MINID)
    np.testing.assert_array_equal(_host(res.level), lv)
    np.testing.assert_array_equal(_host(res.parent), pr)
    return edges, reached


@pytest.fixture(scope="module")
def rmat12():
    h = xbtrav.HostCSR.rmat(12, 16, seed=101)
    return h.arrays()


@pytest.mark.parametrize("layout", range(len(LAYOUTS)))
@pytest.mark.parametrize("chains", [1, 3])
def test_single_graph_device_outputs(ctx, rmat12, layout, chains):
    ro, ci = rmat12
    src = xbtrav.select_sources_csr(ro, 5, 200)
    _tune(ctx, chains=chains, **LAYOUTS[layout])
    g = ctx.upload_arrays(ro, ci)
    res, st = ctx.traverse_batched([(g, src)])
    edges, reached = _check(ro, ci, src, res[0])
    assert st["edges_traversed"] == edges
    assert st["reached"] == reached
    g.close()


@pytest.mark.parametrize("layout", [0, 2, 3, 4])
@pytest.mark.parametrize("heavy", [32, 256])
def test_launch_tile_one(ctx, rmat12, layout, heavy):
    """xb_tuning.tile = 1 (two rounds in flight per heavy-pull warp, 8-warp
    table blocks): same tables as the oracle, with most vertices routed
    through the heavy pull when the cutoff is 32."""
    ro, ci = rmat12
    _tune(ctx, chains=2, heavy_degree=heavy, tile=1, **LAYOUTS[layout])
    g = ctx.upload_arrays(ro, ci)
    src = xbtrav.select_sources_csr(ro, 77, 200)
    res, _ = ctx.traverse_batched([(g, src)])
    _check(ro, ci, src, res[0])
    _check(ro, ci, src, ctx.traverse(g, src))
    g.close()
    _tune(ctx)


@pytest.mark.parametrize("beta", [2.0, 24.0])
@pytest.mark.parametrize("layout", [0, 4])
@pytest.mark.parametrize("heavy", [32, 256])
def test_tail_push_rule(ctx, rmat12, beta, layout, heavy):
    """tuning.push_beta: after a pull step, a frontier under n/push_beta
    vertices is pushed (parents of its bits searched by the table pass,
    heavy ones by the heavy-vertex search): same tables as the oracle on the
    batched and the plain path."""
    ro, ci = rmat12
    _tune(ctx, chains=2, heavy_degree=heavy, pull_alpha=1024.0, push_beta=beta, **LAYOUTS[layout])
    g = ctx.upload_arrays(ro, ci)
    src = xbtrav.select_sources_csr(ro, 91, 150)
    res, st = ctx.traverse_batched([(g, src)])
    _check(ro, ci, src, res[0])
    r = ctx.traverse(g, src)
    _check(ro, ci, src, r)
    if beta == 2.0:  # beyond each pass's first (push) level, the tail was pushed
        spp = LAYOUTS[layout]["word_bits"] * LAYOUTS[layout]["words"]
        assert r.stats["push_levels"] > (len(src) + spp - 1) // spp
    g.close()
    _tune(ctx)


@pytest.mark.parametrize("alpha", [1e-6, 1e6])
@pytest.mark.parametrize("heavy", [32, 2048])
def test_forced_push_or_pull(ctx, rmat12, alpha, heavy):
    """alpha=1e-6: push while any unfinished edge remains (parents searched
    by the table pass); alpha=1e6: every level pulls; heavy=32 routes most
    vertices through the per-vertex and hub kernels inside the captured
    switch bodies.  The device-side decisions equal the plain path's."""
    ro, ci = rmat12
    src = xbtrav.select_sources_csr(ro, 6, 130)
    _tune(ctx, pull_alpha=alpha, heavy_degree=heavy)
    g = ctx.upload_arrays(ro, ci)
    res, st = ctx.traverse_batched([(g, src)])
    _check(ro, ci, src, res[0])
    plain = ctx.traverse(g, src).stats
    assert (st["push_levels"], st["pull_levels"]) == (plain["push_levels"], plain["pull_levels"])
    if alpha == 1e6:
        assert st["push_levels"] == 0
    else:
        assert st["push_levels"] > st["pull_levels"]
    g.close()


def _uneven_graphs():
    """Graphs of uneven sizes and degrees, ragged query sizes (1..130)."""
    rng = np.random.default_rng(7)
    gs = []
    for i, (scale, ef) in enumerate([(8, 4), (10, 32), (12, 8), (9, 16), (11, 4)]):
        gs.append(xbtrav.HostCSR.rmat(scale, ef, seed=200 + i).arrays())
    gs.append(xbtrav.HostCSR.er(3000, 9000, seed=300).arrays())
    queries = []
    for gi, (ro, _) in enumerate(gs):
        for k in rng.choice([1, 3, 17, 64, 65, 130], size=2, replace=False):
            queries.append((gi, xbtrav.select_sources_csr(ro, int(rng.integers(1 << 30)), int(k))))
    return gs, queries


@pytest.mark.parametrize("out", ["device", "host"])
@pytest.mark.parametrize("chains", [1, 4])
def test_uneven_multi_graph_batch(ctx, out, chains):
    gs, queries = _uneven_graphs()
    _tune(ctx, chains=chains)
    dg = [ctx.upload_arrays(ro, ci) for ro, ci in gs]
    res, st = ctx.traverse_batched([(dg[gi], src) for gi, src in queries], out=out)
    tot_e = tot_r = 0
    for (gi, src), r in zip(queries, res):
        e, rc = _check(*gs[gi], src, r)
        tot_e += e
        tot_r += rc
    assert st["edges_traversed"] == tot_e
    assert st["reached"] == tot_r
    for g in dg:
        g.close()


@pytest.mark.parametrize("chains", [2, 8])
def test_concatenated_csr_instances(ctx, chains):
    """Instances uploaded as one concatenated CSR (xb_graph_upload_batch)
    traverse exactly like separately uploaded graphs, on both paths."""
    gs, queries = _uneven_graphs()
    _tune(ctx, chains=chains)
    views = ctx.upload_batch(gs)
    assert [v.n for v in views] == [len(ro) - 1 for ro, _ in gs]
    res, st = ctx.traverse_batched([(views[gi], src) for gi, src in queries])
    for (gi, src), r in zip(queries, res):
        _check(*gs[gi], src, r)
        plain = ctx.traverse(views[gi], src)
        np.testing.assert_array_equal(plain.level, _host(r.level))
        np.testing.assert_array_equal(plain.parent, _host(r.parent))
    # freeing some views leaves the others usable
    for v in views[::2]:
        v.close()
    gi, src = next((q for q in queries if q[0] % 2 == 1))
    r = ctx.traverse(views[gi], src)
    _check(*gs[gi], src, r)
    for v in views[1::2]:
        v.close()


def test_same_results_as_plain_path(ctx):
    h = xbtrav.HostCSR.rmat(14, 16, seed=9)
    ro, ci = h.arrays()
    src = xbtrav.select_sources_csr(ro, 10, 192)
    _tune(ctx)
    g = ctx.upload_arrays(ro, ci)
    plain = ctx.traverse(g, src, out="device")
    res, st = ctx.traverse_batched([(g, src)])
    assert bool((plain.level == res[0].level).all())
    assert bool((plain.parent == res[0].parent).all())
    assert st["edges_traversed"] == plain.stats["edges_traversed"]
    assert st["algo_bytes"] > 0
    g.close()


def test_cached_launch_reused_with_new_sources_and_outputs(ctx, rmat12):
    """The second and third calls hit the cached graph (same shape); sources
    and device output tensors differ each time."""
    import torch

    ro, ci = rmat12
    _tune(ctx)
    g = ctx.upload_arrays(ro, ci)
    for seed in (1, 2, 3):
        src = xbtrav.select_sources_csr(ro, seed, 77)
        dev = torch.device("cuda", 0)
        outs = [(torch.full((77, g.n), 7, dtype=torch.int32, device=dev),
                 torch.full((77, g.n), 7, dtype=torch.int32, device=dev))]
        res, _ = ctx.traverse_batched([(g, src)], outputs=outs)
        _check(ro, ci, src, res[0])
    g.close()


def test_sources_of_two_queries_share_words(ctx, rmat12):
    """Queries of 40 + 40 + 1 sources on one graph pack into two words; each
    query's rows still land in its own tables."""
    ro, ci = rmat12
    _tune(ctx)
    g = ctx.upload_arrays(ro, ci)
    qs = [xbtrav.select_sources_csr(ro, s, k) for s, k in ((11, 40), (12, 40), (13, 1))]
    res, st = ctx.traverse_batched([(g, q) for q in qs])
    assert st["batches"] == 2
    for q, r in zip(qs, res):
        _check(ro, ci, q, r)
    g.close()


def test_graph_freed_and_replaced(ctx):
    _tune(ctx)
    for seed in (31, 32):
        ro, ci = xbtrav.HostCSR.rmat(10, 8, seed=seed).arrays()
        g = ctx.upload_arrays(ro, ci)
        src = xbtrav.select_sources_csr(ro, seed, 50)
        res, _ = ctx.traverse_batched([(g, src)])
        _check(ro, ci, src, res[0])
        g.close()


def test_errors_and_empty_items(ctx, rmat12):
    ro, ci = rmat12
    _tune(ctx)
    g = ctx.upload_arrays(ro, ci)
    res, st = ctx.traverse_batched([])
    assert res == [] and st["edges_traversed"] == 0
    res, st = ctx.traverse_batched([(g, np.zeros(0, np.int32))])
    assert st["batches"] == 0
    with pytest.raises(xbtrav.XbError) as e:
        ctx.traverse_batched([(g, np.array([0, g.n], np.int32))])
    assert e.value.status == xbtrav.XB_ERR_ARG
    pageable = [(np.empty((2, g.n), np.int32), np.empty((2, g.n), np.int32))]
    with pytest.raises(xbtrav.XbError) as e:
        ctx.traverse_batched([(g, np.array([0, 1], np.int32))], out="host", outputs=pageable)
    assert e.value.status == xbtrav.XB_ERR_ARG
    # the context still works afterwards
    src = xbtrav.select_sources_csr(ro, 3, 10)
    res, _ = ctx.traverse_batched([(g, src)])
    _check(ro, ci, src, res[0])
    g.close()
