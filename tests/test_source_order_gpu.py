"""Pass grouping of the sources (xb_tuning.source_order): 0 (default) packs a
call's sources into passes by out-degree, highest first; 1 keeps the given
order.  Either way every source's level and parent rows land in the row the
caller gave it.

Bar: bit-exact tables against the oracle (min-id and FIFO parent rules) for
both groupings, on the plain and the batched path, with device and host
output tables, with repeated sources and with source lists in no degree
order; host-table batched calls with new sources at the same buffers (the
captured copies are keyed on the grouping) still land every row.
"""
import numpy as np
import pytest

import xbtrav
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _tune(ctx, order, **kw):
    base = dict(word_bits=64, words=1, pull_alpha=64.0, heavy_degree=256, timing=0, chains=2, tile=0,
                push_beta=0.0, source_order=order)
    base.update(kw)
    ctx.set_tuning(**base)


def _host(t):
    return t.cpu().numpy() if hasattr(t, "cpu") else np.asarray(t)


@pytest.fixture(scope="module")
def rmat12():
    return xbtrav.HostCSR.rmat(12, 16, seed=202).arrays()


def _sources(ro, seed, k):
    """k sources in shuffled order with a few repeats, so grouping by degree
    moves rows between passes."""
    rng = np.random.default_rng(seed)
    src = np.asarray(xbtrav.select_sources_csr(ro, seed, k), dtype=np.int32)
    src[rng.choice(k, size=k // 10, replace=False)] = src[0]
    return src[rng.permutation(k)]


@pytest.mark.parametrize("order", [0, 1])
@pytest.mark.parametrize("layout", [dict(word_bits=64, words=1), dict(word_bits=32, words=2),
                                    dict(word_bits=64, words=4)])
@pytest.mark.parametrize("out", ["device", "host"])
def test_plain_rows_land_where_asked(ctx, rmat12, order, layout, out):
    ro, ci = rmat12
    _tune(ctx, order, **layout)
    g = ctx.upload_arrays(ro, ci)
    src = _sources(ro, 3, 600)
    lv, pr, _, _ = O.msbfs(ro, ci, src, rule=O.RULE_MINID)
    r = ctx.traverse(g, src, out=out)
    np.testing.assert_array_equal(_host(r.level), lv)
    np.testing.assert_array_equal(_host(r.parent), pr)
    g.close()


@pytest.mark.parametrize("order", [0, 1])
def test_plain_fifo_parents_under_grouping(ctx, rmat12, order):
    ro, ci = rmat12
    _tune(ctx, order)
    g = ctx.upload_arrays(ro, ci)
    src = _sources(ro, 4, 300)
    lv, pr, _, _ = O.msbfs(ro, ci, src, rule=O.RULE_FIFO)
    r = ctx.traverse(g, src, parent_rule="fifo")
    np.testing.assert_array_equal(r.level, lv)
    np.testing.assert_array_equal(r.parent, pr)
    g.close()


@pytest.mark.parametrize("order", [0, 1])
@pytest.mark.parametrize("out", ["device", "host"])
def test_batched_queries_under_grouping(ctx, rmat12, order, out):
    """Three queries on one graph: grouping by degree interleaves their rows
    across passes; each query's tables still match the oracle."""
    ro, ci = rmat12
    _tune(ctx, order, chains=3)
    g = ctx.upload_arrays(ro, ci)
    qs = [_sources(ro, s, k) for s, k in ((21, 150), (22, 90), (23, 7))]
    res, st = ctx.traverse_batched([(g, q) for q in qs], out=out)
    e_all = 0
    for q, r in zip(qs, res):
        lv, pr, e, _ = O.msbfs(ro, ci, q, rule=O.RULE_MINID)
        np.testing.assert_array_equal(_host(r.level), lv)
        np.testing.assert_array_equal(_host(r.parent), pr)
        e_all += e
    assert st["edges_traversed"] == e_all
    g.close()


def test_host_tables_new_sources_same_buffers(ctx, rmat12):
    """Host-table batched calls at the same buffers with new sources: the
    grouping changes with the sources, and so do the captured copies."""
    import torch

    ro, ci = rmat12
    _tune(ctx, 0, chains=2)
    g = ctx.upload_arrays(ro, ci)
    k = 200
    hl = torch.empty((k, g.n), dtype=torch.int32, pin_memory=True)
    hp = torch.empty((k, g.n), dtype=torch.int32, pin_memory=True)
    for seed in (31, 32, 31):
        src = _sources(ro, seed, k)
        res, _ = ctx.traverse_batched([(g, src)], out="host", outputs=[(hl, hp)])
        lv, pr, _, _ = O.msbfs(ro, ci, src, rule=O.RULE_MINID)
        np.testing.assert_array_equal(_host(res[0].level), lv)
        np.testing.assert_array_equal(_host(res[0].parent), pr)
    g.close()


def test_grouping_changes_nothing_but_speed(ctx, rmat12):
    """Both groupings give the same tables and the same edge count."""
    ro, ci = rmat12
    g = ctx.upload_arrays(ro, ci)
    src = _sources(ro, 5, 500)
    outs = []
    for order in (0, 1):
        _tune(ctx, order, words=4)
        r = ctx.traverse(g, src)
        outs.append((r.level, r.parent, r.stats["edges_traversed"]))
    np.testing.assert_array_equal(outs[0][0], outs[1][0])
    np.testing.assert_array_equal(outs[0][1], outs[1][1])
    assert outs[0][2] == outs[1][2]
    g.close()


def test_source_order_validated(ctx):
    with pytest.raises(xbtrav.XbError):
        ctx.set_tuning(source_order=2)
    _tune(ctx, 0)


def test_source_order_api_is_the_degree_grouping(ctx, rmat12):
    """xb_graph_source_order: indices by out-degree, highest first, equal
    degrees by the sum of the neighbours' degrees, highest first, then in the
    given order; out-of-range sources are refused."""
    ro, ci = rmat12
    ro, ci = np.asarray(ro), np.asarray(ci)
    g = ctx.upload_arrays(ro, ci)
    src = _sources(ro, 6, 400)
    dall = np.diff(ro)
    deg = dall[src]
    r2 = np.array([dall[ci[ro[s]:ro[s + 1]]].sum() for s in src])
    want = np.lexsort((np.arange(len(src)), -r2, -deg))
    np.testing.assert_array_equal(g.source_order(src), want)
    assert (np.diff(deg[want]) <= 0).all()
    assert len(g.source_order(np.zeros(0, np.int32))) == 0
    with pytest.raises(xbtrav.XbError):
        g.source_order(np.array([0, g.n], np.int32))
    g.close()
