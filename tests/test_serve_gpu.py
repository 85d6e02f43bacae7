"""Serving loop (xbtrav.serve over the slot entry points): continuous batching
of queries that arrive while others run, admission by free HBM, digests.

Bar: every query's result is the same alone and in the mix -- tables
bit-identical to xb_traverse's and to the oracle's (min-id parents), digests
equal to the digests of the oracle's tables.
"""
import numpy as np
import pytest

import xbtrav
from oracle import oracle as O
from xbtrav import serve

pytestmark = pytest.mark.gpu


def _tune(ctx, **kw):
    base = dict(word_bits=64, words=1, pull_alpha=256.0, heavy_degree=256, timing=0, chains=2, tile=0, push_beta=0.0)
    base.update(kw)
    ctx.set_tuning(**base)


def _oracle_digest(lv, pr):
    """Digests of the oracle's tables: reached, level sum, position-sensitive
    row hash, depth (xb_row_digest)."""
    return O.row_digests(lv, pr)


@pytest.fixture(scope="module")
def graphs():
    return [xbtrav.HostCSR.rmat(12, 16, seed=501).arrays(), xbtrav.HostCSR.er(5000, 20000, seed=502).arrays()]


@pytest.mark.parametrize("slots", [1, 3])
def test_mix_equals_alone(ctx, graphs, slots):
    _tune(ctx)
    dg = [ctx.upload_arrays(ro, ci) for ro, ci in graphs]
    rng = np.random.default_rng(11)
    srv = serve.Server(ctx, slots=slots, reserve_bytes=1 << 30)
    qs = []
    for i in range(14):
        gi = i % 2
        k = int(rng.choice([1, 5, 40, 64, 65, 150]))
        src = dg[gi].select_sources(1000 + i, k)
        qs.append((gi, src, srv.submit(dg[gi], src, want="tables" if i % 3 else "digest")))
        if i == 6:  # the second half arrives while the first half runs
            for _ in range(3):
                srv.step()
    srv.drain()
    for gi, src, q in qs:
        assert q.done and q.latency_s >= 0
        ro, ci = graphs[gi]
        lv, pr, _, _ = O.msbfs(ro, ci, src, rule=O.RULE_MINID)
        if q.want == "tables":
            np.testing.assert_array_equal(q.level.cpu().numpy(), lv)
            np.testing.assert_array_equal(q.parent.cpu().numpy(), pr)
            alone = ctx.traverse(dg[gi], src)
            np.testing.assert_array_equal(alone.level, lv)
        else:
            np.testing.assert_array_equal(q.digest, _oracle_digest(lv, pr))
    for g in dg:
        g.close()


def test_poisson_trace_latency(ctx, graphs):
    _tune(ctx)
    dg = [ctx.upload_arrays(ro, ci) for ro, ci in graphs]
    srv = serve.Server(ctx, slots=4)
    trace = serve.poisson_trace(dg, rate_per_s=400.0, count=40, seed=5, kmax=300)
    out = srv.run_trace(trace)
    assert out["queries"] == 40
    assert 0 <= out["p50_ms"] <= out["p99_ms"]
    assert out["gteps"] > 0
    # spot-check a few digests against the oracle
    for q in srv.completed[:5]:
        gi = 0 if q.graph is dg[0] else 1
        lv, pr, _, _ = O.msbfs(*graphs[gi], q.sources, rule=O.RULE_MINID)
        np.testing.assert_array_equal(q.digest, _oracle_digest(lv, pr))
    for g in dg:
        g.close()


def test_admission_waits_for_free_memory(ctx, graphs):
    """With a reserve that leaves no room, a tables query waits while digest
    queries behind it run; it is admitted once the reserve is lowered."""
    import torch

    _tune(ctx)
    g = ctx.upload_arrays(*graphs[0])
    free = torch.cuda.mem_get_info()[0]
    srv = serve.Server(ctx, slots=2, reserve_bytes=free)
    src = g.select_sources(3, 10)
    qt = srv.submit(g, src, want="tables")
    qd = srv.submit(g, src, want="digest")
    for _ in range(50):
        srv.step(wait=True)
        if qd.done:
            break
    assert qd.done and not qt.done and qt.admitted is None
    srv.reserve = 0
    srv.drain()
    assert qt.done
    np.testing.assert_array_equal(qt.level.cpu().numpy(), O.msbfs(*graphs[0], src)[0])
    with pytest.raises(ValueError):  # can never fit: refused at submission
        serve.Server(ctx, reserve_bytes=1 << 62).submit(g, src, want="tables")
    g.close()


def test_slot_api_errors(ctx, graphs):
    _tune(ctx)
    g = ctx.upload_arrays(*graphs[0])
    with pytest.raises(xbtrav.XbError) as e:
        ctx.slot_poll(5)  # nothing in flight
    assert e.value.status == xbtrav.XB_ERR_STATE
    with pytest.raises(xbtrav.XbError) as e:
        ctx.slot_launch(0, g, np.arange(65, dtype=np.int32))
    assert e.value.status == xbtrav.XB_ERR_ARG
    ctx.slot_launch(0, g, np.array([0, 1], np.int32))
    with pytest.raises(xbtrav.XbError) as e:
        ctx.slot_launch(0, g, np.array([2], np.int32))
    assert e.value.status == xbtrav.XB_ERR_STATE
    done, st, dig = ctx.slot_poll(0, wait=True)
    assert done and dig.shape == (2, 4)
    lv, pr, _, _ = O.msbfs(*graphs[0], np.array([0, 1], np.int32))
    np.testing.assert_array_equal(dig, _oracle_digest(lv, pr))
    ctx.slots_release()
    g.close()


def test_digests_on_a_larger_graph_match_the_oracle():
    """R-MAT 20 (hubs above degree 4096) at the default four-word layout:
    digest-only queries of ragged sizes, submitted while earlier ones run;
    every row's digest (with its position-sensitive row hash) equals the
    digest of the oracle's tables."""
    csr = xbtrav.HostCSR.rmat(20, 16, seed=0x5EED + 20)
    ro, ci = csr.arrays()
    c = xbtrav.Context(0)
    g = c.upload(csr)
    srv = serve.Server(c, slots=3, reserve_bytes=1 << 30)
    qs = []
    for i, k in enumerate((1, 37, 130, 5, 64)):
        src = g.select_sources(4000 + i, k)
        qs.append((src, srv.submit(g, src, want="digest")))
        srv.step()
    srv.drain()
    for src, q in qs:
        assert q.done
        lv, pr, _, _ = O.msbfs(ro, ci, src)
        np.testing.assert_array_equal(q.digest, _oracle_digest(lv, pr))
    c.slots_release()
    g.close()
    c.close()


def _path_csr(n):
    ro = np.zeros(n + 1, np.int64)
    ci = []
    for v in range(n):
        nb = [u for u in (v - 1, v + 1) if 0 <= u < n]
        ci.extend(nb)
        ro[v + 1] = ro[v] + len(nb)
    return ro, np.array(ci, np.int32)


@pytest.mark.parametrize("layout", [dict(word_bits=64, words=1), dict(word_bits=32, words=2),
                                    dict(word_bits=64, words=4)])
@pytest.mark.parametrize("alpha,heavy", [(256.0, 256), (1e-6, 32), (1e6, 32)])
def test_all_digest_pass_sums_digests_in_the_table_pass(ctx, graphs, layout, alpha, heavy):
    """A slot pass whose rows are all digest-only computes the digests inside
    the table pass (no rows written); they equal the oracle's, with pushed
    bits (parents searched), heavy vertices (recorded parents) and levels
    past 255 (deep plane decode) among them."""
    _tune(ctx, pull_alpha=alpha, heavy_degree=heavy, **layout)
    cases = list(graphs) + [_path_csr(700)]
    spp = layout["word_bits"] * layout["words"]
    for ro, ci in cases:
        g = ctx.upload_arrays(ro, ci)
        for seed, k in ((7, spp), (8, max(1, spp // 3))):
            src = g.select_sources(seed, k)
            if len(ro) == 701:  # the path: include both ends and the middle
                src = np.array([0, 699, 350][:k] + list(src[3:k]), np.int32) if k >= 3 else src
            ctx.slot_launch(0, g, src, None)
            done, st, dig = ctx.slot_poll(0, wait=True)
            lv, pr, edges, _ = O.msbfs(ro, ci, src, rule=O.RULE_MINID)
            np.testing.assert_array_equal(dig, _oracle_digest(lv, pr))
            assert st["edges_traversed"] == edges
        g.close()
    ctx.slots_release()
    _tune(ctx)


def test_adaptive_width_server_matches_the_oracle(ctx, graphs):
    """Shortest-first scheduling with passes 1, 2 or 4 words wide: every
    query's tables and digests equal the oracle's."""
    _tune(ctx)
    dg = [ctx.upload_arrays(ro, ci) for ro, ci in graphs]
    srv = serve.Server(ctx, slots=2, reserve_bytes=1 << 30, max_words=4)
    qs = []
    for i, k in enumerate([300, 3, 70, 1, 130, 256, 9]):
        gi = i % 2
        src = dg[gi].select_sources(2000 + i, k)
        qs.append((gi, src, srv.submit(dg[gi], src, want="tables" if i % 3 == 1 else "digest")))
    srv.drain()
    for gi, src, q in qs:
        lv, pr, _, _ = O.msbfs(*graphs[gi], src, rule=O.RULE_MINID)
        if q.want == "tables":
            np.testing.assert_array_equal(q.level.cpu().numpy(), lv)
            np.testing.assert_array_equal(q.parent.cpu().numpy(), pr)
        else:
            np.testing.assert_array_equal(q.digest, _oracle_digest(lv, pr))
    ctx.slots_release()
    ctx.set_tuning(words=1)
    for g in dg:
        g.close()


def test_slot_priority_and_express_lane(ctx, graphs):
    """xb_slot_set_priority: a priority-1 slot runs the same passes (digests
    equal the oracle's), the setting is refused on a busy slot and for bad
    arguments; a server with an express slot gives every query the oracle's
    results."""
    _tune(ctx)
    ro, ci = graphs[0]
    g = ctx.upload_arrays(ro, ci)
    ctx.slot_set_priority(0, 1)
    src = g.select_sources(31, 64)
    ctx.slot_launch(0, g, src, None)
    with pytest.raises(xbtrav.XbError):
        ctx.slot_set_priority(0, 0)  # busy
    _, _, dig = ctx.slot_poll(0, wait=True)
    lv, pr, _, _ = O.msbfs(ro, ci, src, rule=O.RULE_MINID)
    np.testing.assert_array_equal(dig, _oracle_digest(lv, pr))
    for bad in ((0, 2), (-1, 0), (99, 1)):
        with pytest.raises(xbtrav.XbError):
            ctx.slot_set_priority(*bad)
    ctx.slot_set_priority(0, 0)
    srv = serve.Server(ctx, slots=3, max_words=4, express=1)
    qs = [(s, srv.submit(g, s, want="digest")) for s in (g.select_sources(40 + i, k) for i, k in
                                                             enumerate([500, 3, 64, 1, 200, 17]))]
    srv.drain()
    for s, q in qs:
        lv, pr, _, _ = O.msbfs(ro, ci, s, rule=O.RULE_MINID)
        np.testing.assert_array_equal(q.digest, _oracle_digest(lv, pr))
    ctx.slots_release()
    for slot in range(3):
        ctx.slot_set_priority(slot, 0)
    ctx.set_tuning(words=1)
    g.close()
