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
    base = dict(word_bits=64, words=1, pull_alpha=256.0, heavy_degree=256, timing=0, chains=2, tile=0)
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
