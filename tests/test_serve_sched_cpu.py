"""Launch order of the serving scheduler (xbtrav.serve.Server), on the CPU.

A fake context stands in for the slot API: it records every pass the server
starts and finishes it at once, so the tests see exactly which sources each
pass carried.  Results do not depend on this order (tests/test_serve_gpu.py
checks every query alone and in the mix on the GPU); latency does.
"""
import numpy as np
import pytest

from xbtrav import serve


class _Handle:
    def __init__(self, v):
        self.value = v


class FakeGraph:
    def __init__(self, h, n=100, order=None):
        self._h = _Handle(h)
        self.n = n
        self.order = order  # source_order(src) -> order(src); None = as given

    def source_order(self, src):
        return np.arange(len(src), dtype=np.int32) if self.order is None else self.order(src)


class FakeCtx:
    device = 0

    def __init__(self, words=1):
        self.words = words
        self.launches = []  # (slot, graph handle, sources)
        self.inflight = {}

    def tuning(self):
        return {"word_bits": 64, "words": self.words}

    def set_tuning(self, **kw):
        self.words = kw.get("words", self.words)

    def slot_set_priority(self, slot, priority):
        assert slot not in self.inflight
        self.priority = getattr(self, "priority", {})
        self.priority[slot] = priority

    def slot_launch(self, slot, g, src, rows):
        assert slot not in self.inflight
        assert 1 <= len(src) <= 64 * self.words  # a pass holds at most one layout's sources
        self.launches.append((slot, g._h.value, np.array(src)))
        self.inflight[slot] = np.array(src)

    def slot_poll(self, slot, wait=False):
        src = self.inflight.pop(slot)
        dig = np.zeros((len(src), 4), np.int64)
        dig[:, 0] = src  # each digest row names its source
        return True, {"edges_traversed": 10 * len(src)}, dig


class Clock:
    def __init__(self):
        self.t = 0.0

    def __call__(self):
        return self.t


def _server(slots=1, age_s=1.0, max_words=None, express=0):
    ctx, clk = FakeCtx(), Clock()
    return serve.Server(ctx, slots=slots, clock=clk, age_s=age_s, max_words=max_words, express=express), ctx, clk


def _origin(srcs, queries):
    """Which query each launched source came from (sources are disjoint)."""
    owner = {int(s): q.qid for q in queries for s in q.sources}
    return [owner[int(s)] for s in srcs]


def test_small_queries_open_the_next_pass():
    srv, ctx, clk = _server()
    g = FakeGraph(1)
    big = srv.submit(g, np.arange(0, 256), want="digest")
    small = srv.submit(g, np.arange(1000, 1003), want="digest")
    mid = srv.submit(g, np.arange(2000, 2010), want="digest")
    srv.drain()
    first = _origin(ctx.launches[0][2], [big, small, mid])
    # shortest first: 3 sources, then 10, then the large query fills the word
    assert first[:3] == [small.qid] * 3
    assert first[3:13] == [mid.qid] * 10
    assert first[13:] == [big.qid] * 51
    assert len(ctx.launches) == 5  # 269 sources in words of 64
    assert all(q.done for q in (big, small, mid))
    launched = np.concatenate([x[2] for x in ctx.launches])
    assert sorted(launched.tolist()) == sorted(np.concatenate([big.sources, small.sources, mid.sources]).tolist())


def test_query_arriving_mid_stream_overtakes_a_large_one():
    srv, ctx, clk = _server()
    g = FakeGraph(1)
    big = srv.submit(g, np.arange(0, 640), want="digest")  # ten passes
    srv.step()
    clk.t = 0.1
    late = srv.submit(g, np.arange(5000, 5002), want="digest")
    srv.step()  # collects the first pass, starts the second
    srv.drain()
    second = _origin(ctx.launches[1][2], [big, late])
    assert second[:2] == [late.qid] * 2
    assert late.done_at <= big.done_at


def test_aged_query_goes_first():
    srv, ctx, clk = _server(age_s=0.5)
    g = FakeGraph(1)
    big = srv.submit(g, np.arange(0, 128), want="digest")
    clk.t = 1.0  # big has waited past age_s; the new small query has not
    small = srv.submit(g, np.arange(900, 905), want="digest")
    srv.step()
    first = _origin(ctx.launches[0][2], [big, small])
    assert first == [big.qid] * 64


def test_passes_hold_one_graph():
    srv, ctx, clk = _server(slots=2)
    g1, g2 = FakeGraph(1), FakeGraph(2)
    a = srv.submit(g1, np.arange(0, 5), want="digest")
    b = srv.submit(g2, np.arange(100, 103), want="digest")
    c = srv.submit(g1, np.arange(200, 207), want="digest")
    srv.drain()
    for slot, h, src in ctx.launches:
        owners = _origin(src, [a, b, c])
        graphs = {1 if o in (a.qid, c.qid) else 2 for o in owners}
        assert graphs == {h}
    # the 3-source query of g2 opens the first pass; g1's two queries share the second
    assert ctx.launches[0][1] == 2
    assert _origin(ctx.launches[1][2], [a, b, c]) == [a.qid] * 5 + [c.qid] * 7


def test_trace_latencies_reported():
    srv, ctx, clk = _server(slots=2)
    g = FakeGraph(1)
    trace = [(0.0, g, np.arange(0, 70), "digest"), (0.0, g, np.arange(100, 101), "digest")]
    out = srv.run_trace(trace)
    assert out["queries"] == 2 and out["passes"] == 2
    assert out["p50_ms"] >= 0.0 and out["p99_ms"] >= out["p50_ms"]


@pytest.mark.parametrize("want", ["tables"])
def test_tables_queries_need_device_memory_to_be_admitted(want, monkeypatch):
    srv, ctx, clk = _server()
    g = FakeGraph(1, n=10)
    # never fits: larger than the whole device
    monkeypatch.setattr(srv.torch.cuda, "mem_get_info", lambda dev: (1 << 20, 1 << 20))
    with pytest.raises(ValueError):
        srv.submit(g, np.arange(0, 64), want=want)


def test_adaptive_width_follows_the_opening_query():
    srv, ctx, clk = _server(max_words=4)
    g = FakeGraph(1)
    big = srv.submit(g, np.arange(0, 600), want="digest")
    srv.drain()
    sizes = [len(x[2]) for x in ctx.launches]
    assert sizes == [256, 256, 88]  # 600 = 256 + 256 + 88 (the last opens a two-word pass)
    assert big.done
    small = srv.submit(g, np.arange(1000, 1010), want="digest")
    srv.drain()
    assert len(ctx.launches[-1][2]) == 10 and ctx.words == 1 and small.done


def test_adaptive_width_warmup_visits_every_width():
    srv, ctx, clk = _server(slots=2, max_words=4)

    class G(FakeGraph):
        def select_sources(self, seed, k):
            return np.arange(k) + 1000 * seed

    srv.warmup(G(1))
    assert [len(x[2]) for x in ctx.launches] == [64, 64, 128, 128, 256, 256]


def test_max_words_validated():
    with pytest.raises(ValueError):
        _server(max_words=3)


def test_refused_launch_keeps_its_sources_waiting():
    srv, ctx, clk = _server()
    g = FakeGraph(1)
    real = ctx.slot_launch
    calls = {"n": 0}

    def refuse_once(slot, gr, src, rows):
        calls["n"] += 1
        if calls["n"] == 1:
            raise RuntimeError("XB_ERR_OOM")
        real(slot, gr, src, rows)

    ctx.slot_launch = refuse_once
    q = srv.submit(g, np.arange(0, 100), want="digest")
    with pytest.raises(RuntimeError):
        srv.step()
    assert q.rows_launched == 0 and srv.waiting == [q]
    srv.drain()
    assert q.done and sorted(np.concatenate([x[2] for x in ctx.launches]).tolist()) == list(range(100))


def test_express_slot_takes_only_passes_opened_by_small_queries():
    srv, ctx, clk = _server(slots=2, max_words=4, express=1)
    assert ctx.priority == {0: 1, 1: 0}
    g = FakeGraph(1)
    big = srv.submit(g, np.arange(0, 600), want="digest")
    srv.step()  # slot 0 (express) finds no small query; slot 1 takes a wide pass
    assert [x[0] for x in ctx.launches] == [1] and len(ctx.launches[0][2]) == 256
    small = srv.submit(g, np.arange(5000, 5010), want="digest")
    srv.step()  # slot 1's pass is collected; the express slot opens a one-word pass with the small query
    express = [x for x in ctx.launches if x[0] == 0]
    assert express and _origin(express[0][2], [big, small])[:10] == [small.qid] * 10
    assert len(express[0][2]) == 64  # the rest of the word filled from the large query
    srv.drain()
    assert big.done and small.done
    launched = np.concatenate([x[2] for x in ctx.launches]).tolist()
    assert sorted(launched) == sorted(list(range(600)) + list(range(5000, 5010)))


def test_express_needs_an_ordinary_slot():
    with pytest.raises(ValueError):
        _server(slots=1, express=1)


def test_query_over_several_passes_launches_in_the_graphs_order():
    """A 150-source query (three one-word passes) launches its sources in the
    order the graph's source_order gives; every digest lands at its source's
    row of the query."""
    srv, ctx, clk = _server()
    g = FakeGraph(1, order=lambda src: np.argsort(-np.asarray(src), kind="stable").astype(np.int32))
    src = np.random.default_rng(3).permutation(np.arange(500, 650)).astype(np.int32)
    q = srv.submit(g, src, want="digest")
    srv.drain()
    launched = np.concatenate([s for _, _, s in ctx.launches])
    np.testing.assert_array_equal(launched, np.sort(src)[::-1])
    assert [len(s) for _, _, s in ctx.launches] == [64, 64, 22]
    np.testing.assert_array_equal(q.digest[:, 0], src)


def test_one_word_query_keeps_its_order():
    """A query that fits one word is launched as given (one pass either way)."""
    srv, ctx, clk = _server()
    g = FakeGraph(1, order=lambda src: np.arange(len(src))[::-1].astype(np.int32))
    src = np.arange(10, 74).astype(np.int32)
    q = srv.submit(g, src, want="digest")
    srv.drain()
    np.testing.assert_array_equal(ctx.launches[0][2], src)
    np.testing.assert_array_equal(q.digest[:, 0], src)
