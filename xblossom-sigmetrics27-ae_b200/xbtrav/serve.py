"""Serving loop with continuous batching over the engine's slots.

Queries (a graph and a set of sources) arrive at any time.  The server keeps
the graphs resident, admits queries by free HBM, and packs the sources of
whatever queries are waiting -- several queries per pass, a query spread over
many passes -- into passes of up to word_bits x words sources that run on its
slots (xb_slot_launch: one pass in flight per slot, each slot with its own
stream and workspace, so passes of different slots overlap on the device).  A
query that arrives while others are on the GPU joins the next pass any slot
starts; nothing waits for a batch to fill.

With express > 0, the first `express` slots run at the device's greatest
stream priority (xb_slot_set_priority) and only take one-word passes opened
by a query that fits one: a small query neither waits for a slot behind the
wide passes of large ones nor yields the SMs to them while it runs.

Passes are filled shortest query first: the query with the fewest sources
still to launch opens the pass, and the rest of it takes the other waiting
queries of the same graph in the same order.  A pass costs about the same
whatever share of its word the sources fill (every unfinished vertex is
scanned), so a small query served behind a large one would wait for all of
the large one's passes; shortest-first serves it in the next pass any slot
starts.  A query that has waited longer than `age_s` since admission opens
the next pass regardless of its size, so large queries cannot starve.

With max_words above the context's words per vertex, each pass is as wide
as the query that opens it needs (1, 2 or 4 words, never above max_words):
a wide pass serves many sources at a lower cost per source, a narrow one
finishes sooner, so large queries take wide passes and small ones narrow
passes.  The context's tuning.words is switched before each launch (the
server owns the context); every slot keeps a workspace and scratch rows for
the widest pass it has run.

A query of more than one word's sources launches them grouped by
out-degree, highest first (xb_graph_source_order, the grouping the library's
own calls use under tuning.source_order 0): its passes then hold sources
whose traversals grow alike.  Rows, tables and digests stay at the
positions of the query's source list.

Each query asks for one of two results:
  want="tables": the full int32 level / parent tables (k x n each) in device
      memory.  The tables are allocated when the query is admitted, which
      happens once they fit into free HBM above a reserve, in arrival order;
      digest queries may pass a tables query that waits for memory.
  want="digest": per source the reached-vertex count, level sum, a
      position-sensitive hash of its (vertex, level, parent) entries and the
      depth (xb_row_digest), computed on the device from the slot's
      scratch rows; no admission memory.  This is the mode for graphs whose
      tables cannot be held (R-MAT scale 25: 268 MB per source).

The reference has no serving path; results equal xb_traverse's for the same
sources (tests/test_serve_gpu.py checks every query alone and in the mix).

    srv = Server(ctx, slots=4)
    q = srv.submit(graph, sources, want="tables")
    srv.drain()
    q.level, q.parent, q.latency_s
"""
from __future__ import annotations

import collections
import time
from dataclasses import dataclass, field

import numpy as np


@dataclass
class Query:
    qid: int
    graph: object
    sources: np.ndarray
    want: str
    arrival: float
    level: object = None   # torch (k, n) int32 on the device (want="tables")
    parent: object = None
    digest: np.ndarray = None  # (k, 4) int64: reached, level_sum, row_hash, depth (want="digest")
    admitted: float = None
    done_at: float = None
    rows_done: int = 0
    rows_launched: int = 0
    passes: set = field(default_factory=set)
    order: np.ndarray = None  # launch position -> row of sources / tables / digest

    @property
    def k(self) -> int:
        return len(self.sources)

    @property
    def done(self) -> bool:
        return self.done_at is not None

    @property
    def latency_s(self) -> float:
        return self.done_at - self.arrival


class Server:
    def __init__(self, ctx, slots: int = 4, reserve_bytes: int = 4 << 30, clock=time.perf_counter,
                 age_s: float = 1.0, max_words: int | None = None, express: int = 0):
        import torch

        self.torch = torch
        self.ctx = ctx
        self.nslots = slots
        self.reserve = reserve_bytes
        self.clock = clock
        t = ctx.tuning()
        self.word_bits = t["word_bits"]
        self.base_words = t["words"]
        self.max_words = max(self.base_words, max_words or self.base_words)
        if self.max_words not in (1, 2, 4):
            raise ValueError("max_words must be 1, 2 or 4")
        self.cur_words = self.base_words
        self.rows_per_pass = self.word_bits * self.base_words
        self.dev = torch.device("cuda", ctx.device)
        self.age_s = age_s
        # a query over several passes launches its sources grouped by degree,
        # as the library's own calls do (xb_tuning.source_order 0)
        self.group = t.get("source_order", 0) == 0
        if not 0 <= express < slots:
            raise ValueError("express must leave at least one ordinary slot")
        self.express = express
        for s in range(slots):
            ctx.slot_set_priority(s, 1 if s < express else 0)
        self.admit_q = collections.deque()      # queries waiting for memory
        self.waiting = []                       # admitted queries with sources not yet launched
        self.slot_rows = [None] * slots         # rows of the pass in flight per slot
        self.slot_pass = [0] * slots
        self.completed = []
        self.edges = 0
        self.passes = 0
        self._next = 0

    # queries ---------------------------------------------------------------
    def submit(self, graph, sources, want: str = "digest", arrival: float | None = None) -> Query:
        if want not in ("tables", "digest"):
            raise ValueError("want must be 'tables' or 'digest'")
        src = np.ascontiguousarray(sources, dtype=np.int32)
        if want == "tables":
            total = self.torch.cuda.mem_get_info(self.dev)[1]
            if 8 * len(src) * graph.n + self.reserve > total:
                raise ValueError("the query's tables can never fit into device memory; ask for want='digest'")
        q = Query(self._next, graph, src, want, self.clock() if arrival is None else arrival)
        self._next += 1
        q.order = (graph.source_order(src) if self.group and q.k > self.word_bits
                   else np.arange(q.k, dtype=np.int32))
        if q.k == 0:
            q.admitted = q.done_at = q.arrival
            self.completed.append(q)
            return q
        self.admit_q.append(q)
        self._admit()
        return q

    def _admit(self) -> None:
        free = None
        keep = collections.deque()
        while self.admit_q:
            q = self.admit_q.popleft()
            if q.want == "digest":
                q.digest = np.zeros((q.k, 4), np.int64)
                self._enqueue(q)
                continue
            need = 8 * q.k * q.graph.n
            if free is None:
                free = self.torch.cuda.mem_get_info(self.dev)[0]
            if keep or need + self.reserve > free:
                keep.append(q)  # tables queries keep their arrival order
                continue
            q.level = self.torch.empty((q.k, q.graph.n), dtype=self.torch.int32, device=self.dev)
            q.parent = self.torch.empty((q.k, q.graph.n), dtype=self.torch.int32, device=self.dev)
            free -= need
            self._enqueue(q)
        self.admit_q = keep

    def _enqueue(self, q: Query) -> None:
        q.admitted = self.clock()
        self.waiting.append(q)

    # slots ------------------------------------------------------------------
    def _order(self, now: float) -> list:
        """Waiting queries in launch order: those past age_s by admission
        time, then the rest by sources still to launch (ties: admission)."""
        aged = sorted((q for q in self.waiting if now - q.admitted > self.age_s), key=lambda q: q.admitted)
        rest = sorted((q for q in self.waiting if now - q.admitted <= self.age_s),
                      key=lambda q: (q.k - q.rows_launched, q.admitted, q.qid))
        return aged + rest

    def _launch(self, slot: int) -> bool:
        """Starts a pass on an idle slot: the first query in launch order
        opens it, other waiting queries of its graph fill the rest.  An
        express slot takes only one-word passes opened by a query that fits
        one."""
        if not self.waiting:
            return False
        order = self._order(self.clock())
        if slot < self.express:
            narrow = self.word_bits * self.base_words
            small = [q for q in order if q.k - q.rows_launched <= narrow]
            if not small:
                return False
            order = small + [q for q in order if q.k - q.rows_launched > narrow]  # the rest fills the word
        g = order[0].graph
        cap = self._width(order[0].k - order[0].rows_launched)
        take = []
        for q in order:
            if q.graph._h.value != g._h.value:
                continue
            n = min(cap - len(take), q.k - q.rows_launched)
            take.extend((q, j) for j in range(q.rows_launched, q.rows_launched + n))
            q.rows_launched += n
            if len(take) == cap:
                break
        src = np.array([q.sources[q.order[j]] for q, j in take], dtype=np.int32)
        rows = []
        for q, j in take:
            r = int(q.order[j])
            rows.append(None if q.want == "digest" else (q.level[r].data_ptr(), q.parent[r].data_ptr()))
        try:
            self.ctx.slot_launch(slot, g, src, rows)
        except Exception:
            # a pass the library refused: its sources wait again
            for q, j in take:
                q.rows_launched = min(q.rows_launched, j)
            raise
        self.waiting = [q for q in self.waiting if q.rows_launched < q.k]
        self.slot_rows[slot] = take
        self.passes += 1
        self.slot_pass[slot] = self.passes
        return True

    def _width(self, rows: int) -> int:
        """Rows of the next pass for an opening query with `rows` sources
        left: the narrowest allowed width that holds them (the widest if none
        does); switches the context's layout when it changes."""
        words = self.base_words
        while words < self.max_words and rows > self.word_bits * words:
            words *= 2
        if words != self.cur_words:
            self.ctx.set_tuning(words=words)
            self.cur_words = words
        return self.word_bits * words

    def warmup(self, graph, seed: int = 1) -> None:
        """One full pass per slot and per width, so that workspaces, scratch
        rows and the slots' captured pass graphs exist before timing (and the
        graph's source grouping data, computed on its first use)."""
        if self.group:
            graph.source_order(graph.select_sources(seed, 2))
        words = self.base_words
        while True:
            self.ctx.set_tuning(words=words)
            self.cur_words = words
            for s in range(self.nslots):
                self.ctx.slot_launch(s, graph, graph.select_sources(seed + s, self.word_bits * words), None)
            for s in range(self.nslots):
                self.ctx.slot_poll(s, wait=True)
            if words >= self.max_words:
                break
            words *= 2

    def _collect(self, slot: int, wait: bool) -> bool:
        done, st, dig = self.ctx.slot_poll(slot, wait=wait)
        if not done:
            return False
        now = self.clock()
        self.edges += st["edges_traversed"]
        for r, (q, j) in enumerate(self.slot_rows[slot]):
            if q.want == "digest":
                q.digest[q.order[j]] = dig[r]
            q.rows_done += 1
            if q.rows_done == q.k:
                q.done_at = now
                self.completed.append(q)
        self.slot_rows[slot] = None
        return True

    def step(self, wait: bool = False) -> int:
        """Collects finished passes, admits waiting queries, fills idle slots.
        Returns the number of passes in flight."""
        for s in range(self.nslots):
            if self.slot_rows[s] is not None:
                self._collect(s, wait=False)
        self._admit()
        for s in range(self.nslots):
            if self.slot_rows[s] is None and not self._launch(s) and s >= self.express:
                break  # nothing waits (an express slot may only lack small queries)
        busy = [s for s in range(self.nslots) if self.slot_rows[s] is not None]
        if not busy and self.admit_q and not self.waiting:
            raise RuntimeError("queries wait for device memory that nothing in flight will free "
                               "(tables of finished queries are still held)")
        if wait and busy:
            # block on the pass that started first
            self._collect(min(busy, key=lambda s: self.slot_pass[s]), wait=True)
        return sum(r is not None for r in self.slot_rows)

    def pending(self) -> bool:
        return bool(self.admit_q) or bool(self.waiting) or any(r is not None for r in self.slot_rows)

    def drain(self) -> None:
        while self.pending():
            self.step(wait=True)

    def run_trace(self, trace) -> dict:
        """Replays (arrival_offset_s, graph, sources, want) entries in real time
        and returns throughput and latency percentiles."""
        trace = sorted(trace, key=lambda x: x[0])
        t0 = self.clock()
        i = 0
        first = len(self.completed)
        while i < len(trace) or self.pending():
            now = self.clock() - t0
            while i < len(trace) and trace[i][0] <= now:
                off, g, src, want = trace[i]
                self.submit(g, src, want=want, arrival=t0 + off)
                i += 1
            self.step(wait=False)
            if i < len(trace) and not self.pending():
                time.sleep(max(0.0, min(0.001, trace[i][0] - (self.clock() - t0))))
        span = self.clock() - t0
        qs = self.completed[first:]
        lat = np.array([q.latency_s for q in qs]) if qs else np.zeros(1)
        return {
            "queries": len(qs), "passes": self.passes, "seconds": span,
            "gteps": self.edges / span / 1e9 if span > 0 else 0.0,
            "p50_ms": float(np.percentile(lat, 50) * 1e3), "p99_ms": float(np.percentile(lat, 99) * 1e3),
            "mean_ms": float(lat.mean() * 1e3), "max_ms": float(lat.max() * 1e3),
        }


def poisson_trace(graphs, rate_per_s: float, count: int, seed: int, kmax: int = 4096, want: str = "digest"):
    """Seeded arrivals: exponential gaps at rate_per_s, k log-uniform in
    [1, kmax], sources drawn from the query's graph (xb_select_sources)."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for i in range(count):
        t += float(rng.exponential(1.0 / rate_per_s))
        g = graphs[int(rng.integers(len(graphs)))]
        k = int(np.floor(np.exp(rng.uniform(0.0, np.log(kmax + 1.0)))))
        k = max(1, min(kmax, k))
        out.append((t, g, g.select_sources(seed * 7919 + i, k), want))
    return out
