"""Serving loop with continuous batching over the engine's slots.

Queries (a graph and a set of sources) arrive at any time.  The server keeps
the graphs resident, admits queries by free HBM, and packs the sources of
whatever queries are waiting -- several queries per pass, a query spread over
many passes -- into passes of up to word_bits x words sources that run on its
slots (xb_slot_launch: one pass in flight per slot, each slot with its own
stream and workspace, so passes of different slots overlap on the device).  A
query that arrives while others are on the GPU joins the next pass any slot
starts; nothing waits for a batch to fill.

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
    passes: set = field(default_factory=set)

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
    def __init__(self, ctx, slots: int = 4, reserve_bytes: int = 4 << 30, clock=time.perf_counter):
        import torch

        self.torch = torch
        self.ctx = ctx
        self.nslots = slots
        self.reserve = reserve_bytes
        self.clock = clock
        t = ctx.tuning()
        self.rows_per_pass = t["word_bits"] * t["words"]
        self.dev = torch.device("cuda", ctx.device)
        self.admit_q = collections.deque()      # queries waiting for memory
        self.rows = collections.OrderedDict()   # graph handle -> deque of (query, source index)
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
        key = q.graph._h.value
        dq = self.rows.setdefault(key, collections.deque())
        dq.extend((q, j) for j in range(q.k))

    # slots ------------------------------------------------------------------
    def _launch(self, slot: int) -> bool:
        """Starts a pass on an idle slot from the graph whose waiting row is oldest."""
        best, best_t = None, None
        for key, dq in self.rows.items():
            if dq and (best is None or dq[0][0].admitted < best_t):
                best, best_t = key, dq[0][0].admitted
        if best is None:
            return False
        dq = self.rows[best]
        take = [dq.popleft() for _ in range(min(self.rows_per_pass, len(dq)))]
        g = take[0][0].graph
        src = np.array([q.sources[j] for q, j in take], dtype=np.int32)
        rows = []
        for q, j in take:
            rows.append(None if q.want == "digest" else (q.level[j].data_ptr(), q.parent[j].data_ptr()))
        self.ctx.slot_launch(slot, g, src, rows)
        self.slot_rows[slot] = take
        self.passes += 1
        self.slot_pass[slot] = self.passes
        return True

    def _collect(self, slot: int, wait: bool) -> bool:
        done, st, dig = self.ctx.slot_poll(slot, wait=wait)
        if not done:
            return False
        now = self.clock()
        self.edges += st["edges_traversed"]
        for r, (q, j) in enumerate(self.slot_rows[slot]):
            if q.want == "digest":
                q.digest[j] = dig[r]
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
            if self.slot_rows[s] is None and not self._launch(s):
                break
        busy = [s for s in range(self.nslots) if self.slot_rows[s] is not None]
        if not busy and self.admit_q and not any(self.rows.values()):
            raise RuntimeError("queries wait for device memory that nothing in flight will free "
                               "(tables of finished queries are still held)")
        if wait and busy:
            # block on the pass that started first
            self._collect(min(busy, key=lambda s: self.slot_pass[s]), wait=True)
        return sum(r is not None for r in self.slot_rows)

    def pending(self) -> bool:
        return bool(self.admit_q) or any(self.rows.values()) or any(r is not None for r in self.slot_rows)

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
