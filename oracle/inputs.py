"""Seeded benchmark inputs for the CPU arms, built without the product library.

TEST AND BENCHMARK INFRASTRUCTURE ONLY.  bench.py's reference arm times the
reference's own CPU BFS (oracle/_ref) and must not load libxbtrav.so on its
way there, so the graph and the sources it traverses are rebuilt here in
numpy, following the same published recipes as the product's host generator:

  R-MAT (Chakrabarti, Zhan, Faloutsos 2004): for every sample i, a splitmix64
  stream (Steele, Lea, Flood 2014) seeded by a per-sample counter hash picks
  one quadrant per level with probabilities a, b, c, 1-a-b-c; the pairs are
  symmetrised, self-loops and duplicates removed, adjacency sorted ascending.
  Sources: a partial Fisher-Yates shuffle of the vertices of non-zero degree,
  driven by one splitmix64 stream.

tests/test_oracle_inputs.py checks that both give the product generator's
exact CSR and source lists.
"""
from __future__ import annotations

import os
from concurrent.futures import ThreadPoolExecutor

import numpy as np

_GOLDEN = np.uint64(0x9E3779B97F4A7C15)
_M1 = np.uint64(0xBF58476D1CE4E5B9)
_M2 = np.uint64(0x94D049BB133111EB)
_SAMPLE_XOR = 0x5851F42D4C957F2D
_SAMPLE_MUL = np.uint64(0xD1342543DE82EF95)
_MASK64 = (1 << 64) - 1


def _mix(z: np.ndarray) -> np.ndarray:
    """splitmix64 output function of an already advanced state (vectorised)."""
    z = (z ^ (z >> np.uint64(30))) * _M1
    z = (z ^ (z >> np.uint64(27))) * _M2
    return z ^ (z >> np.uint64(31))


def _splitmix_scalar(state: int) -> tuple[int, int]:
    """(new state, output) of one splitmix64 step on a Python int."""
    state = (state + 0x9E3779B97F4A7C15) & _MASK64
    z = state
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & _MASK64
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & _MASK64
    return state, z ^ (z >> 31)


def _rmat_pairs(scale: int, seed: int, lo: int, hi: int, a: float, ab: float, abc: float):
    """(u, v) of samples lo..hi-1."""
    _, h = _splitmix_scalar(seed ^ _SAMPLE_XOR)
    with np.errstate(over="ignore"):
        i = np.arange(lo, hi, dtype=np.uint64)
        s = _mix(np.uint64(h) + i * _SAMPLE_MUL + _GOLDEN)  # per-sample stream state
        u = np.zeros(hi - lo, np.uint32)
        v = np.zeros(hi - lo, np.uint32)
        for level in range(scale):
            s = s + _GOLDEN
            r = (_mix(s) >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)
            bit = np.uint32(1 << (scale - 1 - level))
            set_v = ((r >= a) & (r < ab)) | (r >= abc)
            set_u = r >= ab
            v |= np.where(set_v, bit, np.uint32(0))
            u |= np.where(set_u, bit, np.uint32(0))
    return u, v


def _csr_from_pairs(n: int, u: np.ndarray, v: np.ndarray, threads: int) -> tuple[np.ndarray, np.ndarray]:
    """Symmetrised, loop-free, duplicate-free CSR with sorted adjacency."""
    u = u.astype(np.int64)
    v = v.astype(np.int64)
    keep = u != v
    u, v = u[keep], v[keep]
    keys = np.concatenate([u * n + v, v * n + u])  # (row, column) of both directions
    del u, v
    # sort + unique in parallel: bucket the keys by the high bits of their
    # row (a stable radix argsort of small ints), then sort each bucket
    shift = max(0, int(n - 1).bit_length() - 10)
    bucket = ((keys // n) >> np.int64(shift)).astype(np.uint16)
    order = np.argsort(bucket, kind="stable")
    edges = np.concatenate([[0], np.cumsum(np.bincount(bucket))])
    del bucket
    keys = keys[order]
    del order
    with ThreadPoolExecutor(max_workers=threads) as ex:
        parts = list(ex.map(lambda j: np.unique(keys[edges[j]:edges[j + 1]]), range(len(edges) - 1)))
    keys = np.concatenate(parts) if parts else np.zeros(0, np.int64)
    del parts
    src = keys // n
    ci = (keys - src * n).astype(np.int32)
    ro = np.zeros(n + 1, np.int64)
    np.cumsum(np.bincount(src, minlength=n), out=ro[1:])
    return ro, ci


def _threads(threads: int) -> int:
    return threads if threads > 0 else (os.cpu_count() or 1)


def rmat_csr(scale: int, edge_factor: int, a: float = 0.57, b: float = 0.19, c: float = 0.19, seed: int = 0x5EED,
             threads: int = 0) -> tuple[np.ndarray, np.ndarray]:
    """Undirected R-MAT CSR: (row offsets int64 [n+1], column indices int32)."""
    n = 1 << scale
    ns = n * edge_factor
    ab, abc = a + b, a + b + c
    chunk = 1 << 22
    bounds = [(lo, min(ns, lo + chunk)) for lo in range(0, ns, chunk)]
    threads = _threads(threads)
    with ThreadPoolExecutor(max_workers=threads) as ex:
        parts = list(ex.map(lambda r: _rmat_pairs(scale, seed, r[0], r[1], a, ab, abc), bounds))
    u = np.concatenate([p[0] for p in parts])
    v = np.concatenate([p[1] for p in parts])
    del parts
    return _csr_from_pairs(n, u, v, threads)


def _er_pairs(n: int, seed: int, lo: int, hi: int):
    _, h = _splitmix_scalar(seed ^ _SAMPLE_XOR)
    with np.errstate(over="ignore"):
        i = np.arange(lo, hi, dtype=np.uint64)
        s = _mix(np.uint64(h) + i * _SAMPLE_MUL + _GOLDEN)
        s = s + _GOLDEN
        u = _mix(s) % np.uint64(n)
        s = s + _GOLDEN
        v = _mix(s) % np.uint64(n)
    return u, v


def er_csr(n: int, m_pairs: int, seed: int = 0x5EED, threads: int = 0) -> tuple[np.ndarray, np.ndarray]:
    """Uniform random graph of m_pairs sampled vertex pairs, same cleaning."""
    chunk = 1 << 22
    bounds = [(lo, min(m_pairs, lo + chunk)) for lo in range(0, m_pairs, chunk)]
    threads = _threads(threads)
    with ThreadPoolExecutor(max_workers=threads) as ex:
        parts = list(ex.map(lambda r: _er_pairs(n, seed, r[0], r[1]), bounds))
    u = np.concatenate([p[0] for p in parts]) if parts else np.zeros(0, np.uint64)
    v = np.concatenate([p[1] for p in parts]) if parts else np.zeros(0, np.uint64)
    return _csr_from_pairs(n, u, v, threads)


def select_sources(ro: np.ndarray, seed: int, k: int) -> np.ndarray:
    """k distinct vertices of non-zero degree (partial Fisher-Yates)."""
    cand = np.nonzero(np.diff(ro) > 0)[0].astype(np.int32)
    cnt = len(cand)
    if k > cnt:
        raise ValueError(f"asked for {k} sources but only {cnt} vertices have edges")
    out = np.empty(k, np.int32)
    state = seed & _MASK64
    for i in range(k):
        state, r = _splitmix_scalar(state)
        j = i + r % (cnt - i)
        cand[i], cand[j] = cand[j], cand[i]
        out[i] = cand[i]
    return out


def symmetric_weights(ro: np.ndarray, ci: np.ndarray, seed: int, wmin: int = 1, wmax: int = 100) -> np.ndarray:
    """Seeded int32 edge weights in [wmin, wmax], one per column index, equal
    for both directions of an edge (a hash of the unordered pair)."""
    ro = np.ascontiguousarray(ro, dtype=np.int64)
    ci = np.ascontiguousarray(ci, dtype=np.int64)
    if wmax < wmin:
        raise ValueError("wmax < wmin")
    u = np.repeat(np.arange(len(ro) - 1, dtype=np.int64), np.diff(ro))
    a, b = np.minimum(u, ci), np.maximum(u, ci)
    h = (a * 1000003 + b * 7919 + int(seed) % (1 << 31)) % (wmax - wmin + 1)
    return (h + wmin).astype(np.int32)
