"""Generates tests/golden/*.npz from the reference's own BFS code.

Run where the reference tree is mounted (it builds oracle/_ref/ from the
reference sources first):

    python tests/golden/make_golden.py <reference root>

For every fixture graph it records
  ro, ci, sources                          the input (int64 / int32 CSR)
  ligra_parent  (k, n) int64, -1 = unreached
      Parents from Ligra's BFS_F + edgeMap (apps/ligra/apps/BFS.C:26-53), the
      reference's BFS baseline; schedule dependent (CAS), run on 1 thread so
      the fixture is reproducible.
  pair_src_idx, pair_dst, pair_level, pair_parent
      For every (source, vertex) pair Ligra reached: the path returned by
      xblossom::Graph::findShortestPath (apps/xb/src/include/graph/xgraph.h:155-191),
      its length (= the level) and the vertex before the destination (= the
      FIFO-first-discoverer parent).  Pairs whose source has no edges are
      skipped (findShortestPath returns an empty path for vertices without an
      adjacency list).
The graphs are built with the product's seeded generators or by hand; the
fixture stores the CSR itself, so later generator changes do not affect it.
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "xblossom-sigmetrics27-ae_b200"))

from oracle import oracle as O  # noqa: E402
import xbtrav  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))


def csr_from_edges(n: int, edges) -> tuple[np.ndarray, np.ndarray]:
    adj = [set() for _ in range(n)]
    for u, v in edges:
        if u != v:
            adj[u].add(v)
            adj[v].add(u)
    ro = np.zeros(n + 1, np.int64)
    ci = []
    for v in range(n):
        nb = sorted(adj[v])
        ci.extend(nb)
        ro[v + 1] = ro[v] + len(nb)
    return ro, np.array(ci, np.int32)


def fixtures():
    rng = np.random.default_rng(20261203)
    out = {}
    g = xbtrav.HostCSR.rmat(8, 4, seed=101)
    ro, ci = g.arrays()
    out["rmat8_ef4"] = (ro, ci, xbtrav.select_sources_csr(ro, 102, 16))
    g = xbtrav.HostCSR.rmat(10, 8, seed=201)
    ro, ci = g.arrays()
    out["rmat10_ef8"] = (ro, ci, xbtrav.select_sources_csr(ro, 202, 40))
    g = xbtrav.HostCSR.er(600, 420, seed=301)  # sparse: many components
    ro, ci = g.arrays()
    out["er600_sparse"] = (ro, ci, xbtrav.select_sources_csr(ro, 302, 70))
    n = 50
    ro, ci = csr_from_edges(n, [(i, i + 1) for i in range(n - 1)])
    out["path50"] = (ro, ci, np.array([0, 49, 25, 7, 0], np.int32))  # duplicate source on purpose
    n = 33
    ro, ci = csr_from_edges(n, [(0, i) for i in range(1, n)])
    out["star33"] = (ro, ci, np.array([0, 5, 32], np.int32))
    n = 8
    ro, ci = csr_from_edges(n, [(i, j) for i in range(n) for j in range(i + 1, n)])
    out["clique8"] = (ro, ci, np.arange(8, dtype=np.int32))
    # two triangles, a tail and isolated vertices; sources include an isolated one
    n = 12
    ro, ci = csr_from_edges(n, [(0, 1), (1, 2), (2, 0), (4, 5), (5, 6), (6, 4), (6, 7), (7, 8)])
    out["islands12"] = (ro, ci, np.array([0, 4, 8, 3, 11], np.int32))
    # cycle with chords: several equal-length paths (parent tie-breaks matter)
    n = 64
    e = [(i, (i + 1) % n) for i in range(n)] + [(i, (i + 8) % n) for i in range(0, n, 4)]
    ro, ci = csr_from_edges(n, e)
    out["cycle64_chords"] = (ro, ci, rng.choice(n, 9, replace=False).astype(np.int32))
    # deep: a 200-vertex path (levels beyond 7 bit-planes: depth 199)
    n = 200
    ro, ci = csr_from_edges(n, [(i, i + 1) for i in range(n - 1)])
    out["path200"] = (ro, ci, np.array([0, 199, 100], np.int32))
    # no edges at all
    ro = np.zeros(6, np.int64)
    out["empty5"] = (ro, np.zeros(0, np.int32), np.array([0, 3], np.int32))
    return out


def main() -> None:
    if len(sys.argv) < 2:
        sys.exit("usage: make_golden.py <reference root>")
    O.build(sys.argv[1])
    assert O.ligra_available() and O.xgraph_available(), "reference checkers were not built"
    for name, (ro, ci, src) in fixtures().items():
        n, k = len(ro) - 1, len(src)
        par, _, _ = O.ligra_bfs(ro, ci, src, threads=1)
        lp = par.astype(np.int64)
        lp[par == np.uint32(0xFFFFFFFF)] = -1
        deg = np.diff(ro)
        S, D = np.nonzero(lp >= 0)
        keep = deg[src[S]] > 0
        S, D = S[keep], D[keep]
        if len(S):
            pl, pp = O.xgraph_paths(ro, ci, src[S], D)
        else:
            pl = pp = np.zeros(0, np.int32)
        np.savez_compressed(os.path.join(OUT, f"{name}.npz"), ro=ro, ci=ci, sources=src, ligra_parent=lp,
                            pair_src_idx=S.astype(np.int32), pair_dst=D.astype(np.int32),
                            pair_level=pl.astype(np.int32), pair_parent=pp.astype(np.int32))
        print(f"{name}: n={n} m={len(ci)} k={k} pairs={len(S)}")


if __name__ == "__main__":
    main()
