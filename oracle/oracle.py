"""CPU oracle loader -- TEST INFRASTRUCTURE ONLY.

Loads the C restatement (oracle/liboracle_msbfs.so, built from
oracle/msbfs_oracle.c) and, where it was built, the reference's own code
compiled from the reference sources into oracle/_ref/ (Ligra BFS and
xblossom::Graph::findShortestPath).  Only tests/, __graft_entry__.smoke()
and bench.py's CPU-baseline legs import this module; the product never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle_msbfs.so")
REF_DIR = os.path.join(HERE, "_ref")
LIGRA_SO = os.path.join(REF_DIR, "libligra_bfs_ref.so")
XGRAPH_SO = os.path.join(REF_DIR, "libxgraph_fifo_ref.so")
MSSSP_SO = os.path.join(REF_DIR, "libligra_msssp_ref.so")
MATCH_SO = os.path.join(REF_DIR, "libxb_match_ref.so")

RULE_MINID = 0
RULE_FIFO = 1

_o = None
_lig = None
_xg = None


def build(ref_root: str | None = None) -> None:
    """Builds the C restatement, and the reference checkers when a reference
    checkout is given (ref_root, else the XB_REF_ROOT environment variable)."""
    subprocess.run(["make", "-s", "-C", HERE, "all"], check=True)
    root = ref_root or os.environ.get("XB_REF_ROOT", "")
    if root and os.path.isdir(os.path.join(root, "apps")):
        subprocess.run(["make", "-s", "-C", HERE, "ref", f"REF_ROOT={root}"], check=True)


def _load() -> C.CDLL:
    global _o
    if _o is None:
        if not os.path.exists(ORACLE_SO):
            build()
        L = C.CDLL(ORACLE_SO)
        L.oracle_msbfs.restype = C.c_int
        L.oracle_msbfs.argtypes = [C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.c_int32,
                                   C.c_void_p, C.c_void_p, C.POINTER(C.c_longlong), C.POINTER(C.c_longlong),
                                   C.c_int32]
        L.oracle_check_parents.restype = C.c_longlong
        L.oracle_check_parents.argtypes = [C.c_int64, C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p]
        _o = L
    return _o


def msbfs(ro: np.ndarray, ci: np.ndarray, sources: np.ndarray, rule: int = RULE_MINID, threads: int = 0,
          want_tables: bool = True):
    """Plain multi-source BFS on the CPU.  Returns (level, parent, edges_traversed, reached)."""
    ro = np.ascontiguousarray(ro, dtype=np.int64)
    ci = np.ascontiguousarray(ci, dtype=np.int32)
    src = np.ascontiguousarray(sources, dtype=np.int32)
    n, k = len(ro) - 1, len(src)
    lvl = np.empty((k, n), np.int32) if want_tables else None
    par = np.empty((k, n), np.int32) if want_tables else None
    e, r = C.c_longlong(), C.c_longlong()
    if threads <= 0:
        threads = os.cpu_count() or 1
    rc = _load().oracle_msbfs(n, ro.ctypes.data, ci.ctypes.data if len(ci) else None, src.ctypes.data, k, rule,
                              lvl.ctypes.data if want_tables else None, par.ctypes.data if want_tables else None,
                              C.byref(e), C.byref(r), threads)
    if rc != 0:
        raise ValueError("oracle_msbfs rejected its arguments")
    return lvl, par, e.value, r.value


def msssp(ro, ci, weights, sources) -> np.ndarray:
    """Multi-source SSSP distances (float32, n) on the CPU: the restatement of
    Ligra's MultiSSSP (one shared distance array, every source at 0)."""
    ro = np.ascontiguousarray(ro, dtype=np.int64)
    ci = np.ascontiguousarray(ci, dtype=np.int32)
    w = np.ascontiguousarray(weights, dtype=np.int32)
    src = np.ascontiguousarray(sources, dtype=np.int32)
    dist = np.empty(len(ro) - 1, np.float32)
    L = _load()
    L.oracle_msssp.restype = C.c_int
    L.oracle_msssp.argtypes = [C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p]
    rc = L.oracle_msssp(len(ro) - 1, ro.ctypes.data, ci.ctypes.data if len(ci) else None,
                        w.ctypes.data if len(w) else None, src.ctypes.data, len(src), dist.ctypes.data)
    if rc != 0:
        raise ValueError("oracle_msssp rejected its arguments")
    return dist


def check_parents(ro, ci, s: int, level_row: np.ndarray, parent_row: np.ndarray) -> int:
    """Number of entries of parent_row that are not a valid BFS predecessor under level_row."""
    ro = np.ascontiguousarray(ro, dtype=np.int64)
    ci = np.ascontiguousarray(ci, dtype=np.int32)
    lv = np.ascontiguousarray(level_row, dtype=np.int32)
    pr = np.ascontiguousarray(parent_row, dtype=np.int32)
    return int(_load().oracle_check_parents(len(ro) - 1, ro.ctypes.data, ci.ctypes.data if len(ci) else None, s,
                                            lv.ctypes.data, pr.ctypes.data))


# ---- the reference's own code (built from its sources) ---------------------

def ligra_available() -> bool:
    return os.path.exists(LIGRA_SO)


def xgraph_available() -> bool:
    return os.path.exists(XGRAPH_SO)


def max_match(ro, ci, init=None) -> tuple[int, np.ndarray]:
    """Maximum-cardinality matching (Edmonds' blossom algorithm restated in
    C): (size, mate) with mate[v] = -1 for exposed vertices.  init: an
    optional starting matching (mate array)."""
    ro = np.ascontiguousarray(ro, dtype=np.int64)
    ci = np.ascontiguousarray(ci, dtype=np.int32)
    n = len(ro) - 1
    mate = np.full(n, -1, np.int32) if init is None else np.array(init, dtype=np.int32, copy=True)
    L = _load()
    L.oracle_max_match.restype = C.c_int64
    L.oracle_max_match.argtypes = [C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p]
    size = L.oracle_max_match(n, ro.ctypes.data, ci.ctypes.data if len(ci) else None, mate.ctypes.data)
    if size < 0:
        raise ValueError("oracle_max_match rejected its arguments")
    return int(size), mate


def alt_forest(ro, ci, mate) -> tuple[np.ndarray, np.ndarray, np.ndarray, int]:
    """Alternating forest of a matching from every exposed vertex (level,
    parent, owner per vertex; -1 unreached) and the number of rounds."""
    ro = np.ascontiguousarray(ro, dtype=np.int64)
    ci = np.ascontiguousarray(ci, dtype=np.int32)
    mate = np.ascontiguousarray(mate, dtype=np.int32)
    n = len(ro) - 1
    lv, pr, ow = (np.empty(n, np.int32) for _ in range(3))
    L = _load()
    L.oracle_alt_forest.restype = C.c_int64
    L.oracle_alt_forest.argtypes = [C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                    C.c_void_p]
    r = L.oracle_alt_forest(n, ro.ctypes.data, ci.ctypes.data if len(ci) else None, mate.ctypes.data,
                            lv.ctypes.data, pr.ctypes.data, ow.ctypes.data)
    if r < 0:
        raise ValueError("oracle_alt_forest rejected its arguments")
    return lv, pr, ow, int(r)


def ref_match_available() -> bool:
    return os.path.exists(MATCH_SO)


def ref_max_match(ro, ci, threads: int = 1, init=None) -> tuple[int, np.ndarray]:
    """The reference's own CPU maximum-matching engine
    (apps/xb/src/xblsm_cpu/par_pro_pernode.cu) built into oracle/_ref."""
    ro = np.ascontiguousarray(ro, dtype=np.int64)
    ci = np.ascontiguousarray(ci, dtype=np.int32)
    n = len(ro) - 1
    mate = np.full(n, -1, np.int32) if init is None else np.array(init, dtype=np.int32, copy=True)
    L = C.CDLL(MATCH_SO)
    L.xb_ref_max_match.restype = C.c_int64
    L.xb_ref_max_match.argtypes = [C.c_int64, C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p]
    size = L.xb_ref_max_match(n, ro.ctypes.data, ci.ctypes.data if len(ci) else None, threads, mate.ctypes.data)
    if size < 0:
        raise ValueError("xb_ref_max_match failed")
    return int(size), mate


def check_matching(ro, ci, mate) -> int:
    """Number of violations: mate not symmetric, or a matched pair that is not an edge."""
    ro = np.asarray(ro, dtype=np.int64)
    ci = np.asarray(ci, dtype=np.int32)
    mate = np.asarray(mate)
    n = len(ro) - 1
    bad = 0
    for v in np.nonzero(mate >= 0)[0]:
        m = int(mate[v])
        if m >= n or mate[m] != v or m == v:
            bad += 1
            continue
        adj = ci[ro[v]:ro[v + 1]]
        i = np.searchsorted(adj, m)
        if i >= len(adj) or adj[i] != m:
            bad += 1
    return bad


def ligra_msssp_available() -> bool:
    return os.path.exists(MSSSP_SO)


def ligra_msssp(ro, ci, weights, sources, threads: int = 1) -> np.ndarray:
    """Reference Ligra MultiSSSP (apps/ligra/apps/MultiSSSP.C) distances."""
    ro = np.ascontiguousarray(ro, dtype=np.int64)
    ci = np.ascontiguousarray(ci, dtype=np.int32)
    w = np.ascontiguousarray(weights, dtype=np.int32)
    src = np.ascontiguousarray(sources, dtype=np.int32)
    L = C.CDLL(MSSSP_SO)
    L.ligra_ref_msssp.restype = C.c_int
    L.ligra_ref_msssp.argtypes = [C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p,
                                  C.c_int32]
    dist = np.empty(len(ro) - 1, np.float32)
    rc = L.ligra_ref_msssp(len(ro) - 1, ro.ctypes.data, ci.ctypes.data if len(ci) else None,
                           w.ctypes.data if len(w) else None, src.ctypes.data, len(src), dist.ctypes.data, threads)
    if rc != 0:
        raise ValueError("ligra_ref_msssp rejected its arguments")
    return dist


def _ligra() -> C.CDLL:
    global _lig
    if _lig is None:
        L = C.CDLL(LIGRA_SO)
        L.ligra_ref_bfs.restype = C.c_double
        L.ligra_ref_bfs.argtypes = [C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p,
                                    C.POINTER(C.c_int64), C.c_int32]
        L.ligra_ref_workers.restype = C.c_int32
        _lig = L
    return _lig


def ligra_bfs(ro, ci, sources, threads: int = 0, want_parents: bool = True):
    """Reference Ligra BFS (apps/ligra/apps/BFS.C).  Returns (parents uint32 (k,n) or None, seconds, edges)."""
    ro = np.ascontiguousarray(ro, dtype=np.int64)
    ci = np.ascontiguousarray(ci, dtype=np.int32)
    src = np.ascontiguousarray(sources, dtype=np.int32)
    n, k = len(ro) - 1, len(src)
    par = np.empty((k, n), np.uint32) if want_parents else None
    e = C.c_int64()
    secs = _ligra().ligra_ref_bfs(n, ro.ctypes.data, ci.ctypes.data if len(ci) else None, src.ctypes.data, k,
                                  par.ctypes.data if want_parents else None, C.byref(e), threads)
    if secs < 0:
        raise ValueError("ligra_ref_bfs rejected its arguments")
    return par, secs, e.value


def ligra_workers() -> int:
    return int(_ligra().ligra_ref_workers())


def _xgraph() -> C.CDLL:
    global _xg
    if _xg is None:
        L = C.CDLL(XGRAPH_SO)
        L.xgraph_ref_paths.restype = C.c_int32
        L.xgraph_ref_paths.argtypes = [C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64,
                                       C.c_void_p, C.c_void_p]
        _xg = L
    return _xg


def xgraph_paths(ro, ci, src: np.ndarray, dst: np.ndarray):
    """Reference findShortestPath (apps/xb/src/include/graph/xgraph.h:155-191) per (src, dst) pair.

    Returns (level, fifo_parent) per pair.  dst must be reachable from src."""
    ro32 = np.ascontiguousarray(ro, dtype=np.int32)
    ci32 = np.ascontiguousarray(ci, dtype=np.int32)
    s = np.ascontiguousarray(src, dtype=np.int32)
    d = np.ascontiguousarray(dst, dtype=np.int32)
    lv = np.empty(len(s), np.int32)
    pr = np.empty(len(s), np.int32)
    rc = _xgraph().xgraph_ref_paths(len(ro32) - 1, ro32.ctypes.data, ci32.ctypes.data if len(ci32) else None,
                                    s.ctypes.data, d.ctypes.data, len(s), lv.ctypes.data, pr.ctypes.data)
    if rc != 0:
        raise ValueError("xgraph_ref_paths rejected its arguments")
    return lv, pr


def row_entry_hash(v: np.ndarray, level: np.ndarray, parent: np.ndarray) -> np.ndarray:
    """Hash of (vertex, level, parent) entries as the serving digests define
    it: the splitmix64 finalizer of (v * 0x9E3779B97F4A7C15) XOR ((uint32 level
    << 32) | uint32 parent), as uint64."""
    with np.errstate(over="ignore"):
        z = v.astype(np.uint64) * np.uint64(0x9E3779B97F4A7C15)
        z ^= (level.astype(np.int64).astype(np.uint64) & np.uint64(0xFFFFFFFF)) << np.uint64(32)
        z ^= parent.astype(np.int64).astype(np.uint64) & np.uint64(0xFFFFFFFF)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        return z ^ (z >> np.uint64(31))


def row_digests(level: np.ndarray, parent: np.ndarray) -> np.ndarray:
    """Serving digests of (k, n) level / parent tables: int64 (k, 4) rows of
    reached, level sum, row hash (wrapping sum of row_entry_hash over reached
    vertices, as the int64 with the same bits) and depth."""
    level = np.atleast_2d(level)
    parent = np.atleast_2d(parent)
    k, n = level.shape
    out = np.zeros((k, 4), np.int64)
    v = np.arange(n, dtype=np.int64)
    for r in range(k):
        m = level[r] >= 0
        h = row_entry_hash(v[m], level[r][m], parent[r][m])
        with np.errstate(over="ignore"):
            out[r, 2] = np.sum(h, dtype=np.uint64).astype(np.int64)
        out[r, 0] = int(m.sum())
        out[r, 1] = int(level[r][m].astype(np.int64).sum())
        out[r, 3] = int(level[r][m].max()) if m.any() else -1
    return out
