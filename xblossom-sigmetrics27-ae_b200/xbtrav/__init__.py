"""xbtrav -- Python binding of libxbtrav.so over its C ABI (include/xbtrav.h).

The binding is a thin ctypes layer: every call goes through the extern "C"
entry points of the in-tree shared library, the same ones a C/C++ caller of
the reference-style API binds.  There is no Python or CPU fallback for the
traversal: if the library or a CUDA device is missing the calls raise.

Reference-facing names (paths relative to the X-Blossom project):
  HostCSR.load_text(row, col)   <- zblossom::HGraph(row_path, col_path)
                                   apps/xb/src/include/graph/hgraph.h:37-48
  Context.upload(csr)           <- zblossom::DGraph(const HGraph&)
                                   apps/xb/src/include/graph/dgraph.h:50-63
  Context.traverse_batched(...) <- (no counterpart: many queries per launch)
  Context.traverse(...)         <- the expand phase of
                                   apps/xb/src/xblsm_gpu/xblossom_gpu_engine_10.cu:270-359
                                   returning level (root_distance_) and parent
                                   (PathTable) tables per source.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, field

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(os.path.dirname(_HERE), "libxbtrav.so")

XB_OK = 0
XB_ERR_ARG = -1
XB_ERR_OOM = -2
XB_ERR_CAPACITY = -3
XB_ERR_TIMEOUT = -4
XB_ERR_CUDA = -5
XB_ERR_IO = -6
XB_ERR_NODEV = -7
XB_ERR_STATE = -8

XB_MODE_PLAIN = 0
XB_MODE_ALTERNATING = 1
XB_OUT_DEVICE = 1
XB_SOURCES_DEVICE = 2
XB_PARENT_FIFO = 4
XB_MAX_SLOTS = 16
SLOT_MAX_ROWS = 256  # sources per slot pass at most (64 per word x 4 words)


class XbError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"xbtrav status {status}: {msg}")
        self.status = status


class XbStats(C.Structure):
    _fields_ = [
        ("edges_traversed", C.c_int64),
        ("reached", C.c_int64),
        ("edges_scanned", C.c_int64),
        ("vertices_scanned", C.c_int64),
        ("vertices_swept", C.c_int64),
        ("parent_edges_scanned", C.c_int64),
        ("algo_bytes", C.c_int64),
        ("levels", C.c_int32),
        ("push_levels", C.c_int32),
        ("pull_levels", C.c_int32),
        ("batches", C.c_int32),
        ("device_ms", C.c_double),
        ("class_launches", C.c_int64 * 3),
        ("class_ms", C.c_double * 3),
        ("class_bytes", C.c_int64 * 3),
    ]

    def as_dict(self) -> dict:
        d = {}
        for name, _ in self._fields_:
            v = getattr(self, name)
            d[name] = list(v) if hasattr(v, "__len__") else v
        return d


class XbTuning(C.Structure):
    _fields_ = [
        ("word_bits", C.c_int32),
        ("words", C.c_int32),
        ("pull_alpha", C.c_float),
        ("heavy_degree", C.c_int32),
        ("timing", C.c_int32),
        ("chains", C.c_int32),
        ("level_cap", C.c_int32),
        ("tile", C.c_int32),
        ("workspace_cap", C.c_int64),
        ("push_beta", C.c_float),
        ("source_order", C.c_int32),
    ]


class XbRowDigest(C.Structure):
    _fields_ = [
        ("reached", C.c_int64),
        ("level_sum", C.c_int64),
        ("row_hash", C.c_int64),
        ("depth", C.c_int32),
        ("pad", C.c_int32),
    ]


class XbBatchItem(C.Structure):
    _fields_ = [
        ("graph", C.c_void_p),
        ("sources", C.c_void_p),
        ("k", C.c_int32),
        ("flags", C.c_uint32),
        ("level", C.c_void_p),
        ("parent", C.c_void_p),
    ]


_lib = None


def lib() -> C.CDLL:
    """Loads libxbtrav.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise FileNotFoundError(f"{LIB_PATH} is missing: build it with __graft_entry__.build()")
    L = C.CDLL(LIB_PATH)
    vp, i32, i64, u64, u32 = C.c_void_p, C.c_int32, C.c_int64, C.c_uint64, C.c_uint32
    P = C.POINTER
    sig = {
        "xb_status_str": (C.c_char_p, [i32]),
        "xb_last_error": (C.c_char_p, []),
        "xb_abi_version": (i32, []),
        "xb_csr_gen_rmat": (i32, [i32, i32, C.c_double, C.c_double, C.c_double, u64, i32, P(vp)]),
        "xb_csr_gen_er": (i32, [i64, i64, u64, i32, P(vp)]),
        "xb_csr_from_arrays": (i32, [i64, vp, vp, P(vp)]),
        "xb_csr_load_text": (i32, [C.c_char_p, C.c_char_p, P(vp)]),
        "xb_csr_save_text": (i32, [vp, C.c_char_p, C.c_char_p]),
        "xb_csr_save_binary": (i32, [vp, C.c_char_p]),
        "xb_csr_load_binary": (i32, [C.c_char_p, P(vp)]),
        "xb_csr_save_ligra": (i32, [vp, C.c_char_p]),
        "xb_csr_save_mtx": (i32, [vp, C.c_char_p]),
        "xb_csr_load_mtx": (i32, [C.c_char_p, P(vp)]),
        "xb_sources_load": (i32, [C.c_char_p, vp, i32, P(i32)]),
        "xb_sources_save": (i32, [C.c_char_p, vp, i32, C.c_char_p]),
        "xb_csr_info": (i32, [vp, P(i64), P(i64), P(i64), P(i64)]),
        "xb_csr_arrays": (i32, [vp, P(vp), P(vp)]),
        "xb_csr_free": (None, [vp]),
        "xb_select_sources_csr": (i32, [i64, vp, u64, i32, vp]),
        "xb_ctx_create": (i32, [i32, P(vp)]),
        "xb_ctx_destroy": (i32, [vp]),
        "xb_ctx_set_tuning": (i32, [vp, P(XbTuning)]),
        "xb_ctx_get_tuning": (i32, [vp, P(XbTuning)]),
        "xb_ctx_workspace_bytes": (i32, [vp, P(i64)]),
        "xb_ctx_get_stream": (i32, [vp, P(vp)]),
        "xb_graph_upload": (i32, [vp, i64, vp, i32, i64, vp, P(vp)]),
        "xb_graph_from_host_csr": (i32, [vp, vp, P(vp)]),
        "xb_graph_upload_batch": (i32, [vp, i32, vp, vp, vp, P(vp)]),
        "xb_graph_load_csr_text": (i32, [vp, C.c_char_p, C.c_char_p, P(vp)]),
        "xb_graph_free": (i32, [vp]),
        "xb_graph_info": (i32, [vp, P(i64), P(i64), P(i64)]),
        "xb_select_sources": (i32, [vp, u64, i32, vp]),
        "xb_graph_source_order": (i32, [vp, vp, i32, vp]),
        "xb_traverse": (i32, [vp, vp, vp, i32, i32, vp, vp, vp, vp, u32, P(XbStats)]),
        "xb_traverse_batched": (i32, [vp, P(XbBatchItem), i32, P(XbStats)]),
        "xb_slot_launch": (i32, [vp, i32, vp, vp, i32, vp, vp]),
        "xb_slot_poll": (i32, [vp, i32, P(i32), P(XbStats), vp]),
        "xb_slot_wait": (i32, [vp, i32, P(XbStats), vp]),
        "xb_slots_release": (i32, [vp]),
        "xb_slot_set_priority": (i32, [vp, i32, i32]),
        "xb_graph_set_weights": (i32, [vp, vp, i64]),
        "xb_multi_sssp": (i32, [vp, vp, vp, i32, vp, u32, P(XbStats)]),
        "xb_max_match": (i32, [vp, vp, vp, u32, P(XbStats)]),
        "xb_graph_offset_bytes": (i32, [vp, P(i32)]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


def declared_symbols() -> list[str]:
    """Function names declared in include/*.h (parsed from the headers)."""
    import re

    inc = os.path.join(os.path.dirname(os.path.dirname(_HERE)), "include")
    names = []
    for fn in sorted(os.listdir(inc)):
        if not fn.endswith(".h"):
            continue
        text = open(os.path.join(inc, fn)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?[A-Za-z_][A-Za-z0-9_]*\s*\*?\s*(xb_[a-z0-9_]+)\s*\(", text, re.M):
            names.append(m.group(1))
    return names


def _check(st: int) -> None:
    if st != XB_OK:
        L = lib()
        msg = L.xb_last_error().decode() or L.xb_status_str(st).decode()
        raise XbError(st, msg)


class HostCSR:
    """Host-resident CSR (int64 row offsets, int32 column indices)."""

    def __init__(self, handle: int):
        self._h = C.c_void_p(handle)

    @classmethod
    def rmat(cls, scale: int, edge_factor: int, a=0.57, b=0.19, c=0.19, seed=0x5EED, threads=0) -> "HostCSR":
        h = C.c_void_p()
        _check(lib().xb_csr_gen_rmat(scale, edge_factor, a, b, c, seed, threads, C.byref(h)))
        return cls(h.value)

    @classmethod
    def er(cls, n: int, m_pairs: int, seed=0x5EED, threads=0) -> "HostCSR":
        h = C.c_void_p()
        _check(lib().xb_csr_gen_er(n, m_pairs, seed, threads, C.byref(h)))
        return cls(h.value)

    @classmethod
    def from_arrays(cls, row_offsets, col_indices) -> "HostCSR":
        ro = np.ascontiguousarray(row_offsets, dtype=np.int64)
        ci = np.ascontiguousarray(col_indices, dtype=np.int32)
        h = C.c_void_p()
        _check(lib().xb_csr_from_arrays(len(ro) - 1, ro.ctypes.data, ci.ctypes.data if len(ci) else None,
                                        C.byref(h)))
        return cls(h.value)

    @classmethod
    def load_text(cls, row_path: str, col_path: str) -> "HostCSR":
        h = C.c_void_p()
        _check(lib().xb_csr_load_text(row_path.encode(), col_path.encode(), C.byref(h)))
        return cls(h.value)

    def save_text(self, row_path: str, col_path: str) -> None:
        _check(lib().xb_csr_save_text(self._h, row_path.encode(), col_path.encode()))

    @classmethod
    def load_binary(cls, path: str) -> "HostCSR":
        h = C.c_void_p()
        _check(lib().xb_csr_load_binary(path.encode(), C.byref(h)))
        return cls(h.value)

    def save_binary(self, path: str) -> None:
        _check(lib().xb_csr_save_binary(self._h, path.encode()))

    @classmethod
    def load_mtx(cls, path: str) -> "HostCSR":
        h = C.c_void_p()
        _check(lib().xb_csr_load_mtx(path.encode(), C.byref(h)))
        return cls(h.value)

    def save_mtx(self, path: str) -> None:
        _check(lib().xb_csr_save_mtx(self._h, path.encode()))

    def save_ligra(self, path: str) -> None:
        _check(lib().xb_csr_save_ligra(self._h, path.encode()))

    def info(self) -> dict:
        n, m, md, iso = C.c_int64(), C.c_int64(), C.c_int64(), C.c_int64()
        _check(lib().xb_csr_info(self._h, C.byref(n), C.byref(m), C.byref(md), C.byref(iso)))
        return {"n": n.value, "m": m.value, "max_degree": md.value, "isolated": iso.value}

    def arrays(self) -> tuple[np.ndarray, np.ndarray]:
        """Copies of (row_offsets int64[n+1], col_indices int32[m])."""
        inf = self.info()
        ro, ci = C.c_void_p(), C.c_void_p()
        _check(lib().xb_csr_arrays(self._h, C.byref(ro), C.byref(ci)))
        r = np.ctypeslib.as_array(C.cast(ro, C.POINTER(C.c_int64)), shape=(inf["n"] + 1,)).copy()
        if inf["m"]:
            c = np.ctypeslib.as_array(C.cast(ci, C.POINTER(C.c_int32)), shape=(inf["m"],)).copy()
        else:
            c = np.zeros(0, np.int32)
        return r, c

    def close(self) -> None:
        if self._h and self._h.value:
            lib().xb_csr_free(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def load_sources(path: str) -> np.ndarray:
    """Source-list file ("#" comments, ids separated by white space)."""
    cnt = C.c_int32(0)
    st = lib().xb_sources_load(path.encode(), None, 0, C.byref(cnt))
    if st not in (XB_OK, XB_ERR_CAPACITY):
        _check(st)
    out = np.zeros(cnt.value, np.int32)
    if cnt.value:
        _check(lib().xb_sources_load(path.encode(), out.ctypes.data, cnt.value, C.byref(cnt)))
    return out


def save_sources(path: str, sources, comment: str = "") -> None:
    src = np.ascontiguousarray(sources, dtype=np.int32)
    _check(lib().xb_sources_save(path.encode(), src.ctypes.data if len(src) else None, len(src),
                                 comment.encode() if comment else None))


def select_sources_csr(row_offsets: np.ndarray, seed: int, k: int) -> np.ndarray:
    ro = np.ascontiguousarray(row_offsets, dtype=np.int64)
    out = np.zeros(k, np.int32)
    _check(lib().xb_select_sources_csr(len(ro) - 1, ro.ctypes.data, seed, k, out.ctypes.data))
    return out


def symmetric_weights(row_offsets, col_indices, seed: int, wmin: int = 1, wmax: int = 100) -> np.ndarray:
    """Seeded int32 edge weights in [wmin, wmax], one per column index, equal
    for the two directions of an undirected edge (a hash of the unordered
    pair), so a symmetric CSR stays a symmetric weighted graph."""
    ro = np.ascontiguousarray(row_offsets, dtype=np.int64)
    ci = np.ascontiguousarray(col_indices, dtype=np.int64)
    if wmax < wmin:
        raise ValueError("wmax < wmin")
    u = np.repeat(np.arange(len(ro) - 1, dtype=np.int64), np.diff(ro))
    a, b = np.minimum(u, ci), np.maximum(u, ci)
    h = (a * 1000003 + b * 7919 + int(seed) % (1 << 31)) % (wmax - wmin + 1)
    return (h + wmin).astype(np.int32)


class Graph:
    """Device-resident CSR owned by a Context."""

    def __init__(self, ctx: "Context", handle: int):
        self.ctx = ctx
        self._h = C.c_void_p(handle)
        n, m, md = C.c_int64(), C.c_int64(), C.c_int64()
        _check(lib().xb_graph_info(self._h, C.byref(n), C.byref(m), C.byref(md)))
        self.n, self.m, self.max_degree = n.value, m.value, md.value

    def select_sources(self, seed: int, k: int) -> np.ndarray:
        out = np.zeros(k, np.int32)
        _check(lib().xb_select_sources(self._h, seed, k, out.ctypes.data))
        return out

    def source_order(self, sources) -> np.ndarray:
        """The engine's pass grouping of `sources` (xb_graph_source_order):
        indices into sources by out-degree, highest first, ties in order."""
        src = np.ascontiguousarray(sources, dtype=np.int32)
        out = np.zeros(len(src), np.int32)
        _check(lib().xb_graph_source_order(self._h, src.ctypes.data, len(src), out.ctypes.data))
        return out

    @property
    def offset_bytes(self) -> int:
        """Width of the device row offsets (4, or 8 for huge graphs and under XB_OFFSETS64=1)."""
        b = C.c_int32()
        _check(lib().xb_graph_offset_bytes(self._h, C.byref(b)))
        return b.value

    def set_weights(self, weights) -> None:
        """Attaches int32 edge weights, one per column index (xb_graph_set_weights)."""
        w = np.ascontiguousarray(weights, dtype=np.int32)
        if w.shape != (self.m,):
            raise ValueError(f"weights must have shape ({self.m},)")
        _check(lib().xb_graph_set_weights(self._h, w.ctypes.data if len(w) else None, self.m))

    def close(self) -> None:
        if self._h and self._h.value:
            _check(lib().xb_graph_free(self._h))
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


@dataclass
class TraversalResult:
    level: object  # np.ndarray (host) or torch.Tensor (device), shape (k, n)
    parent: object
    stats: dict = field(default_factory=dict)


class Context:
    """A device context: stream, workspace, tuning (xb_ctx)."""

    def __init__(self, device: int = 0):
        h = C.c_void_p()
        _check(lib().xb_ctx_create(device, C.byref(h)))
        self._h = h
        self.device = device

    # tuning -----------------------------------------------------------------
    def tuning(self) -> dict:
        t = XbTuning()
        _check(lib().xb_ctx_get_tuning(self._h, C.byref(t)))
        return {f: getattr(t, f) for f, _ in XbTuning._fields_}

    def set_tuning(self, **kw) -> None:
        cur = self.tuning()
        cur.update(kw)
        t = XbTuning(**cur)
        _check(lib().xb_ctx_set_tuning(self._h, C.byref(t)))

    def workspace_bytes(self) -> int:
        b = C.c_int64()
        _check(lib().xb_ctx_workspace_bytes(self._h, C.byref(b)))
        return b.value

    def stream_handle(self) -> int:
        """The engine's cudaStream_t as an integer (for torch.cuda.ExternalStream)."""
        p = C.c_void_p()
        _check(lib().xb_ctx_get_stream(self._h, C.byref(p)))
        return p.value or 0

    # graphs -----------------------------------------------------------------
    def upload(self, csr: HostCSR) -> Graph:
        h = C.c_void_p()
        _check(lib().xb_graph_from_host_csr(self._h, csr._h, C.byref(h)))
        return Graph(self, h.value)

    def upload_arrays(self, row_offsets, col_indices) -> Graph:
        ro = np.ascontiguousarray(row_offsets, dtype=np.int64)
        ci = np.ascontiguousarray(col_indices, dtype=np.int32)
        h = C.c_void_p()
        _check(lib().xb_graph_upload(self._h, len(ro) - 1, ro.ctypes.data, 1, int(ro[-1]),
                                     ci.ctypes.data if len(ci) else None, C.byref(h)))
        return Graph(self, h.value)

    def upload_batch(self, graphs) -> list:
        """Uploads several graphs as ONE device CSR with per-instance offsets
        (xb_graph_upload_batch); graphs: list of HostCSR or (row_offsets,
        col_indices) pairs.  Returns one Graph per instance."""
        ros, cis, ns = [], [], []
        for gr in graphs:
            ro, ci = gr.arrays() if isinstance(gr, HostCSR) else gr
            ros.append(np.ascontiguousarray(ro, dtype=np.int64))
            cis.append(np.ascontiguousarray(ci, dtype=np.int32))
            ns.append(len(ros[-1]) - 1)
        ro_all = np.concatenate(ros)
        ci_all = np.concatenate(cis) if sum(len(c) for c in cis) else np.zeros(1, np.int32)
        n_arr = np.array(ns, dtype=np.int64)
        hs = (C.c_void_p * len(ns))()
        _check(lib().xb_graph_upload_batch(self._h, len(ns), n_arr.ctypes.data, ro_all.ctypes.data,
                                           ci_all.ctypes.data, hs))
        return [Graph(self, h) for h in hs]

    def load_text(self, row_path: str, col_path: str) -> Graph:
        h = C.c_void_p()
        _check(lib().xb_graph_load_csr_text(self._h, row_path.encode(), col_path.encode(), C.byref(h)))
        return Graph(self, h.value)

    # traversal --------------------------------------------------------------
    def traverse(self, graph: Graph, sources, out: str = "host", level=None, parent=None,
                 parent_rule: str = "minid") -> TraversalResult:
        """Plain multi-source traversal through xb_traverse.

        out="host": numpy (k, n) int32 tables (host buffers, the drop-in path);
        out="device": torch int32 CUDA tensors (k, n) (allocated here unless
        given).  sources: numpy int32 (host) or a torch int32 CUDA tensor.
        parent_rule: "minid" (smallest-id neighbour one level up) or "fifo"
        (the reference's sequential FIFO search, XB_PARENT_FIFO).
        """
        st = XbStats()
        if parent_rule not in ("minid", "fifo"):
            raise ValueError("parent_rule must be 'minid' or 'fifo'")
        flags = XB_PARENT_FIFO if parent_rule == "fifo" else 0
        src_keep = sources
        if hasattr(sources, "data_ptr"):
            flags |= XB_SOURCES_DEVICE
            k = int(sources.numel())
            sptr = sources.data_ptr()
        else:
            src_keep = np.ascontiguousarray(sources, dtype=np.int32)
            k = len(src_keep)
            sptr = src_keep.ctypes.data
        n = graph.n
        if out == "device":
            import torch

            flags |= XB_OUT_DEVICE
            dev = torch.device("cuda", self.device)
            if level is None:
                level = torch.empty((k, n), dtype=torch.int32, device=dev)
            if parent is None:
                parent = torch.empty((k, n), dtype=torch.int32, device=dev)
            torch.cuda.synchronize(dev)
            lp, pp = level.data_ptr(), parent.data_ptr()
        else:
            if level is None:
                level = np.empty((k, n), np.int32)
            if parent is None:
                parent = np.empty((k, n), np.int32)
            lp, pp = level.ctypes.data, parent.ctypes.data
        _check(lib().xb_traverse(self._h, graph._h, sptr, k, XB_MODE_PLAIN, None, lp, pp, None, flags,
                                 C.byref(st)))
        return TraversalResult(level, parent, st.as_dict())

    def multi_sssp(self, graph: Graph, sources, out: str = "host", dist=None) -> tuple[object, dict]:
        """Multi-source shortest-path distances through xb_multi_sssp on a
        graph with weights (Graph.set_weights): float32 (n,), FLT_MAX / 4 for
        unreached vertices, all -FLT_MAX / 4 after a negative cycle.
        out="host" gives numpy, out="device" a torch CUDA tensor."""
        st = XbStats()
        flags = 0
        src_keep = sources
        if hasattr(sources, "data_ptr"):
            flags |= XB_SOURCES_DEVICE
            k = int(sources.numel())
            sptr = sources.data_ptr()
        else:
            src_keep = np.ascontiguousarray(sources, dtype=np.int32)
            k = len(src_keep)
            sptr = src_keep.ctypes.data
        if out == "device":
            import torch

            flags |= XB_OUT_DEVICE
            if dist is None:
                dist = torch.empty(graph.n, dtype=torch.float32, device=torch.device("cuda", self.device))
            torch.cuda.synchronize(dist.device)
            dp = dist.data_ptr()
        else:
            if dist is None:
                dist = np.empty(graph.n, np.float32)
            dp = dist.ctypes.data
        _check(lib().xb_multi_sssp(self._h, graph._h, sptr, k, dp, flags, C.byref(st)))
        return dist, st.as_dict()

    def alternating_forest(self, graph: Graph, mate) -> tuple[np.ndarray, np.ndarray, np.ndarray, dict]:
        """xb_traverse in XB_MODE_ALTERNATING: the alternating forest of the
        matching `mate` (-1 exposed) from all exposed vertices; numpy (level,
        parent, owner, stats), or torch CUDA tensors when mate is one."""
        st = XbStats()
        if hasattr(mate, "data_ptr"):
            import torch

            lv, pr, ow = (torch.empty_like(mate) for _ in range(3))
            torch.cuda.synchronize(mate.device)
            _check(lib().xb_traverse(self._h, graph._h, None, 0, XB_MODE_ALTERNATING, mate.data_ptr(), lv.data_ptr(),
                                     pr.data_ptr(), ow.data_ptr(), XB_OUT_DEVICE, C.byref(st)))
            return lv, pr, ow, st.as_dict()
        m = np.ascontiguousarray(mate, dtype=np.int32)
        if m.shape != (graph.n,):
            raise ValueError(f"mate must have shape ({graph.n},)")
        lv, pr, ow = (np.empty(graph.n, np.int32) for _ in range(3))
        _check(lib().xb_traverse(self._h, graph._h, None, 0, XB_MODE_ALTERNATING, m.ctypes.data, lv.ctypes.data,
                                 pr.ctypes.data, ow.ctypes.data, 0, C.byref(st)))
        return lv, pr, ow, st.as_dict()

    def max_match(self, graph: Graph, init=None, out: str = "host") -> tuple[object, dict]:
        """Maximum-cardinality matching through xb_max_match: (mate, stats),
        mate[v] = -1 for exposed vertices.  init: starting matching (numpy
        or a torch int32 CUDA tensor, -1 exposed), empty when None.  A torch
        tensor is updated in place; out="device" returns a torch tensor."""
        st = XbStats()
        if hasattr(init, "data_ptr"):
            import torch

            torch.cuda.synchronize(init.device)
            _check(lib().xb_max_match(self._h, graph._h, init.data_ptr(), XB_OUT_DEVICE, C.byref(st)))
            return init, st.as_dict()
        mate = (np.full(graph.n, -1, np.int32) if init is None
                else np.array(init, dtype=np.int32, copy=True))
        if mate.shape != (graph.n,):
            raise ValueError(f"init must have shape ({graph.n},)")
        if out == "device":
            import torch

            t = torch.from_numpy(mate).to(torch.device("cuda", self.device))
            torch.cuda.synchronize(t.device)
            _check(lib().xb_max_match(self._h, graph._h, t.data_ptr(), XB_OUT_DEVICE, C.byref(st)))
            return t, st.as_dict()
        _check(lib().xb_max_match(self._h, graph._h, mate.ctypes.data, 0, C.byref(st)))
        return mate, st.as_dict()

    def traverse_batched(self, queries, out: str = "device", outputs=None) -> tuple[list, dict]:
        """All queries in one launch through xb_traverse_batched.

        queries: list of (graph, sources) pairs (sources as in traverse).
        out="device": torch int32 CUDA tensors (k, n) per query; out="host":
        numpy views of page-locked torch tensors (the launch copies into
        them).  outputs: optional list of (level, parent) to fill instead
        (device tensors, or page-locked host tensors / arrays for "host").
        Returns ([TraversalResult per query], batch stats).
        """
        import torch

        items = (XbBatchItem * max(len(queries), 1))()
        keep, results = [], []
        dev = torch.device("cuda", self.device)
        for i, (graph, sources) in enumerate(queries):
            flags = 0
            if hasattr(sources, "data_ptr"):
                flags |= XB_SOURCES_DEVICE
                k = int(sources.numel())
                sptr = sources.data_ptr()
                keep.append(sources)
            else:
                arr = np.ascontiguousarray(sources, dtype=np.int32)
                keep.append(arr)
                k = len(arr)
                sptr = arr.ctypes.data
            n = graph.n
            if outputs is not None:
                level, parent = outputs[i]
            elif out == "device":
                level = torch.empty((k, n), dtype=torch.int32, device=dev)
                parent = torch.empty((k, n), dtype=torch.int32, device=dev)
            else:
                level = torch.empty((k, n), dtype=torch.int32, pin_memory=True)
                parent = torch.empty((k, n), dtype=torch.int32, pin_memory=True)
            if out == "device":
                flags |= XB_OUT_DEVICE
            keep.extend([level, parent])

            def ptr(t):
                return t.data_ptr() if hasattr(t, "data_ptr") else t.ctypes.data

            items[i] = XbBatchItem(graph._h.value, sptr if k else None, k, flags, ptr(level) if k else None,
                                   ptr(parent) if k else None)
            if out == "host" and hasattr(level, "numpy"):
                level, parent = level.numpy(), parent.numpy()
            results.append([level, parent])
        if out == "device":
            torch.cuda.synchronize(dev)
        st = XbStats()
        _check(lib().xb_traverse_batched(self._h, items, len(queries), C.byref(st)))
        stats = st.as_dict()
        return [TraversalResult(lv, pr, {}) for lv, pr in results], stats

    # serving slots ------------------------------------------------------------
    def slot_launch(self, slot: int, graph: Graph, sources, rows=None) -> None:
        """Queues one pass on a serving slot (xb_slot_launch).  rows: per source
        a (level_row, parent_row) pair of device addresses, or None for a
        digest-only source (default: all digest-only)."""
        src = np.ascontiguousarray(sources, dtype=np.int32)
        kb = len(src)
        lv = (C.c_void_p * max(kb, 1))()
        pr = (C.c_void_p * max(kb, 1))()
        if rows is not None:
            for j, r in enumerate(rows):
                if r is not None:
                    lv[j], pr[j] = r
        _check(lib().xb_slot_launch(self._h, slot, graph._h, src.ctypes.data, kb, lv, pr))
        # only a launch the library accepted replaces the slot's record
        self._slot_keep = getattr(self, "_slot_keep", {})
        self._slot_keep[slot] = (src, lv, pr)

    def slot_poll(self, slot: int, wait: bool = False):
        """(done, stats, digests) of a slot's pass; digests: int64 (kb, 4)
        array of reached, level_sum, row_hash, depth (depth -1 for rows
        written to caller buffers)."""
        keep = getattr(self, "_slot_keep", {}).get(slot)
        kb = len(keep[0]) if keep is not None else 0
        st = XbStats()
        dig = (XbRowDigest * SLOT_MAX_ROWS)()  # the library writes one entry per row of the pass
        if wait:
            _check(lib().xb_slot_wait(self._h, slot, C.byref(st), dig))
            done = 1
        else:
            d = C.c_int32(0)
            _check(lib().xb_slot_poll(self._h, slot, C.byref(d), C.byref(st), dig))
            done = d.value
        if not done:
            return False, None, None
        arr = np.array([(x.reached, x.level_sum, x.row_hash, x.depth) for x in dig[:kb]], dtype=np.int64)
        return True, st.as_dict(), arr.reshape(kb, 4)

    def slots_release(self) -> None:
        _check(lib().xb_slots_release(self._h))

    def slot_set_priority(self, slot: int, priority: int) -> None:
        """Stream priority of an idle slot (xb_slot_set_priority): 0 default,
        1 the device's greatest."""
        _check(lib().xb_slot_set_priority(self._h, slot, priority))

    def close(self) -> None:
        if self._h and self._h.value:
            _check(lib().xb_ctx_destroy(self._h))
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
