"""nwgr_b200 -- B200-native direction-optimizing BFS behind NWGraph's interface.

Python host side of libnwgr_b200.so (C ABI: include/nwg_bfs.h).  The
functions mirror NWGraph's BFS header, include/nwgraph/algorithms/bfs.hpp:

    bfs(out_graph, in_graph, root, num_bins=32, alpha=15, beta=18) -> parents
        nw::graph::bfs, bfs.hpp:160-311 (direction-optimizing)
    bfs_serial(graph, root) -> parents
        nw::graph::bfs(graph, root), bfs.hpp:110-140 (top-down only)
    bfs_verifier(out_graph, in_graph, root, parents) -> bool
        nw::graph::BFSVerifier, bfs.hpp:44-98 (host check)

Graphs are registered once (uploaded to HBM) and reused by every call; the
traversal runs entirely on the GPU.  There is no CPU fallback: importing the
package raises if the CUDA library is missing, and every call raises
NwgError on a non-zero status.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, field

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libnwgr_b200.so")

NULL_VERTEX = 0xFFFFFFFF
TRACE_CAP = 256

NWG_OK, NWG_EINVAL, NWG_ENOMEM, NWG_ECUDA, NWG_ETIMEDOUT, NWG_EOVERFLOW, NWG_ESTATE = 0, -1, -2, -3, -4, -5, -6
REG_DEVICE = 0x1
REG_VALIDATE = 0x2

# Every symbol include/nwg_bfs.h declares (checked by the CPU test suite).
EXPORTED = (
    "nwg_version", "nwg_last_error", "nwg_graph_register", "nwg_graph_register_u32off", "nwg_graph_release",
    "nwg_graph_info", "nwg_bfs", "nwg_bfs_roots", "nwg_ws_create", "nwg_ws_destroy", "nwg_bfs_async", "nwg_ws_stats",
    "nwg_bfs_topdown", "nwg_bfs_stepped", "nwg_component_edges", "nwg_graph_copy_csr", "nwg_gen_rmat", "nwg_gen_uniform",
    "nwg_gen_grid", "nwg_pick_roots", "nwg_bfs_noalloc", "nwg_msbfs_ws_create", "nwg_msbfs_ws_destroy",
    "nwg_msbfs", "nwg_msbfs_ex", "nwg_ragged_register", "nwg_ragged_release", "nwg_ragged_info", "nwg_ragged_bfs",
    "nwg_server_create", "nwg_server_destroy", "nwg_server_submit", "nwg_server_wait", "nwg_server_run_trace",
    "nwg_verify", "nwg_graph_read", "nwg_graph_write_nwbin", "nwg_bc", "nwg_selftest_wait_timeout",
)


class NwgError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"nwg error {code}: {msg}")
        self.code = code


class Stats(C.Structure):
    _fields_ = [
        ("status", C.c_int32), ("steps", C.c_uint32), ("levels", C.c_uint32), ("td_steps", C.c_uint32),
        ("bu_steps", C.c_uint32), ("b2q_steps", C.c_uint32), ("reached", C.c_uint64), ("device_ms", C.c_float),
        ("trace_len", C.c_uint32), ("trace_dir", C.c_uint8 * TRACE_CAP),
        ("trace_frontier", C.c_uint64 * TRACE_CAP), ("trace_found", C.c_uint64 * TRACE_CAP),
        ("trace_end_ns", C.c_uint64 * TRACE_CAP), ("first_decide_ns", C.c_uint64),
        ("kernel_launches", C.c_uint32),
    ]

    def trace(self):
        k = self.trace_len
        return {
            "dir": np.frombuffer(bytes(self.trace_dir), np.uint8)[:k].copy(),
            "frontier": np.ctypeslib.as_array(self.trace_frontier)[:k].copy(),
            "found": np.ctypeslib.as_array(self.trace_found)[:k].copy(),
            "end_ns": np.ctypeslib.as_array(self.trace_end_ns)[:k].copy(),
        }

    def step_ns(self):
        """Device time of each step (launch gaps included), from the trace."""
        end = np.ctypeslib.as_array(self.trace_end_ns)[: self.trace_len].astype(np.int64)
        return np.diff(np.concatenate([[int(self.first_decide_ns)], end]))


MS_TRACE_CAP = 64
# Direction switch of the multi-source BFS: a level pulls when its frontier's
# out-edges exceed the unexplored edges / MS_ALPHA.  Lower than the
# single-source alpha (15): a multi-source pull ORs every in-edge of a vertex
# until all sources have reached it, so it rarely stops early.
MS_ALPHA = 4


class MsStats(C.Structure):
    _fields_ = [("status", C.c_int32), ("passes", C.c_uint32), ("levels", C.c_uint32),
                ("push_levels", C.c_uint32), ("pull_levels", C.c_uint32), ("device_ms", C.c_float),
                ("trace_len", C.c_uint32), ("trace_pull", C.c_uint8 * MS_TRACE_CAP),
                ("trace_ms", C.c_float * MS_TRACE_CAP), ("trace_frontier_edges", C.c_uint64 * MS_TRACE_CAP),
                ("trace_discovered", C.c_uint64 * MS_TRACE_CAP), ("deep_sources", C.c_uint32)]

    def trace(self):
        k = self.trace_len
        return [{"pull": int(self.trace_pull[i]), "ms": float(self.trace_ms[i]),
                 "frontier_edges": int(self.trace_frontier_edges[i]), "discovered": int(self.trace_discovered[i])}
                for i in range(k)]


class RaggedItem(C.Structure):
    _fields_ = [("graph", C.c_uint32), ("root", C.c_uint32), ("alpha", C.c_int32), ("beta", C.c_int32),
                ("warp_min", C.c_uint32)]


class RaggedResult(C.Structure):
    _fields_ = [("status", C.c_int32), ("steps", C.c_uint32), ("levels", C.c_uint32), ("td_steps", C.c_uint32),
                ("bu_steps", C.c_uint32), ("b2q_steps", C.c_uint32), ("reached", C.c_uint64)]


class ServerConfig(C.Structure):
    _fields_ = [("slots", C.c_uint32), ("max_batch", C.c_uint32), ("budget_bytes", C.c_uint64), ("alpha", C.c_int32),
                ("depth_bytes", C.c_uint32)]


class ServerStats(C.Structure):
    _fields_ = [("queries", C.c_uint64), ("batches", C.c_uint64), ("failed", C.c_uint64), ("wall_s", C.c_double),
                ("qps", C.c_double), ("mean_batch", C.c_double), ("mean_ms", C.c_double), ("p50_ms", C.c_double),
                ("p99_ms", C.c_double), ("max_ms", C.c_double), ("peak_state_bytes", C.c_uint64),
                ("budget_bytes", C.c_uint64), ("slot_bytes", C.c_uint64), ("slots", C.c_uint32),
                ("peak_in_flight", C.c_uint32), ("batch_time_s", C.c_double)]

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_}


class VerifyResult(C.Structure):
    _fields_ = [("valid", C.c_int32), ("reason", C.c_uint32), ("first_bad", C.c_uint64), ("reached", C.c_uint64),
                ("levels", C.c_uint32), ("device_ms", C.c_float)]

    REASONS = {0: "ok", 1: "source wrong", 2: "wrong depths", 3: "no edge from the parent",
               4: "reachability mismatch"}


class BcStats(C.Structure):
    _fields_ = [("sources", C.c_uint32), ("lanes", C.c_uint32), ("max_levels", C.c_uint32), ("device_ms", C.c_float)]


_vp = C.c_void_p
_u32, _u64, _int = C.c_uint32, C.c_uint64, C.c_int


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is not built; run `python nwgr_b200/build.py` (nvcc, sm_100a)")
    lib = C.CDLL(LIB_PATH)
    sig = {
        "nwg_version": (C.c_char_p, []),
        "nwg_last_error": (_int, [C.c_char_p, C.c_size_t]),
        "nwg_graph_register": (_int, [_vp, _vp, _u64, _vp, _vp, _u32, C.POINTER(_vp)]),
        "nwg_graph_register_u32off": (_int, [_vp, _vp, _u64, _vp, _vp, _u32, C.POINTER(_vp)]),
        "nwg_graph_release": (_int, [_vp]),
        "nwg_graph_info": (_int, [_vp, C.POINTER(_u64), C.POINTER(_u64), C.POINTER(_u64)]),
        "nwg_bfs": (_int, [_vp, _u32, _int, _int, _vp, _vp, C.POINTER(Stats)]),
        "nwg_bfs_roots": (_int, [_vp, _vp, _u64, _int, _int, _vp, _vp]),
        "nwg_ws_create": (_int, [_vp, C.POINTER(_vp)]),
        "nwg_ws_destroy": (_int, [_vp]),
        "nwg_bfs_async": (_int, [_vp, _u32, _int, _int, _vp, _vp]),
        "nwg_ws_stats": (_int, [_vp, C.POINTER(Stats)]),
        "nwg_bfs_topdown": (_int, [_vp, _u32, _vp, _vp, C.POINTER(Stats)]),
        "nwg_bfs_stepped": (_int, [_vp, _u32, _int, _int, _vp, C.POINTER(Stats)]),
        "nwg_component_edges": (_int, [_vp, _vp, C.POINTER(_u64), C.POINTER(_u64)]),
        "nwg_graph_copy_csr": (_int, [_vp, _vp, _vp, _vp, _vp]),
        "nwg_gen_rmat": (_int, [_u32, _u32, _u64, _u32, _u32, _u32, C.POINTER(_vp)]),
        "nwg_gen_uniform": (_int, [_u64, _u32, _u64, C.POINTER(_vp)]),
        "nwg_gen_grid": (_int, [_u32, _u32, _u32, _u64, C.POINTER(_vp)]),
        "nwg_pick_roots": (_int, [_vp, _u64, _u32, _vp]),
        "nwg_bfs_noalloc": (_int, [_vp, _vp, _vp, _vp, _u64, _u32, _int, _int, _vp, _vp]),
        "nwg_msbfs_ws_create": (_int, [_vp, C.POINTER(_vp)]),
        "nwg_msbfs_ws_destroy": (_int, [_vp]),
        "nwg_msbfs": (_int, [_vp, _vp, _u32, _vp, _int, _vp, C.POINTER(MsStats)]),
        "nwg_msbfs_ex": (_int, [_vp, _vp, _u32, _vp, _u32, _vp, _int, _vp, C.POINTER(MsStats)]),
        "nwg_ragged_register": (_int, [_u32, _vp, _vp, _vp, C.POINTER(_vp)]),
        "nwg_ragged_release": (_int, [_vp]),
        "nwg_ragged_info": (_int, [_vp, C.POINTER(_u32), C.POINTER(_u64), C.POINTER(_u64), C.POINTER(_u64)]),
        "nwg_ragged_bfs": (_int, [_vp, _u32, _vp, _vp, _vp, _vp, _u32, C.POINTER(C.c_float)]),
        "nwg_server_create": (_int, [_vp, _u32, C.POINTER(ServerConfig), C.POINTER(_vp)]),
        "nwg_server_destroy": (_int, [_vp]),
        "nwg_server_submit": (_int, [_vp, _u32, _u32, _vp, C.POINTER(_u64)]),
        "nwg_server_wait": (_int, [_vp, _u64, C.POINTER(C.c_double)]),
        "nwg_server_run_trace": (_int, [_vp, _u32, _vp, _vp, _vp, _vp, _vp, _vp, C.POINTER(ServerStats)]),
        "nwg_verify": (_int, [_vp, _u32, _vp, _vp, C.POINTER(VerifyResult)]),
        "nwg_graph_read": (_int, [C.c_char_p, _u32, C.POINTER(_vp)]),
        "nwg_graph_write_nwbin": (_int, [_vp, C.c_char_p]),
        "nwg_bc": (_int, [_vp, _vp, _u32, _int, _u32, _vp, _vp, C.POINTER(BcStats)]),
        "nwg_selftest_wait_timeout": (_int, [_u32, C.POINTER(C.c_int32), C.POINTER(C.c_float)]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


lib = _load()


def last_error() -> str:
    buf = C.create_string_buffer(1024)
    lib.nwg_last_error(buf, len(buf))
    return buf.value.decode(errors="replace")


def check(rc: int) -> None:
    if rc != NWG_OK:
        raise NwgError(rc, last_error())


def version() -> str:
    return lib.nwg_version().decode()


def _ptr(a) -> int | None:
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        return a.ctypes.data
    if hasattr(a, "data_ptr"):  # torch tensor
        return a.data_ptr()
    return int(a)


def rmat_thresholds(a: float = 0.57, b: float = 0.19, c: float = 0.19):
    return int(a * 4294967296.0), int((a + b) * 4294967296.0), int((a + b + c) * 4294967296.0)


class Graph:
    """A CSR pair registered in HBM (nwg_graph).  `in_off`/`in_cols` None
    means symmetric (the in-graph is the out-graph)."""

    def __init__(self, handle: int, keep=None):
        self.h = handle
        self._keep = keep
        n, m, im = _u64(), _u64(), _u64()
        check(lib.nwg_graph_info(handle, C.byref(n), C.byref(m), C.byref(im)))
        self.n, self.m, self.in_m = n.value, m.value, im.value

    @classmethod
    def from_csr(cls, off, cols, in_off=None, in_cols=None, validate=False, device=False):
        """Registers host numpy CSR arrays (uploaded once) or, with
        device=True, device arrays given as torch tensors / integer pointers
        (borrowed).  uint32 offsets select the adjacency<0> layout."""
        h = _vp()
        flags = (REG_VALIDATE if validate else 0) | (REG_DEVICE if device else 0)
        if device:
            n = int(off.numel() - 1) if hasattr(off, "numel") else None
            if n is None:
                raise ValueError("device registration needs tensors")
            fn = lib.nwg_graph_register if off.element_size() == 8 else lib.nwg_graph_register_u32off
            check(fn(_ptr(off), _ptr(cols), n, _ptr(in_off), _ptr(in_cols), flags, C.byref(h)))
            return cls(h.value, keep=(off, cols, in_off, in_cols))
        off = np.ascontiguousarray(off)
        cols = np.ascontiguousarray(cols, dtype=np.uint32)
        if off.dtype == np.uint32:
            fn = lib.nwg_graph_register_u32off
            if in_off is not None:
                in_off = np.ascontiguousarray(in_off, dtype=np.uint32)
        else:
            off = off.astype(np.uint64, copy=False)
            fn = lib.nwg_graph_register
            if in_off is not None:
                in_off = np.ascontiguousarray(in_off, dtype=np.uint64)
        if in_cols is not None:
            in_cols = np.ascontiguousarray(in_cols, dtype=np.uint32)
        check(fn(_ptr(off), _ptr(cols), off.size - 1, _ptr(in_off), _ptr(in_cols), flags, C.byref(h)))
        return cls(h.value)

    @classmethod
    def read(cls, path: str, symmetric: bool = False) -> "Graph":
        """MatrixMarket or NWGraph binary adjacency file (nwg_graph_read)."""
        h = _vp()
        check(lib.nwg_graph_read(os.fsencode(path), 1 if symmetric else 0, C.byref(h)))
        return cls(h.value)

    def write_nwbin(self, path: str) -> None:
        """The out-CSR in NWGraph's binary adjacency format."""
        check(lib.nwg_graph_write_nwbin(self.h, os.fsencode(path)))

    @classmethod
    def rmat(cls, scale: int, edge_factor: int = 16, seed: int = 1, a=0.57, b=0.19, c=0.19):
        h = _vp()
        ta, tab, tabc = rmat_thresholds(a, b, c)
        check(lib.nwg_gen_rmat(scale, edge_factor, seed, ta, tab, tabc, C.byref(h)))
        return cls(h.value)

    @classmethod
    def uniform(cls, n: int, avg_degree: int = 32, seed: int = 1):
        h = _vp()
        check(lib.nwg_gen_uniform(n, avg_degree, seed, C.byref(h)))
        return cls(h.value)

    @classmethod
    def grid(cls, width: int, height: int, shortcut_pct: int = 1, seed: int = 1):
        h = _vp()
        check(lib.nwg_gen_grid(width, height, shortcut_pct, seed, C.byref(h)))
        return cls(h.value)

    def csr(self):
        """Host copy of the out-CSR (offsets uint64, columns uint32)."""
        off = np.empty(self.n + 1, np.uint64)
        cols = np.empty(self.m, np.uint32)
        check(lib.nwg_graph_copy_csr(self.h, _ptr(off), _ptr(cols), None, None))
        return off, cols

    def roots(self, count: int = 64, seed: int = 27491095):
        out = np.empty(count, np.uint32)
        check(lib.nwg_pick_roots(self.h, seed, count, _ptr(out)))
        return out

    def component_edges(self, parents_dev):
        e, v = _u64(), _u64()
        check(lib.nwg_component_edges(self.h, _ptr(parents_dev), C.byref(e), C.byref(v)))
        return e.value, v.value

    def workspace(self):
        return Workspace(self)

    def release(self):
        if self.h:
            check(lib.nwg_graph_release(self.h))
            self.h = None

    def __del__(self):
        try:
            if self.h:
                lib.nwg_graph_release(self.h)
                self.h = None
        except Exception:
            pass


class MsWorkspace:
    """State of the batched multi-source BFS (nwg_msbfs_ws)."""

    def __init__(self, g: Graph):
        self.g = g
        h = _vp()
        check(lib.nwg_msbfs_ws_create(g.h, C.byref(h)))
        self.h = h.value

    def run(self, roots, depths_dev, alpha: int = MS_ALPHA, stream=None) -> MsStats:
        """Depths of every vertex from every root into depths_dev (device
        uint8 [k][n]; 255 = unreached).  Returns the MsStats."""
        roots = np.ascontiguousarray(roots, dtype=np.uint32)
        st = MsStats()
        check(lib.nwg_msbfs(self.h, roots.ctypes.data, roots.size, _ptr(depths_dev), alpha, _ptr(stream), C.byref(st)))
        return st

    def run_ex(self, roots, depths_dev, deep_flags=None, alpha: int = MS_ALPHA, stream=None) -> MsStats:
        """nwg_msbfs_ex: depths_dev is a device [k][n] array of uint8 (255 =
        unreached) or of 16-bit integers (read as uint16, 0xFFFF = unreached).
        uint8 rows of sources whose depths reach 255 stop at 254 and are
        flagged in deep_flags (host uint8 array of k, optional); uint16 rows
        are exact for every source."""
        roots = np.ascontiguousarray(roots, dtype=np.uint32)
        width = depths_dev.element_size() if hasattr(depths_dev, "element_size") else depths_dev.dtype.itemsize
        if deep_flags is not None:
            assert deep_flags.dtype == np.uint8 and deep_flags.size >= roots.size and deep_flags.flags.c_contiguous
        st = MsStats()
        check(lib.nwg_msbfs_ex(self.h, roots.ctypes.data, roots.size, _ptr(depths_dev), int(width),
                               None if deep_flags is None else deep_flags.ctypes.data, alpha, _ptr(stream),
                               C.byref(st)))
        return st

    def close(self):
        if self.h and self.g.h:
            check(lib.nwg_msbfs_ws_destroy(self.h))
        self.h = None


def msbfs(g: Graph, roots, alpha: int = MS_ALPHA, depth_bytes: int = 1):
    """Batched multi-source BFS; returns host depths [k][n] and the MsStats.
    depth_bytes 1: uint8 (255 = unreached; raises NwgError NWG_EOVERFLOW if a
    depth reaches 255); 2: uint16 (0xFFFF = unreached), exact for any
    depth below 65535.  Uses torch for the device output buffer."""
    import torch

    roots = np.ascontiguousarray(roots, dtype=np.uint32)
    ws = MsWorkspace(g)
    try:
        if depth_bytes == 2:
            out = torch.empty((roots.size, g.n), dtype=torch.int16, device="cuda")
            st = ws.run_ex(roots, out, None, alpha)
            return out.cpu().numpy().view(np.uint16), st
        out = torch.empty((roots.size, g.n), dtype=torch.uint8, device="cuda")
        st = ws.run(roots, out, alpha)
    finally:
        ws.close()
    return out.cpu().numpy(), st


class RaggedBatch:
    """Many small CSR graphs packed in HBM (nwg_ragged) and traversed as a
    table of (graph, root) items in one persistent launch."""

    def __init__(self, graphs):
        """graphs: sequence of (offsets uint64[n+1], columns uint32[m])."""
        ns = np.asarray([g[0].size - 1 for g in graphs], np.uint64)
        off = np.ascontiguousarray(np.concatenate([np.asarray(g[0], np.uint64) for g in graphs]))
        cols = np.ascontiguousarray(np.concatenate([np.asarray(g[1], np.uint32) for g in graphs]))
        h = _vp()
        check(lib.nwg_ragged_register(ns.size, ns.ctypes.data, off.ctypes.data, cols.ctypes.data, C.byref(h)))
        self.h = h.value
        self.n = ns
        self.num_graphs = ns.size

    def run(self, items, parents_dev=None, blocks_per_sm: int = 2):
        """items: list of (graph, root, alpha, beta, warp_min).  Returns
        (parents packed as a device tensor, item offsets, results, device ms)."""
        import torch

        k = len(items)
        arr = (RaggedItem * k)(*[RaggedItem(int(g), int(r), int(a), int(b), int(w)) for g, r, a, b, w in items])
        # sizes of valid items only: the C layer rejects bad ones with a message
        total = int(sum(int(self.n[g]) for g, *_ in items if 0 <= int(g) < self.num_graphs))
        if parents_dev is None:
            parents_dev = torch.empty(max(total, 1), dtype=torch.int32, device="cuda")
        offs = np.zeros(k, np.uint64)
        res = (RaggedResult * k)()
        ms = C.c_float(0.0)
        check(lib.nwg_ragged_bfs(self.h, k, arr, _ptr(parents_dev), offs.ctypes.data, res, int(blocks_per_sm),
                                 C.byref(ms)))
        return parents_dev, offs, res, ms.value

    def release(self):
        if self.h:
            check(lib.nwg_ragged_release(self.h))
            self.h = None

    def __del__(self):
        try:
            if self.h:
                lib.nwg_ragged_release(self.h)
                self.h = None
        except Exception:
            pass


class Server:
    """Query server over resident graphs (nwg_server): (graph index, root)
    queries answered as depth rows -- uint8 (255 = unreached) or, with
    depth_bytes=2, uint16 (0xFFFF = unreached) -- same-graph queries
    coalesced into multi-source passes, `slots` batches in flight at once,
    admission against `budget_bytes`."""

    def __init__(self, graphs, slots: int = 16, max_batch: int = 256, budget_bytes: int = 16 << 30, alpha: int = 0,
                 depth_bytes: int = 1):
        self.graphs = list(graphs)  # kept alive: the server borrows them
        self.depth_bytes = int(depth_bytes)
        self.dtype = np.uint16 if self.depth_bytes == 2 else np.uint8
        hs = (_vp * len(self.graphs))(*[g.h for g in self.graphs])
        cfg = ServerConfig(int(slots), int(max_batch), int(budget_bytes), int(alpha), self.depth_bytes)
        h = _vp()
        check(lib.nwg_server_create(hs, len(self.graphs), C.byref(cfg), C.byref(h)))
        self.h = h.value

    def submit(self, graph: int, root: int, out: np.ndarray | None = None) -> int:
        """Queues one query; `out` (uint8, or uint16 with depth_bytes=2; n of
        the graph) receives the answer."""
        if out is not None:
            assert out.dtype == self.dtype and out.flags.c_contiguous and out.size >= self.graphs[graph].n
        t = _u64()
        check(lib.nwg_server_submit(self.h, int(graph), int(root), None if out is None else out.ctypes.data,
                                    C.byref(t)))
        return t.value

    def wait(self, ticket: int) -> float:
        """Blocks until the query is answered; returns its latency in ms."""
        lat = C.c_double()
        check(lib.nwg_server_wait(self.h, int(ticket), C.byref(lat)))
        return lat.value / 1e3

    def run_trace(self, graph_ids, roots, arrival_us, outputs=None):
        """Open-loop replay: query i released at arrival_us[i].  outputs: None
        or a list of arrays of the server's row type (None entries allowed).
        Returns (latency ms per query, batch size per query, ServerStats)."""
        g = np.ascontiguousarray(graph_ids, np.uint32)
        r = np.ascontiguousarray(roots, np.uint32)
        a = np.ascontiguousarray(arrival_us, np.float64)
        k = g.size
        assert r.size == k and a.size == k
        outp = None
        if outputs is not None:
            assert all(o is None or (o.dtype == self.dtype and o.size >= self.graphs[gi].n)
                       for o, gi in zip(outputs, g.tolist()))
            outp = (C.c_void_p * k)(*[None if o is None else o.ctypes.data for o in outputs])
        lat = np.zeros(k, np.float64)
        bs = np.zeros(k, np.uint32)
        st = ServerStats()
        check(lib.nwg_server_run_trace(self.h, k, g.ctypes.data, r.ctypes.data, a.ctypes.data, outp,
                                       lat.ctypes.data, bs.ctypes.data, C.byref(st)))
        return lat / 1e3, bs, st

    def close(self):
        if self.h:
            check(lib.nwg_server_destroy(self.h))
            self.h = None

    def __del__(self):
        try:
            if self.h:
                lib.nwg_server_destroy(self.h)
                self.h = None
        except Exception:
            pass


class Workspace:
    """Per-traversal device state for stream-ordered traversals (nwg_bfs_ws)."""

    def __init__(self, g: Graph):
        self.g = g
        h = _vp()
        check(lib.nwg_ws_create(g.h, C.byref(h)))
        self.h = h.value

    def bfs_async(self, root: int, parents_dev, stream=None, alpha=15, beta=18):
        check(lib.nwg_bfs_async(self.h, int(root), alpha, beta, _ptr(parents_dev), _ptr(stream)))

    def stats(self) -> Stats:
        s = Stats()
        check(lib.nwg_ws_stats(self.h, C.byref(s)))
        return s

    def close(self):
        if self.h and self.g.h:
            check(lib.nwg_ws_destroy(self.h))
        self.h = None


def bfs(out_graph: Graph, in_graph: Graph | None = None, root: int = 0, num_bins: int = 32, alpha: int = 15,
        beta: int = 18, parents_out=None, stats: bool = False):
    """nw::graph::bfs(out_graph, in_graph, root, num_bins, alpha, beta).

    `in_graph` must be the registration that holds the transpose; the C ABI
    registers out/in as one pair, so pass the same Graph (or None).
    `num_bins` is accepted for signature compatibility; the device bins by
    degree.  Returns the parents as a numpy uint32 array (and the Stats).
    """
    if in_graph is not None and in_graph is not out_graph:
        raise ValueError("register the out/in pair as one Graph (Graph.from_csr(off, cols, in_off, in_cols))")
    if num_bins <= 0:
        raise ValueError("num_bins must be positive")
    parents = parents_out if parents_out is not None else np.empty(out_graph.n, np.uint32)
    s = Stats()
    check(lib.nwg_bfs(out_graph.h, int(root), alpha, beta, _ptr(parents), None, C.byref(s) if stats else None))
    return (parents, s) if stats else parents


def bfs_roots(g: Graph, roots, parents_out=None, alpha: int = 15, beta: int = 18, status=None):
    """nw::graph::bfs over many roots (the per-source loop of NWGraph's BFS
    benchmark, bench/bfs.cpp:106-141): row i of the returned (k, n) uint32
    array holds the parents of roots[i].  Two traversals are in flight, so
    root i + 1 traverses while root i's parents are copied; pass a pinned
    `parents_out` (e.g. a pinned torch tensor's numpy view) for overlapped
    copies.  `status`: optional int32 array of k entries, each root's status."""
    r = np.ascontiguousarray(roots, dtype=np.uint32)
    k = int(r.size)
    parents = parents_out if parents_out is not None else np.empty((k, g.n), np.uint32)
    if parents.size < k * g.n or not parents.flags.c_contiguous or parents.dtype.itemsize != 4:
        raise ValueError("parents_out must be a contiguous 4-byte array of at least len(roots) * n entries")
    if status is not None and (status.size < k or status.dtype != np.int32 or not status.flags.c_contiguous):
        raise ValueError("status must be a contiguous int32 array of at least len(roots) entries")
    check(lib.nwg_bfs_roots(g.h, _ptr(r), k, alpha, beta, _ptr(parents), _ptr(status) if status is not None else None))
    return parents


def bfs_device(g: Graph, root: int, parents_dev, alpha: int = 15, beta: int = 18, stats: bool = False):
    """Synchronous traversal writing parents to a device array (torch tensor
    or pointer) without a host copy."""
    s = Stats()
    check(lib.nwg_bfs(g.h, int(root), alpha, beta, None, _ptr(parents_dev), C.byref(s) if stats else None))
    return s if stats else None


def bfs_stepped(g: Graph, root: int, parents_dev=None, alpha: int = 15, beta: int = 18):
    """The same traversal with the level loop driven from the host, one
    kernel launch at a time (for profilers).  Returns the Stats."""
    s = Stats()
    check(lib.nwg_bfs_stepped(g.h, int(root), alpha, beta, _ptr(parents_dev), C.byref(s)))
    return s


def bfs_noalloc(out_off_dev, out_col_dev, n: int, root: int, parents_dev, in_off_dev=None, in_col_dev=None,
                alpha: int = 15, beta: int = 18, stream=None) -> None:
    """nwg_bfs_noalloc: the traversal without any device allocation, for
    callers that may not call cudaMalloc.  All arrays are the caller's device
    memory (torch tensors or integer pointers); limits n <= 2^20, m <= 2^24.
    Calls share one static scratch array: do not overlap them on the GPU."""
    check(lib.nwg_bfs_noalloc(_ptr(out_off_dev), _ptr(out_col_dev), _ptr(in_off_dev), _ptr(in_col_dev), int(n),
                              int(root), alpha, beta, _ptr(parents_dev), _ptr(stream)))


def bfs_serial(graph: Graph, root: int, stats: bool = False):
    """nw::graph::bfs(graph, root): top-down only, out-edges only."""
    parents = np.empty(graph.n, np.uint32)
    s = Stats()
    check(lib.nwg_bfs_topdown(graph.h, int(root), _ptr(parents), None, C.byref(s) if stats else None))
    return (parents, s) if stats else parents


def depths_from_parents(parents: np.ndarray, root: int) -> np.ndarray:
    """Depth of every vertex in the parent tree (NULL_VERTEX where unreached),
    computed level by level with numpy.  Raises ValueError if the parents do
    not form a tree rooted at `root`."""
    parents = np.asarray(parents, dtype=np.uint32)
    n = parents.size
    depth = np.full(n, NULL_VERTEX, np.uint32)
    if parents[root] != root:
        raise ValueError("root is not its own parent")
    depth[root] = 0
    reached = parents != NULL_VERTEX
    if np.any(parents[reached] >= n):
        raise ValueError("parent id out of range")
    pending = np.flatnonzero(reached)
    pending = pending[pending != root]
    d = 0
    while pending.size:
        par = parents[pending]
        ready = depth[par] == d
        if not np.any(ready):
            raise ValueError("parents contain a cycle or a dangling chain")
        depth[pending[ready]] = d + 1
        pending = pending[~ready]
        d += 1
    return depth


def betweenness(g: Graph, sources, normalize: bool = True, lanes: int = 0):
    """brandes_bc<float, double>(graph, sources, ...) on the GPU: (scores as
    a host float32 array, BcStats)."""
    src = np.ascontiguousarray(sources, dtype=np.uint32)
    out = np.zeros(g.n, np.float32)
    st = BcStats()
    check(lib.nwg_bc(g.h, src.ctypes.data, src.size, 1 if normalize else 0, int(lanes), out.ctypes.data, None,
                     C.byref(st)))
    return out, st


def verify(g: Graph, root: int, parents) -> VerifyResult:
    """nw::graph::BFSVerifier on the GPU (bfs.hpp:44-98): parents is a host
    uint32 array or a device tensor.  Returns the VerifyResult (valid, and
    for an invalid array the lowest failing vertex and the reason)."""
    r = VerifyResult()
    if isinstance(parents, np.ndarray):
        p = np.ascontiguousarray(parents, dtype=np.uint32)
        assert p.size >= g.n
        check(lib.nwg_verify(g.h, int(root), p.ctypes.data, None, C.byref(r)))
    else:
        check(lib.nwg_verify(g.h, int(root), None, _ptr(parents), C.byref(r)))
    return r


def bfs_verifier(off, cols, root, parents, in_off=None, in_cols=None) -> bool:
    """nw::graph::BFSVerifier's checks (bfs.hpp:44-98) on host CSR arrays:
    BFS depths from the out-graph; root self-parent at depth 0; every reached
    u has parents[u] among in[u] one level closer; reachability agrees."""
    off = np.asarray(off, np.uint64)
    cols = np.asarray(cols, np.uint32)
    if in_off is None:
        in_off, in_cols = off, cols
    n = off.size - 1
    depth = np.full(n, NULL_VERTEX, np.int64)
    depth[root] = 0
    frontier = np.asarray([root], np.int64)
    d = 0
    deg = (off[1:] - off[:-1]).astype(np.int64)
    while frontier.size:
        starts = off[frontier].astype(np.int64)
        lens = deg[frontier]
        idx = np.repeat(starts - np.cumsum(lens) + lens, lens) + np.arange(lens.sum())
        nbr = np.unique(cols[idx].astype(np.int64))
        nbr = nbr[depth[nbr] == NULL_VERTEX]
        d += 1
        depth[nbr] = d
        frontier = nbr
    parents = np.asarray(parents, np.uint32)
    reached_d = depth != NULL_VERTEX
    reached_p = parents != NULL_VERTEX
    if np.any(reached_d != reached_p):
        return False
    if parents[root] != root:
        return False
    us = np.flatnonzero(reached_p)
    us = us[us != root]
    if us.size == 0:
        return True
    pu = parents[us].astype(np.int64)
    if np.any(depth[pu] != depth[us] - 1):
        return False
    # parents[u] must be an in-neighbour of u
    in_off = np.asarray(in_off, np.uint64)
    in_cols = np.asarray(in_cols, np.uint32)
    ideg = (in_off[1:] - in_off[:-1]).astype(np.int64)
    lens = ideg[us]
    starts = in_off[us].astype(np.int64)
    idx = np.repeat(starts - np.cumsum(lens) + lens, lens) + np.arange(lens.sum())
    owner = np.repeat(np.arange(us.size), lens)
    hit = np.zeros(us.size, bool)
    match = in_cols[idx].astype(np.int64) == pu[owner]
    hit[owner[match]] = True
    return bool(hit.all())
