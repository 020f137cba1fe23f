"""TEST INFRASTRUCTURE ONLY: builds and loads the two CPU oracles.

* ``oracle/_build/libnwgport.so`` -- the plain-C restatement in
  ``oracle/dobfs_port.c`` (always buildable: gcc only).
* ``oracle/_ref/libnwgref.so`` -- the reference's own, unmodified
  include/nwgraph/algorithms/bfs.hpp compiled by ``oracle/ref_dobfs.cpp``
  against the project's TBB compatibility shim.  It can only be (re)built
  where the reference sources exist; elsewhere a previously built copy is
  used if present.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg use
this module, as the checker.  The product never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PORT_SO = os.path.join(HERE, "_build", "libnwgport.so")
REF_SO = os.path.join(HERE, "_ref", "libnwgref.so")
# NWGraph's source tree: $NWG_REFERENCE_ROOT, else a checkout named
# "reference" beside this repository (its include/ holds nwgraph/).
REFERENCE_ROOT = os.environ.get("NWG_REFERENCE_ROOT",
                                os.path.join(os.path.dirname(os.path.dirname(HERE)), "reference"))
REFERENCE_INCLUDE = os.environ.get("NWG_REFERENCE_INCLUDE", os.path.join(REFERENCE_ROOT, "include"))
NULLV = 0xFFFFFFFF

_u64p = np.ctypeslib.ndpointer(dtype=np.uint64, flags="C_CONTIGUOUS")
_u32p = np.ctypeslib.ndpointer(dtype=np.uint32, flags="C_CONTIGUOUS")
_u8p = np.ctypeslib.ndpointer(dtype=np.uint8, flags="C_CONTIGUOUS")
_f32p = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")


GEN_SO = os.path.join(HERE, "_build", "libnwggen.so")
KIND_RMAT, KIND_UNIFORM, KIND_GRID = 0, 1, 2


def build_gen(force: bool = False) -> str:
    src = os.path.join(HERE, "graphgen_host.c")
    if force or not os.path.exists(GEN_SO) or os.path.getmtime(GEN_SO) < os.path.getmtime(src):
        os.makedirs(os.path.dirname(GEN_SO), exist_ok=True)
        subprocess.check_call(["gcc", "-O3", "-std=c11", "-fPIC", "-shared", "-fopenmp", src, "-o", GEN_SO + ".tmp"])
        os.replace(GEN_SO + ".tmp", GEN_SO)
    return GEN_SO


class HostGen:
    """ctypes view of oracle/graphgen_host.c: the seeded generators of
    oracle/graphgen.py built on the host cores (OpenMP).  Same graphs, bit
    for bit, in seconds at scale 24."""

    def __init__(self, threads: int = 0):
        lib = C.CDLL(build_gen())
        lib.nwggen_capacity.restype = C.c_uint64
        lib.nwggen_capacity.argtypes = [C.c_int, C.c_uint64, C.c_uint64, C.c_uint64]
        lib.nwggen_vertices.restype = C.c_uint64
        lib.nwggen_vertices.argtypes = [C.c_int, C.c_uint64, C.c_uint64, C.c_uint64]
        lib.nwggen_csr.restype = C.c_int64
        lib.nwggen_csr.argtypes = [C.c_int, C.c_uint64, C.c_uint64, C.c_uint64, C.c_uint64, C.c_uint32, C.c_uint32,
                                   C.c_uint32, C.c_int, _u64p, _u32p, _u32p, C.c_uint64]
        self.lib = lib
        self.threads = int(threads)

    def _csr(self, kind, a0, a1, a2, seed, thr=(0, 0, 0)):
        cap = int(self.lib.nwggen_capacity(kind, a0, a1, a2))
        n = int(self.lib.nwggen_vertices(kind, a0, a1, a2))
        if cap == 0 and n == 0:
            raise ValueError("bad generator arguments")
        off = np.empty(n + 1, np.uint64)
        tmp = np.empty(max(cap, 1), np.uint32)
        cols = np.empty(max(cap, 1), np.uint32)
        m = self.lib.nwggen_csr(kind, a0, a1, a2, seed & 0xFFFFFFFFFFFFFFFF, *thr, self.threads, off, tmp, cols, cap)
        if m < 0:
            raise ValueError(f"nwggen_csr failed: {m}")
        del tmp
        return off, (cols[:m].copy() if m < cap // 2 else cols[:m])

    def rmat(self, scale: int, edge_factor: int = 16, seed: int = 1, a=0.57, b=0.19, c=0.19):
        from oracle.graphgen import rmat_thresholds

        return self._csr(KIND_RMAT, scale, edge_factor, 0, seed, rmat_thresholds(a, b, c))

    def uniform(self, n: int, avg_degree: int = 32, seed: int = 1):
        return self._csr(KIND_UNIFORM, n, avg_degree, 0, seed)

    def grid(self, width: int, height: int, shortcut_pct: int = 1, seed: int = 1):
        return self._csr(KIND_GRID, width, height, shortcut_pct, seed)


def build_port(force: bool = False) -> str:
    src = os.path.join(HERE, "dobfs_port.c")
    if force or not os.path.exists(PORT_SO) or os.path.getmtime(PORT_SO) < os.path.getmtime(src):
        os.makedirs(os.path.dirname(PORT_SO), exist_ok=True)
        subprocess.check_call(["gcc", "-O2", "-std=c11", "-fPIC", "-shared", src, "-o", PORT_SO])
    return PORT_SO


def reference_available() -> bool:
    return os.path.exists(os.path.join(REFERENCE_INCLUDE, "nwgraph", "algorithms", "bfs.hpp"))


def build_ref(force: bool = False) -> str | None:
    """Compile the reference bfs.hpp (unmodified) into oracle/_ref.  Returns
    the library path, or None when neither the sources nor a built copy exist."""
    src = os.path.join(HERE, "ref_dobfs.cpp")
    if not reference_available():
        return REF_SO if os.path.exists(REF_SO) else None
    shim = os.path.join(HERE, "tbb_compat")
    newest = max(os.path.getmtime(os.path.join(r, f)) for r, _, fs in os.walk(shim) for f in fs)
    newest = max(newest, os.path.getmtime(src))
    if force or not os.path.exists(REF_SO) or os.path.getmtime(REF_SO) < newest:
        os.makedirs(os.path.dirname(REF_SO), exist_ok=True)
        subprocess.check_call(
            ["g++", "-std=c++20", "-O3", "-fPIC", "-shared", "-fvisibility=hidden", "-pthread",
             "-I", shim, "-I", REFERENCE_INCLUDE, src, "-o", REF_SO])
    return REF_SO


DROPIN_BIN = os.path.join(os.path.dirname(HERE), "tests", "cpp", "_build", "dropin_test")


def build_dropin_test(force: bool = False) -> str | None:
    """Compile tests/cpp/dropin_test.cpp: this repository's include/ first (the
    drop-in nwgraph/algorithms/bfs.hpp and nwg_bfs.h), NWGraph's headers
    second, the TBB-compatible shim for NWGraph's other headers, linked to
    libnwgr_b200.so.  Needs the NWGraph sources; returns None without them."""
    root = os.path.dirname(HERE)
    src = os.path.join(root, "tests", "cpp", "dropin_test.cpp")
    lib_dir = os.path.join(root, "nwgr_b200")
    if not reference_available():
        return DROPIN_BIN if os.path.exists(DROPIN_BIN) else None
    deps = [src, os.path.join(root, "include", "nwgraph", "algorithms", "bfs.hpp"),
            os.path.join(root, "include", "nwg_bfs.h")]
    if force or not os.path.exists(DROPIN_BIN) or any(os.path.getmtime(d) > os.path.getmtime(DROPIN_BIN) for d in deps):
        os.makedirs(os.path.dirname(DROPIN_BIN), exist_ok=True)
        subprocess.check_call(
            ["g++", "-std=c++20", "-O2", "-pthread", "-Wno-deprecated-declarations", "-I", os.path.join(root, "include"),
             "-I", os.path.join(HERE, "tbb_compat"), "-I", REFERENCE_INCLUDE, src, "-o", DROPIN_BIN,
             "-L", lib_dir, "-lnwgr_b200", "-Wl,-rpath,$ORIGIN/../../../nwgr_b200"])
    return DROPIN_BIN


class _Trace(C.Structure):
    _fields_ = [("cap", C.c_uint32), ("steps", C.c_uint32), ("dir", C.POINTER(C.c_uint8)),
                ("frontier", C.POINTER(C.c_uint64)), ("found", C.POINTER(C.c_uint64)),
                ("scout", C.POINTER(C.c_uint64))]


class Port:
    """ctypes view of oracle/dobfs_port.c."""

    def __init__(self):
        lib = C.CDLL(build_port())
        lib.nwgport_dobfs.restype = C.c_int64
        lib.nwgport_dobfs.argtypes = [_u64p, _u32p, C.c_void_p, C.c_void_p, C.c_uint64, C.c_uint32, C.c_int,
                                      C.c_int, C.c_int, _u32p, C.POINTER(_Trace)]
        lib.nwgport_bfs_depths.restype = C.c_int64
        lib.nwgport_bfs_depths.argtypes = [_u64p, _u32p, C.c_uint64, C.c_uint32, _u32p]
        lib.nwgport_depths_from_parents.restype = C.c_int64
        lib.nwgport_depths_from_parents.argtypes = [_u32p, C.c_uint64, C.c_uint32, _u32p]
        lib.nwgport_verify.restype = C.c_int
        lib.nwgport_verify.argtypes = [_u64p, _u32p, C.c_void_p, C.c_void_p, C.c_uint64, C.c_uint32, _u32p]
        lib.nwgport_bc.restype = C.c_int64
        lib.nwgport_bc.argtypes = [_u64p, _u32p, C.c_uint64, _u32p, C.c_uint32, C.c_int, _f32p]
        lib.nwgport_msbfs_depths.restype = C.c_int64
        lib.nwgport_msbfs_depths.argtypes = [_u64p, _u32p, C.c_uint64, _u32p, C.c_uint32, _u8p]
        self.lib = lib

    def dobfs(self, off, cols, root, in_off=None, in_cols=None, num_bins=32, alpha=15, beta=18, trace_cap=4096):
        n = off.size - 1
        parents = np.empty(n, np.uint32)
        tr = _Trace()
        buf_dir = np.zeros(trace_cap, np.uint8)
        buf_f = np.zeros(trace_cap, np.uint64)
        buf_d = np.zeros(trace_cap, np.uint64)
        buf_s = np.zeros(trace_cap, np.uint64)
        tr.cap = trace_cap
        tr.steps = 0
        tr.dir = buf_dir.ctypes.data_as(C.POINTER(C.c_uint8))
        tr.frontier = buf_f.ctypes.data_as(C.POINTER(C.c_uint64))
        tr.found = buf_d.ctypes.data_as(C.POINTER(C.c_uint64))
        tr.scout = buf_s.ctypes.data_as(C.POINTER(C.c_uint64))
        io = in_off.ctypes.data if in_off is not None else None
        ic = in_cols.ctypes.data if in_cols is not None else None
        rc = self.lib.nwgport_dobfs(off, cols, io, ic, n, int(root), num_bins, alpha, beta, parents, C.byref(tr))
        if rc < 0:
            raise ValueError(f"nwgport_dobfs failed: {rc}")
        k = min(tr.steps, trace_cap)
        trace = {"dir": buf_dir[:k].copy(), "frontier": buf_f[:k].copy(), "found": buf_d[:k].copy(),
                 "scout": buf_s[:k].copy()}
        return parents, trace

    def depths(self, off, cols, root):
        d = np.empty(off.size - 1, np.uint32)
        if self.lib.nwgport_bfs_depths(off, cols, off.size - 1, int(root), d) < 0:
            raise ValueError("bad root")
        return d

    def depths_from_parents(self, parents, root):
        d = np.empty(parents.size, np.uint32)
        if self.lib.nwgport_depths_from_parents(np.ascontiguousarray(parents, np.uint32), parents.size,
                                                int(root), d) != 0:
            return None
        return d

    def verify(self, off, cols, root, parents, in_off=None, in_cols=None):
        io = in_off.ctypes.data if in_off is not None else None
        ic = in_cols.ctypes.data if in_cols is not None else None
        return self.lib.nwgport_verify(off, cols, io, ic, off.size - 1, int(root),
                                       np.ascontiguousarray(parents, np.uint32)) == 1

    def bc(self, off, cols, sources, normalize=True):
        """BCVerifier's approximate betweenness centrality (float scores)."""
        src = np.ascontiguousarray(sources, np.uint32)
        out = np.zeros(off.size - 1, np.float32)
        if self.lib.nwgport_bc(off, cols, off.size - 1, src, src.size, 1 if normalize else 0, out) < 0:
            raise MemoryError("nwgport_bc")
        return out

    def msbfs_depths(self, off, cols, roots):
        roots = np.ascontiguousarray(roots, np.uint32)
        out = np.empty((roots.size, off.size - 1), np.uint8)
        rc = self.lib.nwgport_msbfs_depths(off, cols, off.size - 1, roots, roots.size, out)
        if rc == -3:
            raise OverflowError("a depth does not fit uint8")
        if rc < 0:
            raise ValueError(f"nwgport_msbfs_depths failed: {rc}")
        return out


class Reference:
    """ctypes view of the reference's own bfs.hpp (oracle/_ref/libnwgref.so)."""

    def __init__(self):
        path = build_ref()
        if path is None or not os.path.exists(path):
            raise FileNotFoundError("reference oracle library is not built and the reference sources are absent")
        lib = C.CDLL(path)
        lib.nwgref_graph_create.restype = C.c_void_p
        lib.nwgref_graph_create.argtypes = [_u64p, _u32p, C.c_void_p, C.c_void_p, C.c_uint64]
        lib.nwgref_graph_free.argtypes = [C.c_void_p]
        lib.nwgref_dobfs.restype = C.c_int
        lib.nwgref_dobfs.argtypes = [C.c_void_p, C.c_uint32, C.c_int, C.c_int, C.c_int, C.c_void_p,
                                     C.POINTER(C.c_double)]
        lib.nwgref_bfs_serial.argtypes = [C.c_void_p, C.c_uint32, _u32p]
        lib.nwgref_verify.restype = C.c_int
        lib.nwgref_verify.argtypes = [C.c_void_p, C.c_uint32, _u32p, C.c_uint64]
        lib.nwgref_bc.restype = C.c_int
        lib.nwgref_bc.argtypes = [C.c_void_p, _u32p, C.c_uint64, C.c_int, C.c_int, _f32p, C.POINTER(C.c_double)]
        lib.nwgref_bc_verify.restype = C.c_int
        lib.nwgref_bc_verify.argtypes = [C.c_void_p, _u32p, C.c_uint64, _f32p, C.c_uint64]
        lib.nwgref_threads.restype = C.c_int
        lib.nwgref_set_threads.argtypes = [C.c_int]
        self.lib = lib

    def threads(self) -> int:
        return self.lib.nwgref_threads()

    def set_threads(self, t: int) -> None:
        self.lib.nwgref_set_threads(int(t))

    class Graph:
        def __init__(self, ref, off, cols, in_off=None, in_cols=None):
            self.ref = ref
            self.n = off.size - 1
            self._keep = (off, cols, in_off, in_cols)
            io = in_off.ctypes.data if in_off is not None else None
            ic = in_cols.ctypes.data if in_cols is not None else None
            self.h = ref.lib.nwgref_graph_create(off, cols, io, ic, self.n)

        def dobfs(self, root, num_bins=32, alpha=15, beta=18, want_parents=True):
            parents = np.empty(self.n, np.uint32) if want_parents else None
            secs = C.c_double(0.0)
            self.ref.lib.nwgref_dobfs(self.h, int(root), num_bins, alpha, beta,
                                      parents.ctypes.data if want_parents else None, C.byref(secs))
            return parents, secs.value

        def bfs_serial(self, root):
            parents = np.empty(self.n, np.uint32)
            self.ref.lib.nwgref_bfs_serial(self.h, int(root), parents)
            return parents

        def verify(self, root, parents):
            return self.ref.lib.nwgref_verify(self.h, int(root), np.ascontiguousarray(parents, np.uint32),
                                              self.n) == 1

        def bc(self, sources, threads=0, normalize=True):
            """brandes_bc<float, double>(out, sources, threads): (scores, seconds)."""
            src = np.ascontiguousarray(sources, np.uint32)
            out = np.zeros(self.n, np.float32)
            secs = C.c_double()
            t = int(threads) if threads else self.ref.threads()
            self.ref.lib.nwgref_bc(self.h, src, src.size, t, 1 if normalize else 0, out, C.byref(secs))
            return out, secs.value

        def bc_verify(self, sources, scores):
            src = np.ascontiguousarray(sources, np.uint32)
            return bool(self.ref.lib.nwgref_bc_verify(self.h, src, src.size, np.ascontiguousarray(scores, np.float32),
                                                      self.n))

        def close(self):
            if self.h:
                self.ref.lib.nwgref_graph_free(self.h)
                self.h = None

        def __del__(self):
            try:
                self.close()
            except Exception:
                pass

    def graph(self, off, cols, in_off=None, in_cols=None):
        return Reference.Graph(self, off, cols, in_off, in_cols)


def read_mtx(path: str):
    """MatrixMarket coordinate reader with read_mm's edge semantics
    (io/mmio.hpp:86-103,172-208): 1-based ids; a symmetric file contributes
    both directions of every off-diagonal entry; a general file contributes
    each entry as given; the vertex count is the header's row count, grown
    to cover every id.  Returns (n, u, v) as uint64 arrays (directed pairs)."""
    with open(path) as f:
        header = f.readline().split()
        symmetric = header[4] == "symmetric"
        line = f.readline()
        while line.startswith("%"):
            line = f.readline()
        n0, n1, nnz = (int(x) for x in line.split()[:3])
        u, v = [], []
        for _ in range(nnz):
            parts = f.readline().split()
            a, b = int(parts[0]) - 1, int(parts[1]) - 1
            u.append(a)
            v.append(b)
            if symmetric and a != b:
                u.append(b)
                v.append(a)
    # edge_list::push_back grows the vertex count to max id + 1 (edge_list.hpp:143-147)
    n = max(n0, n1, (max(max(u), max(v)) + 1) if u else 0)
    return n, np.asarray(u, np.uint64), np.asarray(v, np.uint64)
