"""CPU checks of the C-ABI boundary: libnwgr_b200.so loads, exports exactly
the functions include/nwg_bfs.h declares (and nothing of the reference's
templates), and the argument checks that need no GPU return the documented
status with a message.  No compute call is made here."""
import ctypes as C
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "nwg_bfs.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"^(?:int|const char\*)\s+(nwg_\w+)\s*\(", src, flags=re.M)))


def test_library_exports_every_declared_symbol(nwg):
    decl = declared_functions()
    assert len(decl) >= 20
    for name in decl:
        assert hasattr(nwg.lib, name), name
    assert sorted(nwg.EXPORTED) == decl
    out = subprocess.run(["nm", "-D", "--defined-only", nwg.LIB_PATH], capture_output=True, text=True).stdout
    exported = sorted(l.split()[-1] for l in out.splitlines() if " T " in l)
    assert exported == decl, "the library exports something the header does not declare (or vice versa)"


def test_version_and_error_paths_without_gpu(nwg):
    assert "sm_100a" in nwg.version()
    assert nwg.lib.nwg_graph_release(None) == nwg.NWG_EINVAL
    assert "NULL" in nwg.last_error()
    n = C.c_uint64()
    assert nwg.lib.nwg_graph_info(None, C.byref(n), None, None) == nwg.NWG_EINVAL
    assert nwg.lib.nwg_bfs(None, 0, 15, 18, None, None, None) == nwg.NWG_EINVAL
    # many roots: a NULL graph, or roots without a host output, are refused before any device call
    assert nwg.lib.nwg_bfs_roots(None, None, 0, 15, 18, None, None) == nwg.NWG_EINVAL
    roots = (C.c_uint32 * 2)(0, 1)
    assert nwg.lib.nwg_bfs_roots(C.c_void_p(1), roots, 2, 15, 18, None, None) == nwg.NWG_EINVAL
    assert "NULL" in nwg.last_error()
    assert nwg.lib.nwg_ws_stats(None, None) == nwg.NWG_EINVAL
    assert nwg.lib.nwg_gen_rmat(0, 16, 1, 1, 2, 3, C.byref(C.c_void_p())) == nwg.NWG_EINVAL
    assert nwg.lib.nwg_gen_rmat(10, 16, 1, 5, 2, 3, C.byref(C.c_void_p())) == nwg.NWG_EINVAL
    # the no-allocation entry point refuses out-of-limit sizes before touching the device
    assert nwg.lib.nwg_bfs_noalloc(None, None, None, None, 10, 0, 15, 18, None, None) == nwg.NWG_EINVAL
    # the server refuses an empty graph set and unknown handles without a device
    h = C.c_void_p()
    assert nwg.lib.nwg_server_create(None, 0, None, C.byref(h)) == nwg.NWG_EINVAL and not h.value
    assert nwg.lib.nwg_server_destroy(None) == nwg.NWG_EINVAL
    assert nwg.lib.nwg_server_run_trace(None, 0, None, None, None, None, None, None, None) == nwg.NWG_EINVAL
    buf = C.create_string_buffer(8)
    length = nwg.lib.nwg_last_error(buf, 8)
    assert length > 7 and len(buf.value) == 7  # truncated, NUL-terminated


def test_registration_rejects_bad_host_arguments_before_upload(nwg):
    import numpy as np

    h = C.c_void_p()
    off = np.array([0, 1, 2], np.uint64)
    col = np.array([1, 0], np.uint32)
    # in_off without in_col
    rc = nwg.lib.nwg_graph_register(off.ctypes.data, col.ctypes.data, 2, off.ctypes.data, None, 0, C.byref(h))
    assert rc == nwg.NWG_EINVAL
    rc = nwg.lib.nwg_graph_register(None, col.ctypes.data, 2, None, None, 0, C.byref(h))
    assert rc == nwg.NWG_EINVAL
    rc = nwg.lib.nwg_graph_register(off.ctypes.data, col.ctypes.data, 1 << 32, None, None, 0, C.byref(h))
    assert rc == nwg.NWG_EINVAL


def test_drop_in_header_compiles_standalone(tmp_path):
    """The drop-in header needs NWGraph's own headers; without them only the
    C header can be checked (it must be valid C)."""
    c = tmp_path / "t.c"
    c.write_text('#include "nwg_bfs.h"\nint main(void){ nwg_bfs_stats s; (void)s; return 0; }\n')
    subprocess.check_call(["gcc", "-std=c99", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"), "-c", str(c),
                           "-o", str(tmp_path / "t.o")])
