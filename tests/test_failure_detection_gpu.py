"""Failure detection without a GPU fault: a device wait that runs out.

The persistent small-frontier kernel's grid barrier is run on a grid that
never completes it (nothing ever sets the flag it waits for).  Every block
must give up after its poll limit and report NWG_ETIMEDOUT through the
control block, the host must read that status, and the context must stay
usable for a traversal afterwards.  No trap, assert, bad address or
unbounded loop is involved.
"""
import ctypes as C

import numpy as np
import pytest

from oracle import graphgen as gg

pytestmark = pytest.mark.gpu


def test_barrier_wait_runs_out_and_context_survives(nwg, port):
    status, ms = C.c_int32(), C.c_float()
    assert nwg.lib.nwg_selftest_wait_timeout(1 << 12, C.byref(status), C.byref(ms)) == nwg.NWG_OK
    assert status.value == nwg.NWG_ETIMEDOUT
    assert 0.0 < ms.value < 2000.0
    # more polls wait longer (the limit, not a fault, ends the wait)
    status2, ms2 = C.c_int32(), C.c_float()
    assert nwg.lib.nwg_selftest_wait_timeout(1 << 15, C.byref(status2), C.byref(ms2)) == nwg.NWG_OK
    assert status2.value == nwg.NWG_ETIMEDOUT and ms2.value > ms.value
    # the context still runs traversals correctly
    off, cols = gg.rmat(12, 16, seed=4)
    g = nwg.Graph.from_csr(off, cols)
    r = int(gg.roots(off, 1, seed=1)[0])
    parents = nwg.bfs(g, g, r)
    assert np.array_equal(nwg.depths_from_parents(parents, r), port.depths(off, cols, r))
    g.release()
    assert nwg.lib.nwg_selftest_wait_timeout(0, C.byref(status), C.byref(ms)) == nwg.NWG_EINVAL
