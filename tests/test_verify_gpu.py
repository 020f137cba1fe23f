"""Device BFSVerifier (nwg_verify) against the reference's BFSVerifier.

The verdict must equal the reference's on every input; for an invalid
parent array also the vertex the reference stops at (the lowest failing
vertex) and its failure (include/nwgraph/algorithms/bfs.hpp:44-98).  The
expected failure is restated below from the reference's loop, over the
oracle's serial BFS depths.  Invalid arrays are input data: the mistakes are
planted in a copy of the oracle's parents on the host.
"""
import numpy as np
import pytest

from oracle import graphgen as gg

pytestmark = pytest.mark.gpu

NULL = 0xFFFFFFFF


def reference_verdict(port, off, cols, root, parents, in_off=None, in_cols=None):
    """(valid, first failing vertex, reason) following bfs.hpp:64-96 in order."""
    depth = port.depths(off, cols, int(root))
    io, ic = (off, cols) if in_off is None else (in_off, in_cols)
    for u in range(off.size - 1):
        du, pu = int(depth[u]), int(parents[u])
        if du != NULL and pu != NULL:
            if u == root:
                if not (pu == u and du == 0):
                    return False, u, 1
                continue
            nbrs = ic[io[u]:io[u + 1]]
            if np.any(nbrs == pu):
                if int(depth[pu]) != du - 1:
                    return False, u, 2
            else:
                return False, u, 3
        elif du != pu:
            return False, u, 4
    return True, None, 0


def _check(nwg, g, root, parents, want):
    import torch

    for arg in (parents, torch.from_numpy(parents.view(np.int32)).cuda()):
        r = nwg.verify(g, root, arg)
        assert bool(r.valid) == want[0]
        if not want[0]:
            assert (r.first_bad, r.reason) == (want[1], want[2]), nwg.VerifyResult.REASONS[r.reason]


def test_device_verifier_accepts_device_bfs_results(nwg, port, golden):
    for G in golden:
        g = nwg.Graph.from_csr(G.off, G.cols, G.in_off, G.in_cols)
        for r in G.roots:
            parents = nwg.bfs(g, g, int(r))
            res = nwg.verify(g, int(r), parents)
            assert res.valid == 1, (G.name, int(r), nwg.VerifyResult.REASONS[res.reason], res.first_bad)
            assert res.reached == int(np.count_nonzero(parents != NULL))
            assert port.verify(G.off, G.cols, int(r), parents, G.in_off, G.in_cols)
        g.release()


def test_device_verifier_reports_the_references_failure(nwg, port):
    off, cols = gg.rmat(11, 16, seed=9)
    g = nwg.Graph.from_csr(off, cols)
    r = int(gg.roots(off, 1, seed=1)[0])
    parents, _ = port.dobfs(off, cols, r)
    d = port.depths(off, cols, r)
    n = off.size - 1
    cases = []
    p = parents.copy()  # a parent that is not an in-neighbour
    u = int(np.flatnonzero((d != NULL) & (d > 1))[0])
    nbrs = set(cols[off[u]:off[u + 1]].tolist())
    p[u] = next(x for x in range(n) if x not in nbrs and x != u and d[x] != NULL)
    cases.append(p)
    p = parents.copy()  # a parent two levels up
    u = int(np.flatnonzero(d >= 2)[0])
    p[u] = parents[parents[u]]
    cases.append(p)
    p = parents.copy()  # a reached vertex marked unreached
    p[int(np.flatnonzero((d != NULL) & (np.arange(n) != r))[-1])] = NULL
    cases.append(p)
    if np.any(d == NULL):  # an unreached vertex given a parent
        p = parents.copy()
        p[int(np.flatnonzero(d == NULL)[0])] = r
        cases.append(p)
    p = parents.copy()  # root not its own parent
    p[r] = int(cols[off[r]])
    cases.append(p)
    p = parents.copy()  # a parent id out of range
    p[u] = n + 7
    cases.append(p)
    p = parents.copy()  # several mistakes: the lowest vertex is reported
    for v in np.flatnonzero(d >= 2)[:40:7]:
        p[int(v)] = r
    cases.append(p)
    for p in cases:
        want = reference_verdict(port, off, cols, r, p)
        assert not want[0]
        _check(nwg, g, r, p, want)
    _check(nwg, g, r, parents, (True, None, 0))
    g.release()


def test_device_verifier_directed_and_large(nwg, port):
    rng = np.random.default_rng(5)
    n = 6000
    u = rng.integers(0, n, 50000).astype(np.uint64)
    v = rng.integers(0, n, 50000).astype(np.uint64)
    off, cols = gg.directed_csr(u, v, n)
    in_off, in_cols = gg.transpose(off, cols, n)
    g = nwg.Graph.from_csr(off, cols, in_off, in_cols)
    for r in gg.roots(off, 4, seed=3):
        parents = nwg.bfs(g, g, int(r))
        _check(nwg, g, int(r), parents, (True, None, 0))
        bad = parents.copy()
        reached = np.flatnonzero((parents != NULL) & (np.arange(n) != r))
        w = int(reached[len(reached) // 2])
        bad[w] = int(r) if int(parents[w]) != int(r) else NULL
        _check(nwg, g, int(r), bad, reference_verdict(port, off, cols, r, bad, in_off, in_cols))
    g.release()
    import torch

    g = nwg.Graph.rmat(20, 16, seed=1)
    dev = torch.empty(g.n, dtype=torch.int32, device="cuda")
    for r in g.roots(2, seed=27491095):
        nwg.bfs_device(g, int(r), dev)
        res = nwg.verify(g, int(r), dev)
        assert res.valid == 1 and res.reached == g.component_edges(dev)[1]
    g.release()


def test_device_verifier_argument_errors(nwg):
    off, cols = gg.rmat(8, 4, seed=1)
    g = nwg.Graph.from_csr(off, cols)
    with pytest.raises(nwg.NwgError) as e:
        nwg.verify(g, g.n, np.zeros(g.n, np.uint32))
    assert e.value.code == nwg.NWG_EINVAL
    r = nwg.VerifyResult()
    assert nwg.lib.nwg_verify(g.h, 0, None, None, r) == nwg.NWG_EINVAL
    g.release()
