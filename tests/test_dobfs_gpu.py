"""Parity of the CUDA direction-optimizing BFS with the oracle.

Bar (bit-exact, all integer): per-vertex depths equal the reference's, the
reached set is identical, the parents pass BFSVerifier's rules (checked by
the C restatement, the numpy restatement, and the reference's own
BFSVerifier when oracle/_ref is built), and the device's per-step direction
decisions equal the restatement's (bfs.hpp:186,229,241).
"""
import numpy as np
import pytest

from oracle import graphgen as gg

pytestmark = pytest.mark.gpu

NULL = 0xFFFFFFFF


def _check(nwg, port, reference, off, cols, root, parents, stats, in_off=None, in_cols=None, want_depths=None,
           want_dir=None, want_found=None, numpy_verifier=True):
    n = off.size - 1
    depths = nwg.depths_from_parents(parents, int(root))
    if want_depths is None:
        want_depths = port.depths(off, cols, int(root))
    assert np.array_equal(depths, want_depths), "depths differ from the oracle"
    assert np.array_equal(parents != NULL, want_depths != NULL), "reached set differs"
    assert port.verify(off, cols, root, parents, in_off, in_cols)
    if numpy_verifier:
        assert nwg.bfs_verifier(off, cols, root, parents, in_off, in_cols)
    if reference is not None:
        g = reference.graph(off, cols, in_off, in_cols)
        assert g.verify(int(root), parents), "reference BFSVerifier rejected the device parents"
        g.close()
    if stats is not None:
        tr = stats.trace()
        want_frontier = None
        if want_dir is None:
            _, ptr = port.dobfs(off, cols, int(root), in_off, in_cols)
            want_dir, want_found, want_frontier = ptr["dir"], ptr["found"], ptr["frontier"]
        k = min(len(want_dir), nwg.TRACE_CAP)
        if want_frontier is not None:  # queue sizes entering top-down steps, previous awake counts entering pulls
            assert np.array_equal(tr["frontier"][:k], np.asarray(want_frontier)[:k]), "per-step frontier sizes differ"
        assert stats.status == 0
        assert np.array_equal(tr["dir"][:k], np.asarray(want_dir)[:k]), "direction sequence differs"
        assert np.array_equal(tr["found"][:k], np.asarray(want_found)[:k]), "per-step discoveries differ"
        assert stats.reached == int(np.count_nonzero(want_depths != NULL))
        # the persistent traversal kernel runs the whole traversal in one launch
        assert stats.kernel_launches == 1
        assert stats.levels == int(want_depths[want_depths != NULL].max()) + 1


def test_golden_fixtures(nwg, port, reference, golden):
    for G in golden:
        g = nwg.Graph.from_csr(G.off, G.cols, G.in_off, G.in_cols, validate=True)
        for i, r in enumerate(G.roots):
            parents, st = nwg.bfs(g, g, int(r), 32, 15, 18, stats=True)
            _check(nwg, port, reference, G.off, G.cols, r, parents, st, G.in_off, G.in_cols,
                   want_depths=G.depths[i], want_dir=G.trace_dir[i], want_found=G.trace_found[i])
        g.release()


def test_golden_u32_offsets(nwg, port, reference, golden):
    """NWGraph's default adjacency<0> layout: uint32 offsets, widened on the device."""
    for G in golden[:6]:
        g = nwg.Graph.from_csr(G.off.astype(np.uint32), G.cols,
                               None if G.in_off is None else G.in_off.astype(np.uint32), G.in_cols)
        for i, r in enumerate(G.roots):
            parents = nwg.bfs(g, g, int(r))
            _check(nwg, port, reference, G.off, G.cols, r, parents, None, G.in_off, G.in_cols, want_depths=G.depths[i])
        g.release()


@pytest.mark.parametrize("scale", [12, 16])
def test_rmat_host_graph(nwg, port, reference, scale):
    off, cols = gg.rmat(scale, 16, seed=scale)
    g = nwg.Graph.from_csr(off, cols)
    for r in gg.roots(off, 6, seed=11):
        parents, st = nwg.bfs(g, g, int(r), stats=True)
        _check(nwg, port, reference, off, cols, r, parents, st)
    g.release()


def test_uniform_and_grid_host_graphs(nwg, port, reference):
    for off, cols in (gg.uniform(1 << 14, 32, seed=3), gg.grid(128, 96, 1, seed=4), gg.grid(40, 40, 0, seed=1)):
        g = nwg.Graph.from_csr(off, cols)
        for r in gg.roots(off, 4, seed=5):
            parents, st = nwg.bfs(g, g, int(r), stats=True)
            _check(nwg, port, reference, off, cols, r, parents, st)
        g.release()


def test_directed_graph(nwg, port, reference):
    """out != in: the in-graph is the transpose (bfs.hpp:216 reads in_graph[u])."""
    rng = np.random.default_rng(1)
    n = 5000
    u = rng.integers(0, n, 40000).astype(np.uint64)
    v = rng.integers(0, n, 40000).astype(np.uint64)
    off, cols = gg.directed_csr(u, v, n)
    in_off, in_cols = gg.transpose(off, cols, n)
    g = nwg.Graph.from_csr(off, cols, in_off, in_cols, validate=True)
    for r in gg.roots(off, 6, seed=9):
        parents, st = nwg.bfs(g, g, int(r), stats=True)
        _check(nwg, port, reference, off, cols, r, parents, st, in_off, in_cols)
    g.release()


def test_alpha_beta_variants(nwg, port, reference):
    off, cols = gg.rmat(13, 16, seed=2)
    g = nwg.Graph.from_csr(off, cols)
    r = int(gg.roots(off, 1, seed=3)[0])
    for alpha, beta in ((1, 1), (2, 100), (15, 18), (100, 2), (1000000, 18)):
        parents, st = nwg.bfs(g, g, r, 32, alpha, beta, stats=True)
        _, tr = port.dobfs(off, cols, r, alpha=alpha, beta=beta)
        _check(nwg, port, reference, off, cols, r, parents, st, want_dir=tr["dir"], want_found=tr["found"])
    g.release()


def test_topdown_only(nwg, port):
    off, cols = gg.rmat(12, 16, seed=4)
    g = nwg.Graph.from_csr(off, cols)
    for r in gg.roots(off, 3, seed=1):
        parents, st = nwg.bfs_serial(g, int(r), stats=True)
        assert np.array_equal(nwg.depths_from_parents(parents, int(r)), port.depths(off, cols, int(r)))
        assert st.bu_steps == 0
    g.release()


def test_edge_cases(nwg, port):
    # single vertex, no edges
    g = nwg.Graph.from_csr(np.zeros(2, np.uint64), np.zeros(0, np.uint32))
    assert nwg.bfs(g, g, 0).tolist() == [0]
    g.release()
    # isolated root among edges; self-loops and duplicates
    off, cols = gg.directed_csr(np.array([1, 2, 2, 3, 3], np.uint64), np.array([2, 3, 3, 3, 1], np.uint64), 5)
    g = nwg.Graph.from_csr(off, cols, *gg.transpose(off, cols, 5))
    p = nwg.bfs(g, g, 0)
    assert p.tolist() == [0, NULL, NULL, NULL, NULL]
    p = nwg.bfs(g, g, 1)
    assert nwg.depths_from_parents(p, 1).tolist() == [NULL, 0, 1, 2, NULL]
    g.release()
    # out-of-range root and bad alpha/beta are errors, not faults
    off, cols = gg.rmat(8, 4, seed=1)
    g = nwg.Graph.from_csr(off, cols)
    with pytest.raises(nwg.NwgError) as e:
        nwg.bfs(g, g, g.n)
    assert e.value.code == nwg.NWG_EINVAL
    with pytest.raises(nwg.NwgError):
        nwg.bfs(g, g, 0, 32, 0, 18)
    g.release()
    # malformed CSR is rejected on the host before upload
    with pytest.raises(nwg.NwgError) as e:
        nwg.Graph.from_csr(np.array([0, 1, 2], np.uint64), np.array([1, 7], np.uint32), validate=True)
    assert e.value.code == nwg.NWG_EINVAL
    with pytest.raises(nwg.NwgError):
        nwg.Graph.from_csr(np.array([0, 2, 1], np.uint64), np.array([1, 0], np.uint32), validate=True)
    # an in-CSR with the out-CSR's entry count that is not its transpose:
    # out-edges 0 -> 1, 1 -> 0; the in-CSR claims 2 -> 0, and vertex 2 has no out-edges
    off3, cols3 = np.array([0, 1, 2, 2], np.uint64), np.array([1, 0], np.uint32)
    with pytest.raises(nwg.NwgError) as e:
        nwg.Graph.from_csr(off3, cols3, np.array([0, 1, 2, 2], np.uint64), np.array([2, 0], np.uint32), validate=True)
    assert e.value.code == nwg.NWG_EINVAL and "transpose" in str(e.value)
    g = nwg.Graph.from_csr(off3, cols3, np.array([0, 1, 2, 2], np.uint64), np.array([1, 0], np.uint32), validate=True)
    g.release()


def test_device_generators_match_numpy(nwg):
    cases = [
        (lambda: nwg.Graph.rmat(12, 16, seed=5), lambda: gg.rmat(12, 16, seed=5)),
        (lambda: nwg.Graph.rmat(11, 8, seed=77), lambda: gg.rmat(11, 8, seed=77)),
        (lambda: nwg.Graph.uniform(3000, 12, seed=6), lambda: gg.uniform(3000, 12, seed=6)),
        (lambda: nwg.Graph.grid(70, 33, 1, seed=8), lambda: gg.grid(70, 33, 1, seed=8)),
    ]
    for mk_dev, mk_host in cases:
        g = mk_dev()
        off, cols = g.csr()
        hoff, hcols = mk_host()
        assert np.array_equal(off, hoff)
        assert np.array_equal(cols, hcols)
        assert np.array_equal(g.roots(16, seed=3), gg.roots(hoff, 16, seed=3))
        g.release()


def test_async_workspaces(nwg, port):
    import torch

    off, cols = gg.rmat(14, 16, seed=9)
    g = nwg.Graph.from_csr(off, cols)
    roots = gg.roots(off, 4, seed=2)
    ws = [g.workspace() for _ in range(2)]
    streams = [torch.cuda.Stream() for _ in range(2)]
    outs = [torch.empty(g.n, dtype=torch.int32, device="cuda") for _ in range(2)]
    for k in range(0, roots.size, 2):
        for j in range(2):
            ws[j].bfs_async(int(roots[k + j]), outs[j], streams[j].cuda_stream)
        torch.cuda.synchronize()
        for j in range(2):
            p = outs[j].cpu().numpy().view(np.uint32)
            r = int(roots[k + j])
            assert np.array_equal(nwg.depths_from_parents(p, r), port.depths(off, cols, r))
            assert ws[j].stats().status == 0
    for w in ws:
        w.close()
    g.release()


def test_many_roots_to_host_rows(nwg, port, reference):
    """nwg_bfs_roots: row i is the traversal of roots[i] (odd and even root
    counts, so both lanes end last; a repeated root; a pinned buffer), every
    status is 0; a bad root is refused before anything runs; zero roots is a
    no-op."""
    import torch

    off, cols = gg.rmat(14, 16, seed=21)
    g = nwg.Graph.from_csr(off, cols)
    base = gg.roots(off, 6, seed=4)
    for roots in (base[:5], np.concatenate([base, base[:1]])):
        status = np.full(roots.size, -7, np.int32)
        rows = nwg.bfs_roots(g, roots, status=status)
        assert rows.shape == (roots.size, g.n)
        assert np.all(status == 0)
        for i, r in enumerate(roots):
            _check(nwg, port, reference if i == 0 else None, off, cols, int(r), rows[i], None, numpy_verifier=False)
    pinned = torch.empty((3, g.n), dtype=torch.int32).pin_memory()
    out = nwg.bfs_roots(g, base[:3], parents_out=pinned.numpy().view(np.uint32))
    for i in range(3):
        assert np.array_equal(nwg.depths_from_parents(out[i], int(base[i])), port.depths(off, cols, int(base[i])))
    keep = out.copy()
    with pytest.raises(nwg.NwgError) as ei:
        nwg.bfs_roots(g, np.array([base[0], g.n], np.uint32), parents_out=out)
    assert ei.value.code == nwg.NWG_EINVAL and "roots[1]" in str(ei.value)
    assert np.array_equal(out, keep), "a refused call wrote rows"
    assert nwg.bfs_roots(g, np.zeros(0, np.uint32)).shape == (0, g.n)
    g.release()


def _fan_bipartite(k=100, t=100, n2=1 << 16, d2=16):
    """Root 0 joined to k fan vertices, each joined to all of t targets, beside
    an unreachable uniform component of n2 vertices of degree d2 (one
    symmetric CSR).  From the fan the estimates predict about k * t
    discoveries whose out-degree sum is over twice the switch threshold, but
    the step finds only the t targets (out-degree sum k * t, under the
    threshold), so the reference stays top-down."""
    fan = np.arange(1, k + 1, dtype=np.uint64)
    tgt = np.arange(k + 1, k + t + 1, dtype=np.uint64)
    uu, vv = np.meshgrid(fan, tgt)
    o2, c2 = gg.uniform(n2, d2, seed=3)
    base = 1 + k + t
    src = np.repeat(np.arange(n2, dtype=np.uint64), np.diff(o2).astype(np.int64)) + np.uint64(base)
    u = np.concatenate([np.zeros(k, np.uint64), uu.ravel(), src])
    v = np.concatenate([fan, vv.ravel(), c2.astype(np.uint64) + np.uint64(base)])
    return gg.csr_from_pairs(u, v, base + n2)


def test_marking_topdown_step_that_stays_topdown(nwg, port, reference):
    """A top-down step predicted to hand over to a pull marks its discoveries
    instead of queueing them; when the real out-degree sum keeps the
    traversal top-down (bfs.hpp:186), bitmap -> queue rebuilds the queue
    first.  Depths, parents and the per-step trace equal the oracle's."""
    off, cols = _fan_bipartite()
    g = nwg.Graph.from_csr(off, cols)
    parents, st = nwg.bfs(g, g, 0, 32, 15, 18, stats=True)
    _, tr = port.dobfs(off, cols, 0)
    assert list(tr["dir"]) == [0, 0, 0], "the oracle trace of this graph is top-down only"
    _check(nwg, port, reference, off, cols, 0, parents, st)
    assert st.b2q_steps == 1, "the queue of the fan's step was not rebuilt from its bitmap"
    g.release()


def _path_star(path_n, leaves, fan):
    """A path 0..path_n-1 whose last vertex is a hub with `leaves` leaves,
    each leaf joined to `fan` vertices of a last layer (ids after the
    leaves), as one symmetric CSR."""
    u = list(range(path_n - 1))
    v = list(range(1, path_n))
    hub = path_n - 1
    leaf0 = path_n
    last0 = leaf0 + leaves
    nlast = max(1, leaves // 4)
    rng = np.random.default_rng(5)
    for i in range(leaves):
        u.append(hub)
        v.append(leaf0 + i)
        for t in rng.integers(0, nlast, fan):
            u.append(leaf0 + i)
            v.append(last0 + int(t))
    return gg.csr_from_pairs(np.array(u, np.uint64), np.array(v, np.uint64), last0 + nlast)


def test_solo_levels(nwg, port, reference):
    """Small top-down levels run by one block (solo levels) and handed back to
    the whole grid: a path of 2,000 vertices (eight turns of at most 256 solo
    levels), and a path ending in a hub of 20,000 leaves (the solo frontier
    handed back holds a vertex of 79 chunks, written through hub records).
    Depths, parents, per-step directions, discoveries and frontier sizes
    equal the oracle's; the traversal is still one launch."""
    pn = 2000
    u = np.arange(pn - 1, dtype=np.uint64)
    off, cols = gg.csr_from_pairs(u, u + np.uint64(1), pn)
    g = nwg.Graph.from_csr(off, cols)
    for r in (0, 777, pn - 1):
        parents, st = nwg.bfs(g, g, r, 32, 15, 18, stats=True)
        _check(nwg, port, reference, off, cols, r, parents, st)
    g.release()
    off, cols = _path_star(40, 20000, 3)
    g = nwg.Graph.from_csr(off, cols)
    for r in (0, 20, 39, 40 + 123):
        parents, st = nwg.bfs(g, g, r, 32, 15, 18, stats=True)
        _check(nwg, port, reference, off, cols, r, parents, st)
    g.release()


def test_concurrent_traversals_from_threads(nwg, port):
    """Two host threads, each with its own workspace and stream, run
    traversals at the same time (long paths, whose solo levels keep a
    traversal running while the other is launched, and RMAT); every
    result is exact.  Cooperative launches of a device are chained, so the
    two grids never each hold part of the GPU waiting for the other."""
    import threading

    import torch

    pn = 3000
    u = np.arange(pn - 1, dtype=np.uint64)
    hosts = [gg.csr_from_pairs(u, u + np.uint64(1), pn), gg.rmat(14, 16, seed=4)]
    graphs = [nwg.Graph.from_csr(*h) for h in hosts]
    want = {}
    jobs = []
    for gi, (off, cols) in enumerate(hosts):
        roots = [0, pn // 2] if gi == 0 else [int(r) for r in gg.roots(off, 2, seed=8)]
        for r in roots:
            want[(gi, r)] = port.depths(off, cols, r)
            jobs.append((gi, r))
    errors = []

    def worker(order):
        try:
            stream = torch.cuda.Stream()
            wss = [g.workspace() for g in graphs]
            outs = [torch.empty(g.n, dtype=torch.int32, device="cuda") for g in graphs]
            for _ in range(6):
                for gi, r in order:
                    wss[gi].bfs_async(r, outs[gi], stream.cuda_stream)
                    stream.synchronize()
                    p = outs[gi].cpu().numpy().view(np.uint32)
                    if wss[gi].stats().status != 0 or not np.array_equal(nwg.depths_from_parents(p, r), want[(gi, r)]):
                        errors.append((gi, r, wss[gi].stats().status))
            for w in wss:
                w.close()
        except Exception as e:  # reported below, on the main thread
            errors.append(repr(e))

    threads = [threading.Thread(target=worker, args=(jobs,)), threading.Thread(target=worker, args=(jobs[::-1],))]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    for g in graphs:
        g.release()
    assert not errors, errors[:5]


def test_rmat20_device_graph(nwg, port):
    g = nwg.Graph.rmat(20, 16, seed=1)
    off, cols = g.csr()
    for r in g.roots(3, seed=27491095):
        parents, st = nwg.bfs(g, g, int(r), stats=True)
        _check(nwg, port, None, off, cols, r, parents, st)
        import torch

        dev = torch.empty(g.n, dtype=torch.int32, device="cuda")
        nwg.bfs_device(g, int(r), dev)
        e, v = g.component_edges(dev)
        reached = parents != NULL
        assert v == int(reached.sum())
        assert e == int((off[1:] - off[:-1])[reached].sum())
    g.release()


@pytest.mark.slow
@pytest.mark.parametrize("kind", ["rmat24", "uniform24", "grid4096"])
def test_full_size(nwg, port, kind):
    """The sizes the throughput figures are quoted on; depths bit-exact vs a
    serial BFS of the same CSR copied back to the host."""
    if kind == "rmat24":
        g = nwg.Graph.rmat(24, 16, seed=1)
    elif kind == "uniform24":
        g = nwg.Graph.uniform(1 << 24, 32, seed=1)
    else:
        g = nwg.Graph.grid(4096, 4096, 1, seed=1)
    off, cols = g.csr()
    for r in g.roots(2, seed=27491095):
        parents, st = nwg.bfs(g, g, int(r), stats=True)
        _check(nwg, port, None, off, cols, r, parents, st, numpy_verifier=False)
    g.release()
