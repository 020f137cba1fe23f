"""Batched multi-source BFS (64 sources per 64-bit word, up to 256 per
pass): every source's uint8 depths must equal an independent single-source
BFS of the same root (the oracle), bit for bit; 255 = unreached."""
import numpy as np
import pytest

from oracle import graphgen as gg

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("k", [1, 5, 64, 100, 256, 300])
def test_msbfs_rmat_matches_single_source(nwg, port, k):
    off, cols = gg.rmat(13, 16, seed=21)
    g = nwg.Graph.from_csr(off, cols)
    roots = gg.roots(off, k, seed=k)
    d, st = nwg.msbfs(g, roots)
    assert st.status == 0 and st.passes == (k + 255) // 256
    assert np.array_equal(d, port.msbfs_depths(off, cols, roots))
    g.release()


def test_msbfs_other_graphs_duplicates_and_directed(nwg, port):
    graphs = [gg.uniform(1 << 13, 24, seed=2), gg.grid(60, 50, 1, seed=3), gg.grid(20, 10, 0, seed=1)]
    for off, cols in graphs:
        g = nwg.Graph.from_csr(off, cols)
        roots = np.concatenate([gg.roots(off, 70, seed=4), gg.roots(off, 3, seed=4)])  # duplicated roots
        d, _ = nwg.msbfs(g, roots)
        assert np.array_equal(d, port.msbfs_depths(off, cols, roots))
        g.release()
    rng = np.random.default_rng(5)
    n = 4000
    off, cols = gg.directed_csr(rng.integers(0, n, 30000).astype(np.uint64), rng.integers(0, n, 30000).astype(np.uint64), n)
    ioff, icols = gg.transpose(off, cols, n)
    g = nwg.Graph.from_csr(off, cols, ioff, icols)
    roots = gg.roots(off, 130, seed=6)
    d, _ = nwg.msbfs(g, roots)
    assert np.array_equal(d, port.msbfs_depths(off, cols, roots))
    g.release()


def test_msbfs_depth_overflow_is_refused(nwg):
    n = 400
    u = np.arange(n - 1, dtype=np.uint64)
    off, cols = gg.csr_from_pairs(u, u + np.uint64(1), n)
    g = nwg.Graph.from_csr(off, cols)
    with pytest.raises(nwg.NwgError) as e:
        nwg.msbfs(g, np.array([0, 5], np.uint32))
    assert e.value.code == nwg.NWG_EOVERFLOW
    d, _ = nwg.msbfs(g, np.array([n // 2], np.uint32))  # depth <= 200 fits
    assert d[0, 0] == n // 2 and d[0, n - 1] == n - 1 - n // 2
    g.release()


def test_msbfs_rmat20_device_graph(nwg, port):
    g = nwg.Graph.rmat(20, 16, seed=1)
    off, cols = g.csr()
    roots = g.roots(256, seed=27491095)
    d, st = nwg.msbfs(g, roots)
    sample = [0, 1, 63, 64, 200, 255]
    want = port.msbfs_depths(off, cols, roots[sample])
    assert np.array_equal(d[sample], want)
    assert st.push_levels > 0 and st.pull_levels > 0
    g.release()


def test_msbfs_odd_n_and_unaligned_rows(nwg, port):
    """An odd vertex count and a depth array that starts at an odd address:
    the depth rows are then written byte by byte, and every byte of every
    row must still be right, with nothing written outside the rows."""
    import torch

    off, cols = gg.grid(61, 49, 1, seed=7)  # n = 2989
    n = off.size - 1
    g = nwg.Graph.from_csr(off, cols)
    ws = nwg.MsWorkspace(g)
    for k in (7, 70):
        roots = gg.roots(off, k, seed=k)
        buf = torch.full((k * n + 2,), 7, dtype=torch.uint8, device="cuda")
        ws.run(roots, buf[1 : 1 + k * n])
        h = buf.cpu().numpy()
        assert h[0] == 7 and h[-1] == 7
        assert np.array_equal(h[1:-1].reshape(k, n), port.msbfs_depths(off, cols, roots))
    ws.close()
    g.release()


def test_msbfs_workspace_reuse_after_deep_and_overflowing_passes(nwg, port):
    """One workspace, passes in a row on a 400-vertex path: depths up to 253
    (all eight level planes), passes that stop on a depth overflow, and
    passes after them.  The planes must be clear again after each pass."""
    import torch

    n = 400
    u = np.arange(n - 1, dtype=np.uint64)
    off, cols = gg.csr_from_pairs(u, u + np.uint64(1), n)
    g = nwg.Graph.from_csr(off, cols)
    ws = nwg.MsWorkspace(g)
    d = torch.empty((2, n), dtype=torch.uint8, device="cuda")
    for roots in ([200, 150], [0, 5], [180, 253], [230, 146], [3, 399]):
        roots = np.asarray(roots, np.uint32)
        if max(max(int(r), n - 1 - int(r)) for r in roots) >= 254:  # a level 255 would have to be tried
            with pytest.raises(nwg.NwgError) as e:
                ws.run(roots, d)
            assert e.value.code == nwg.NWG_EOVERFLOW
            continue
        ws.run(roots, d)
        assert np.array_equal(d.cpu().numpy(), port.msbfs_depths(off, cols, roots))
    ws.close()
    g.release()
