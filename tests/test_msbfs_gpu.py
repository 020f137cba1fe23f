"""Batched multi-source BFS (64 sources per 64-bit word, up to 256 per
pass): every source's uint8 depths must equal an independent single-source
BFS of the same root (the oracle), bit for bit; 255 = unreached."""
import numpy as np
import pytest

from oracle import graphgen as gg

pytestmark = pytest.mark.gpu

NULL = 0xFFFFFFFF


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
        if max(max(int(r), n - 1 - int(r)) for r in roots) >= 255:  # a depth beyond uint8
            with pytest.raises(nwg.NwgError) as e:
                ws.run(roots, d)
            assert e.value.code == nwg.NWG_EOVERFLOW
            continue
        ws.run(roots, d)
        assert np.array_equal(d.cpu().numpy(), port.msbfs_depths(off, cols, roots))
    ws.close()
    g.release()


def path_plus_rmat(path_n=400):
    """A path of path_n vertices (ids 0..path_n-1, diameter path_n - 1) beside
    an RMAT-10 graph (ids from path_n on), as one symmetric CSR."""
    u = np.arange(path_n - 1, dtype=np.uint64)
    roff, rcols = gg.rmat(10, 16, seed=3)
    ru = np.repeat(np.arange(roff.size - 1, dtype=np.uint64), (roff[1:] - roff[:-1]).astype(np.int64))
    pu = np.concatenate([u, ru + np.uint64(path_n)])
    pv = np.concatenate([u + np.uint64(1), rcols.astype(np.uint64) + np.uint64(path_n)])
    return gg.csr_from_pairs(pu, pv, path_n + roff.size - 1)


def test_msbfs_deep_sources_fail_alone(nwg, port):
    """Sources whose depths reach 255 share passes with ordinary ones: the
    uint8 call reports them one by one (their rows stop at 254, every other
    row is exact), and the uint16 rows are exact for all of them."""
    import torch

    path_n = 400
    off, cols = path_plus_rmat(path_n)
    n = off.size - 1
    g = nwg.Graph.from_csr(off, cols)
    rng = np.random.default_rng(11)
    roots = np.concatenate([np.array([0, 399, 145, 254, 255, 200, 3], np.uint32),
                            gg.roots(off[path_n:] - off[path_n], 60, seed=2) + path_n])
    rng.shuffle(roots)
    want = np.stack([port.depths(off, cols, int(r)) for r in roots])  # uint32, NULL = unreached
    deep = np.where(want == NULL, 0, want).max(axis=1) >= 255
    assert 0 < deep.sum() < roots.size
    with pytest.raises(nwg.NwgError) as e:
        nwg.msbfs(g, roots)
    assert e.value.code == nwg.NWG_EOVERFLOW
    ws = nwg.MsWorkspace(g)
    d8 = torch.empty((roots.size, n), dtype=torch.uint8, device="cuda")
    flags = np.zeros(roots.size, np.uint8)
    st = ws.run_ex(roots, d8, flags)
    assert st.status == 0 and st.deep_sources == deep.sum()
    assert np.array_equal(flags.astype(bool), deep)
    h8 = d8.cpu().numpy()
    w8 = np.where(want == NULL, 255, np.minimum(want, 255)).astype(np.uint8)
    assert np.array_equal(h8[~deep], w8[~deep])
    assert np.array_equal(np.where(w8[deep] < 255, h8[deep], 255), w8[deep])  # deep rows exact up to 254
    d16 = torch.empty((roots.size, n), dtype=torch.int16, device="cuda")
    flags[:] = 7
    st = ws.run_ex(roots, d16, flags)
    assert st.status == 0 and np.array_equal(flags.astype(bool), deep)
    w16 = np.where(want == NULL, 0xFFFF, want).astype(np.uint16)
    assert np.array_equal(d16.cpu().numpy().view(np.uint16), w16)
    # the workspace is clean after deep passes: a plain pass afterwards is exact
    ok = roots[~deep][:64]
    d8b = torch.empty((ok.size, n), dtype=torch.uint8, device="cuda")
    ws.run(ok, d8b)
    assert np.array_equal(d8b.cpu().numpy(), port.msbfs_depths(off, cols, ok))
    ws.close()
    d, st = nwg.msbfs(g, roots, depth_bytes=2)
    assert np.array_equal(d, w16) and st.deep_sources == deep.sum()
    g.release()


def test_msbfs_many_passes_in_flight(nwg, port):
    """More than 256 sources: up to four passes run at once on their own
    lanes (pass state and stream); every row equals the single-source
    oracle's, in both row widths, and on a second call that reuses the lanes."""
    import torch

    off, cols = gg.rmat(12, 16, seed=5)
    n = off.size - 1
    g = nwg.Graph.from_csr(off, cols)
    roots = gg.roots(off, 1100, seed=9)  # five passes, the last of 76 sources
    want = port.msbfs_depths(off, cols, roots)
    ws = nwg.MsWorkspace(g)
    for _ in range(2):
        d = torch.empty((roots.size, n), dtype=torch.uint8, device="cuda")
        st = ws.run(roots, d)
        assert st.passes == 5 and np.array_equal(d.cpu().numpy(), want)
    d16 = torch.empty((roots.size, n), dtype=torch.int16, device="cuda")
    ws.run_ex(roots, d16)
    w16 = want.astype(np.uint16)
    w16[want == 255] = 0xFFFF
    assert np.array_equal(d16.cpu().numpy().view(np.uint16), w16)
    ws.close()
    g.release()
