"""Ragged batch: many small graphs, (graph, root) items in one persistent
launch (a CUDA graph), per-item direction parameters.  Every item's depths
must equal the oracle's for its graph and root, bit for bit."""
import numpy as np
import pytest

from oracle import graphgen as gg

pytestmark = pytest.mark.gpu
NULL = 0xFFFFFFFF


def _graphs():
    out = []
    for i, scale in enumerate((8, 9, 10, 11, 12, 9, 10, 8)):
        out.append(gg.rmat(scale, 8 + 3 * i, seed=100 + i))
    for i, (w, h) in enumerate(((16, 16), (40, 25), (64, 48), (7, 300), (100, 3))):
        out.append(gg.grid(w, h, 1, seed=200 + i))
    # a graph with isolated vertices and a self-contained small component
    u = np.array([0, 1, 2, 5, 6], np.uint64)
    v = np.array([1, 2, 0, 6, 7], np.uint64)
    out.append(gg.csr_from_pairs(u, v, 10))
    return out


def test_ragged_batch_matches_oracle(nwg, port):
    graphs = _graphs()
    batch = nwg.RaggedBatch(graphs)
    items, want = [], []
    params = [(15, 18, 32), (1, 1, 64), (1000, 18, 256), (15, 100, 32), (4, 2, 128)]
    for gi, (off, cols) in enumerate(graphs):
        rs = list(gg.roots(off, 3, seed=gi))
        if gi == len(graphs) - 1:
            rs.append(3)  # an isolated root
        for j, r in enumerate(rs):
            a, b, wm = params[(gi + j) % len(params)]
            items.append((gi, int(r), a, b, wm))
            want.append(port.depths(off, cols, int(r)))
    for bps in (1, 2):
        parents, offs, res, ms = batch.run(items, blocks_per_sm=bps)
        host = parents.cpu().numpy().view(np.uint32)
        assert ms > 0
        for i, (gi, r, a, b, wm) in enumerate(items):
            off, cols = graphs[gi]
            n = off.size - 1
            p = host[offs[i]:offs[i] + n]
            d = nwg.depths_from_parents(p, r)
            assert np.array_equal(d, want[i]), f"item {i} graph {gi} root {r}"
            assert port.verify(off, cols, r, p)
            assert res[i].status == 0
            assert res[i].reached == int(np.count_nonzero(want[i] != NULL))
            assert res[i].levels == int(want[i][want[i] != NULL].max()) + 1
    # argument errors are refused before any launch
    with pytest.raises(nwg.NwgError):
        batch.run([(len(graphs), 0, 15, 18, 32)])
    with pytest.raises(nwg.NwgError):
        batch.run([(0, 0, 15, 18, 16)])
    batch.release()


def test_autotuner_picks_and_caches(nwg, port, tmp_path):
    from nwgr_b200.ragged import Autotuner, shape_class

    graphs = _graphs()[:8]
    batch = nwg.RaggedBatch(graphs)
    mn = [(o.size - 1, c.size) for o, c in graphs]
    roots = [gg.roots(o, 2, seed=3) for o, _ in graphs]
    path = tmp_path / "cache.json"
    tuner = Autotuner(str(path))
    params, bps = tuner.tune(batch, mn, roots, sample=2)
    assert set(params) == {shape_class(n, m) for n, m in mn}
    assert bps in (1, 2, 3) and path.exists()
    again = Autotuner(str(path))
    assert again.entry["blocks_per_sm"] == bps
    for cls, p in params.items():
        assert again.class_params(cls) == p
    items = Autotuner.items(mn, roots, params)
    parents, offs, res, _ = batch.run(items, blocks_per_sm=bps)
    host = parents.cpu().numpy().view(np.uint32)
    for i, (gi, r, *_rest) in enumerate(items):
        off, cols = graphs[gi]
        d = nwg.depths_from_parents(host[offs[i]:offs[i] + off.size - 1], r)
        assert np.array_equal(d, port.depths(off, cols, r))
    batch.release()
