"""Approximate betweenness centrality (nwg_bc) against the reference.

Bar: the tolerance the reference's BCVerifier states, |score - expected| <=
1e-6 on normalized scores (betweenness_centrality.hpp:117-124), checked here
directly (the reference's check passes its float difference through the
integer abs and so only catches differences of 1 or more), against the C
restatement of BCVerifier's computation and, where oracle/_ref is built,
against NWGraph's brandes_bc<float, double>; its BCVerifier must accept.
Scores are float sums in a different order than the reference's, so they are
compared within that tolerance, not bit for bit; unnormalized scores within
a relative 1e-5.
"""
import numpy as np
import pytest

from oracle import graphgen as gg

pytestmark = pytest.mark.gpu

TOL = 1e-6


def _graphs():
    out = [("rmat10", *gg.rmat(10, 16, seed=1)), ("rmat13", *gg.rmat(13, 16, seed=2)),
           ("uniform", *gg.uniform(4000, 12, seed=3)), ("grid", *gg.grid(40, 30, 1, seed=4)),
           ("grid_plain", *gg.grid(25, 20, 0, seed=5))]
    rng = np.random.default_rng(6)
    n = 3000
    u = rng.integers(0, n, 24000).astype(np.uint64)
    v = rng.integers(0, n, 24000).astype(np.uint64)
    out.append(("directed", *gg.directed_csr(u, v, n)))
    return out


def test_bc_matches_reference(nwg, port, reference):
    for name, off, cols in _graphs():
        g = nwg.Graph.from_csr(off, cols)
        src = gg.roots(off, 16, seed=7)
        got, st = nwg.betweenness(g, src)
        want = port.bc(off, cols, src)
        assert st.sources == src.size and st.max_levels >= 1
        assert np.max(np.abs(got - want)) <= TOL, (name, float(np.max(np.abs(got - want))))
        if reference is not None:
            rg = reference.graph(off, cols)
            theirs, _ = rg.bc(src)
            assert np.max(np.abs(got - theirs)) <= TOL, name
            assert rg.bc_verify(src, got), f"{name}: the reference BCVerifier rejects the device scores"
            rg.close()
        raw, _ = nwg.betweenness(g, src, normalize=False)
        raw_want = port.bc(off, cols, src, normalize=False)
        assert np.allclose(raw, raw_want, rtol=1e-5, atol=1e-5), name
        g.release()


def test_bc_lanes_duplicates_and_edge_cases(nwg, port):
    off, cols = gg.rmat(12, 8, seed=9)
    g = nwg.Graph.from_csr(off, cols)
    src = gg.roots(off, 6, seed=2)
    src = np.concatenate([src, src[:2]])  # duplicate sources count twice, as in the reference
    want = port.bc(off, cols, src)
    for lanes in (1, 3, 8):
        got, st = nwg.betweenness(g, src, lanes=lanes)
        assert st.lanes == min(lanes, src.size)
        assert np.max(np.abs(got - want)) <= TOL
    # a source with no out-edges adds nothing but its own zero dependency
    iso = int(np.flatnonzero(off[1:] == off[:-1])[0])
    got, _ = nwg.betweenness(g, np.array([iso, int(src[0])], np.uint32))
    assert np.max(np.abs(got - port.bc(off, cols, np.array([iso, int(src[0])], np.uint32)))) <= TOL
    with pytest.raises(nwg.NwgError) as e:
        nwg.betweenness(g, np.array([g.n], np.uint32))
    assert e.value.code == nwg.NWG_EINVAL
    g.release()
