"""CPU checks of the oracle itself: the C restatement (oracle/dobfs_port.c)
against the golden vectors made from the reference's own bfs.hpp, the
reference build (oracle/_ref) against the restatement where it exists, the
seeded generators' invariants, and that the verifiers catch planted
mistakes (planted in the oracle, on the CPU)."""
import os

import numpy as np
import pytest

from oracle import graphgen as gg
from oracle import oracle as O

NULL = 0xFFFFFFFF


def test_port_reproduces_golden_depths_and_directions(port, golden):
    assert len(golden) == 23
    for G in golden:
        for i, r in enumerate(G.roots):
            parents, tr = port.dobfs(G.off, G.cols, int(r), G.in_off, G.in_cols)
            d = port.depths_from_parents(parents, int(r))
            assert np.array_equal(d, G.depths[i]), f"{G.name} root {r}"
            assert np.array_equal(tr["dir"], G.trace_dir[i])
            assert np.array_equal(tr["found"], G.trace_found[i])
            assert port.verify(G.off, G.cols, int(r), parents, G.in_off, G.in_cols)
            assert G.ref_ok[i], "the reference's own BFSVerifier rejected its own result"
            # serial BFS depths (bfs.hpp:110-140) agree as well
            assert np.array_equal(port.depths(G.off, G.cols, int(r)), G.depths[i])


def test_golden_edge_cases_present(golden):
    names = {G.name for G in golden}
    # directed inputs (out != in), a file whose ids exceed its header's size,
    # self-loops and duplicate entries kept as read_mm keeps them
    assert {"bktest2", "flowtest", "tree_2"} <= names
    by = {G.name: G for G in golden}
    assert by["bktest2"].in_off is not None and by["flowtest"].in_off is not None
    assert by["tree_2"].n == 18
    selfloops = sum(int(np.any(G.cols[G.off[u]:G.off[u + 1]] == u)) for G in golden for u in range(G.n))
    assert selfloops > 0
    # unreachable vertices and isolated roots appear in the fixtures
    assert any(np.any(G.depths == NULL) for G in golden)


@pytest.mark.parametrize("threads", [1, 4])
def test_reference_build_matches_restatement(reference, port, threads):
    if reference is None:
        pytest.skip("reference oracle not built here")
    reference.set_threads(threads)
    for scale, seed in ((12, 3), (14, 4)):
        off, cols = gg.rmat(scale, 16, seed=seed)
        g = reference.graph(off, cols)
        for r in gg.roots(off, 4, seed=seed):
            parents, secs = g.dobfs(int(r))
            assert secs > 0
            d = port.depths_from_parents(parents, int(r))
            assert np.array_equal(d, port.depths(off, cols, int(r)))
            mine, _ = port.dobfs(off, cols, int(r))
            assert g.verify(int(r), mine), "reference BFSVerifier rejected the restatement's parents"
            assert port.verify(off, cols, int(r), parents)
            assert np.array_equal(g.bfs_serial(int(r)) != NULL, d != NULL)
        g.close()
    reference.set_threads(0)


def test_verifiers_reject_planted_mistakes(port, reference):
    off, cols = gg.rmat(11, 16, seed=9)
    r = int(gg.roots(off, 1, seed=1)[0])
    parents, _ = port.dobfs(off, cols, r)
    d = port.depths(off, cols, r)
    import nwgr_b200 as nwg  # host helpers only; nothing runs on a GPU here

    bad = []
    # a parent that is not an in-neighbour
    p = parents.copy()
    u = int(np.flatnonzero((d != NULL) & (d > 1))[0])
    nbrs = set(cols[off[u]:off[u + 1]].tolist())
    p[u] = next(x for x in range(off.size - 1) if x not in nbrs and x != u and d[x] != NULL)
    bad.append(p)
    # a parent two levels up
    p = parents.copy()
    u = int(np.flatnonzero(d >= 2)[0])
    p[u] = parents[parents[u]]
    bad.append(p)
    # a reached vertex marked unreached, and an unreached vertex given a parent
    p = parents.copy()
    p[int(np.flatnonzero((d != NULL) & (np.arange(d.size) != r))[0])] = NULL
    bad.append(p)
    if np.any(d == NULL):
        p = parents.copy()
        p[int(np.flatnonzero(d == NULL)[0])] = r
        bad.append(p)
    # root not its own parent
    p = parents.copy()
    p[r] = int(cols[off[r]])
    bad.append(p)
    for p in bad:
        assert not port.verify(off, cols, r, p)
        assert not nwg.bfs_verifier(off, cols, r, p)
        if reference is not None:
            g = reference.graph(off, cols)
            assert not g.verify(r, p)
            g.close()
    assert port.verify(off, cols, r, parents) and nwg.bfs_verifier(off, cols, r, parents)


def _check_csr(off, cols, n, symmetric=True):
    assert off.dtype == np.uint64 and cols.dtype == np.uint32
    assert off.size == n + 1 and off[0] == 0 and off[-1] == cols.size
    assert np.all(off[1:] >= off[:-1])
    assert np.all(cols < n)
    src = np.repeat(np.arange(n, dtype=np.uint64), (off[1:] - off[:-1]).astype(np.int64))
    assert not np.any(src == cols), "self-loop"
    key = (src << np.uint64(32)) | cols.astype(np.uint64)
    assert np.all(key[1:] > key[:-1]), "rows not sorted or duplicated entries"
    if symmetric:
        rkey = (cols.astype(np.uint64) << np.uint64(32)) | src
        assert np.array_equal(np.sort(rkey), key), "not symmetric"


def test_generators_invariants_and_determinism():
    off, cols = gg.rmat(12, 16, seed=3)
    _check_csr(off, cols, 4096)
    off2, cols2 = gg.rmat(12, 16, seed=3)
    assert np.array_equal(off, off2) and np.array_equal(cols, cols2)
    off3, _ = gg.rmat(12, 16, seed=4)
    assert not np.array_equal(off, off3)
    deg = off[1:] - off[:-1]
    assert deg.max() > 20 * deg.mean(), "RMAT skew expected"
    # the vertex permutation is a bijection
    x = np.arange(1 << 12, dtype=np.uint64)
    assert np.unique(gg.permute(x, 12, 3)).size == x.size
    uo, uc = gg.uniform(5000, 20, seed=2)
    _check_csr(uo, uc, 5000)
    assert abs(uc.size / 5000 - 20) < 1.0
    go, gc = gg.grid(30, 20, 1, seed=5)
    _check_csr(go, gc, 600)
    gdeg = go[1:] - go[:-1]
    assert gdeg.min() >= 2 and np.median(gdeg) == 4
    go0, gc0 = gg.grid(30, 20, 0, seed=5)
    assert gc0.size == 2 * ((29 * 20) + (30 * 19))


@pytest.mark.parametrize("kind", ["rmat", "rmat_ef8", "uniform", "grid", "grid_noshort", "grid_thin"])
def test_host_generator_matches_numpy(kind):
    """The multi-threaded host generator (the reference arm's graph source)
    builds the numpy restatement's graphs bit for bit."""
    h = O.HostGen(threads=3)
    a, b = {
        "rmat": (lambda: h.rmat(13, 16, seed=5), lambda: gg.rmat(13, 16, seed=5)),
        "rmat_ef8": (lambda: h.rmat(11, 8, seed=1), lambda: gg.rmat(11, 8, seed=1)),
        "uniform": (lambda: h.uniform(3001, 32, seed=7), lambda: gg.uniform(3001, 32, seed=7)),
        "grid": (lambda: h.grid(41, 29, 1, seed=2), lambda: gg.grid(41, 29, 1, seed=2)),
        "grid_noshort": (lambda: h.grid(16, 16, 0, seed=2), lambda: gg.grid(16, 16, 0, seed=2)),
        "grid_thin": (lambda: h.grid(2, 300, 5, seed=9), lambda: gg.grid(2, 300, 5, seed=9)),
    }[kind]
    (ho, hc), (no, nc) = a(), b()
    assert np.array_equal(ho, no) and np.array_equal(hc, nc)


def test_roots_are_seeded_and_have_out_edges():
    off, cols = gg.rmat(12, 16, seed=7)
    a = gg.roots(off, 64, seed=27491095)
    b = gg.roots(off, 64, seed=27491095)
    assert np.array_equal(a, b)
    assert np.all((off[a + 1] - off[a]) > 0)
    assert a.max() < off.size - 1


def test_rmat16_shape_matches_the_calibration():
    # shape of the reference's own generator pipeline at scale 16: 65,536
    # vertices, ~1.82 M directed entries, max degree ~9.7 k, ~18.7 k isolated
    off, cols = gg.rmat(16, 16, seed=1)
    deg = off[1:] - off[:-1]
    assert off.size - 1 == 65536
    assert 1.75e6 < cols.size < 1.9e6
    assert 5000 < deg.max() < 20000
    assert 15000 < int(np.sum(deg == 0)) < 22000


def test_msbfs_oracle_and_uint8_overflow(port):
    off, cols = gg.rmat(10, 16, seed=2)
    roots = gg.roots(off, 5, seed=3)
    d8 = port.msbfs_depths(off, cols, roots)
    for i, r in enumerate(roots):
        d = port.depths(off, cols, int(r))
        assert np.array_equal(np.where(d == NULL, 255, d).astype(np.uint8), d8[i])
    # a path of 300 vertices has depths >= 255: must be refused, not wrapped
    n = 300
    u = np.arange(n - 1, dtype=np.uint64)
    po, pc = gg.csr_from_pairs(u, u + np.uint64(1), n)
    with pytest.raises(OverflowError):
        port.msbfs_depths(po, pc, np.array([0], np.uint32))


def test_depths_from_parents_host_helper(port):
    import nwgr_b200 as nwg

    off, cols = gg.rmat(11, 16, seed=5)
    r = int(gg.roots(off, 1, seed=2)[0])
    parents, _ = port.dobfs(off, cols, r)
    assert np.array_equal(nwg.depths_from_parents(parents, r), port.depths_from_parents(parents, r))
    cyc = parents.copy()
    a = int(np.flatnonzero((parents != NULL) & (np.arange(parents.size) != r))[0])
    b = int(parents[a])
    if b != r:
        cyc[b] = a  # a two-cycle
        with pytest.raises(ValueError):
            nwg.depths_from_parents(cyc, r)


@pytest.mark.skipif(not O.reference_available(), reason="NWGraph sources not present")
def test_mtx_reader_follows_read_mm():
    # sizes as NWGraph's read_mm loads them (n grows to cover every id)
    base = os.path.join(os.path.dirname(O.REFERENCE_INCLUDE), "data")
    want = {"karate": (34, 156), "tree_2": (18, 42), "bktest2": (27, 50), "sherman4": (1104, 3786)}
    for name, (n, m) in want.items():
        nn, u, v = O.read_mtx(os.path.join(base, name + ".mtx"))
        assert (nn, u.size) == (n, m)


def test_nwbin_fixtures_follow_the_reference_layout(golden):
    """tests/golden/*.nwbin were written by NWGraph's serializers: vertex
    count, is_open, magic, the 8-byte N_ field (N + 1 after fill; with 4-byte
    offsets only its low half comes from N_), offsets, then the target ids."""
    import struct

    by = {G.name: G for G in golden}
    here = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
    for name in ("karate", "bktest2", "sherman4"):
        for kind, osz in (("a0", 4), ("u64", 8)):
            d = open(os.path.join(here, f"{name}.{kind}.nwbin"), "rb").read()
            vcount, = struct.unpack_from("<Q", d, 0)
            assert d[9:43] == b"NW GRAPH indexed_struct_of_arrays\x00"
            nfield, noff, offsz = struct.unpack_from("<QQQ", d, 43)
            assert offsz == osz and noff == vcount + 1
            assert (nfield & ((1 << (8 * osz)) - 1)) == noff
            at = 67
            off = np.frombuffer(d, np.uint32 if osz == 4 else np.uint64, noff, at).astype(np.uint64)
            at += noff * osz
            m, narrays, cnt, elsz = struct.unpack_from("<QQQQ", d, at)
            assert narrays == 1 and cnt == m and elsz == 4
            cols = np.frombuffer(d, np.uint32, m, at + 32)
            G = by[name]
            assert np.array_equal(off, G.off)
            rows = [np.sort(cols[off[u]:off[u + 1]]) for u in range(vcount)]
            assert np.array_equal(np.concatenate(rows), G.cols)


def test_bc_restatement_matches_reference(port, reference):
    """nwgport_bc restates BCVerifier's computation; NWGraph's parallel
    brandes_bc<float, double> and its BCVerifier agree with it."""
    if reference is None:
        pytest.skip("reference oracle not built here")
    for scale, seed in ((10, 1), (12, 2)):
        off, cols = gg.rmat(scale, 16, seed=seed)
        src = gg.roots(off, 8, seed=3)
        mine = port.bc(off, cols, src)
        g = reference.graph(off, cols)
        theirs, secs = g.bc(src)
        assert secs > 0
        assert np.max(np.abs(mine - theirs)) <= 1e-6
        assert g.bc_verify(src, mine) and g.bc_verify(src, theirs)
        # errors planted in the oracle's scores: the reference's BCVerifier
        # takes abs() of a float difference through the integer overload
        # (betweenness_centrality.hpp:119), so it misses anything below 1;
        # the tests here compare |difference| <= 1e-6 themselves
        bad = mine.copy()
        bad[int(np.argmax(mine))] -= 1e-3
        assert g.bc_verify(src, bad) and np.max(np.abs(bad - theirs)) > 1e-6
        bad[int(np.argmax(mine))] += 2.0
        assert not g.bc_verify(src, bad)
        g.close()
