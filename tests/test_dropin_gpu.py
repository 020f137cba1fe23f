"""The C++20 drop-in header (include/nwgraph/algorithms/bfs.hpp) used the way
NWGraph's bench/bfs.cpp uses the reference: NWGraph's read_mm, adjacency<1>
as the out-graph, adjacency<0> as the in-graph, nw::graph::bfs and
BFSVerifier (tests/cpp/dropin_test.cpp, built against NWGraph's headers
where they are available).  Depths must equal the reference's golden depths.
"""
import os
import subprocess

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu
NULL = 0xFFFFFFFF


def _write_mtx(path, off, cols):
    """MatrixMarket 'general' file whose adjacency<1> is the given out-CSR:
    an out-edge u -> v is written as the pair (v, u), so row u of
    adjacency<1> (grouped by the second index) holds v."""
    n = off.size - 1
    src = np.repeat(np.arange(n), (off[1:] - off[:-1]).astype(np.int64))
    with open(path, "w") as f:
        f.write("%%MatrixMarket matrix coordinate pattern general\n")
        f.write(f"{n} {n} {cols.size}\n")
        f.write("".join(f"{int(v) + 1} {int(u) + 1}\n" for u, v in zip(src, cols)))


def test_dropin_header_matches_reference(nwg, port, golden, tmp_path):
    exe = O.build_dropin_test()
    if exe is None or not os.path.exists(exe):
        pytest.skip("drop-in test program not built (needs the NWGraph headers at build time)")
    picked = [G for G in golden if G.name in ("karate", "bktest2", "flowtest", "delaunay_n10", "G1", "rmat11")]
    assert len(picked) == 6
    for G in picked:
        mtx = tmp_path / f"{G.name}.mtx"
        _write_mtx(mtx, G.off, G.cols)
        prefix = tmp_path / G.name
        res = subprocess.run([exe, str(mtx), str(prefix)] + [str(int(r)) for r in G.roots], capture_output=True,
                             text=True, timeout=300)
        assert res.returncode == 0, res.stdout + res.stderr
        for i, r in enumerate(G.roots):
            for suffix in (".bin", ".td.bin"):
                p = np.fromfile(f"{prefix}.{int(r)}{suffix}", dtype=np.uint32)
                assert p.size == G.n
                d = nwg.depths_from_parents(p, int(r))
                assert np.array_equal(d, G.depths[i]), f"{G.name} root {r} {suffix}: depths differ"
                assert port.verify(G.off, G.cols, int(r), p, G.in_off, G.in_cols)


def test_dropin_strict_mode_sees_in_place_changes(golden, tmp_path):
    """With NWG_DROPIN_STRICT=1 every drop-in call uploads the graph again: a
    column changed in place at an entry the registry's sampled fingerprint
    does not read is seen by the next call (its depths equal a serial BFS of
    the changed graph), as the reference's bfs would see it."""
    exe = O.build_dropin_test()
    if exe is None or not os.path.exists(exe):
        pytest.skip("drop-in test program not built (needs the NWGraph headers at build time)")
    G = next(G for G in golden if G.name == "rmat11")
    mtx = tmp_path / "rmat11.mtx"
    _write_mtx(mtx, G.off, G.cols)
    env = dict(os.environ, NWG_DROPIN_STRICT="1")
    for r in G.roots[:2]:
        res = subprocess.run([exe, "--mutate", str(mtx), str(int(r))], capture_output=True, text=True, timeout=300,
                             env=env)
        assert res.returncode == 0, res.stdout + res.stderr
        assert "mutation_seen 1" in res.stdout, res.stdout
