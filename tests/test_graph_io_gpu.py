"""Graph files into the registry (nwg_graph_read / nwg_graph_write_nwbin).

NW binary: the files in tests/golden/*.nwbin were written by NWGraph's own
serializers (tests/golden/make_nwbin.py) from its data/ fixtures, with 4- and
8-byte offsets.  MatrixMarket: files written here from the golden CSRs in
both symmetries, with comments, values and CRLF line endings.  Each read
graph must hold exactly the golden CSR (rows sorted, self-loops and
duplicates kept) and give the golden depths.
"""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
NULL = 0xFFFFFFFF


def _by_name(golden):
    return {G.name: G for G in golden}


def _check_graph(nwg, g, G):
    off, cols = g.csr()
    assert np.array_equal(off, G.off) and np.array_equal(cols, G.cols)
    for i, r in enumerate(G.roots):
        parents = nwg.bfs(g, g, int(r))
        assert np.array_equal(nwg.depths_from_parents(parents, int(r)), G.depths[i]), (G.name, int(r))


@pytest.mark.parametrize("kind", ["a0", "u64"])
@pytest.mark.parametrize("name", ["karate", "bktest2", "sherman4"])
def test_reads_reference_written_binaries(nwg, golden, name, kind):
    G = _by_name(golden)[name]
    g = nwg.Graph.read(os.path.join(HERE, f"{name}.{kind}.nwbin"))
    assert g.n == G.n
    _check_graph(nwg, g, G)
    g.release()


def _write_mm(path, G, symmetric, values, crlf):
    nl = "\r\n" if crlf else "\n"
    src = np.repeat(np.arange(G.n, dtype=np.uint64), (G.off[1:] - G.off[:-1]).astype(np.int64))
    dst = G.cols.astype(np.uint64)
    if symmetric:
        keep = src >= dst  # the lower triangle: read_mm adds the other direction
        src, dst = src[keep], dst[keep]
    field = "integer" if values else "pattern"
    lines = [f"%%MatrixMarket matrix coordinate {field} {'symmetric' if symmetric else 'general'}",
             "% written by the test", "%another comment", f"{G.n} {G.n} {src.size}"]
    for k, (a, b) in enumerate(zip(src.tolist(), dst.tolist())):
        lines.append(f"{a + 1} {b + 1} {k % 7 + 1}" if values else f"{a + 1} {b + 1}")
    open(path, "w", newline="").write(nl.join(lines) + nl)


def test_reads_matrix_market_like_read_mm(nwg, golden, tmp_path):
    for G in golden:
        symmetric = G.in_off is None
        for values, crlf in ((False, False), (True, True)):
            p = tmp_path / f"{G.name}.mtx"
            _write_mm(str(p), G, symmetric, values, crlf)
            g = nwg.Graph.read(str(p))
            assert g.n == G.n
            _check_graph(nwg, g, G)
            g.release()


def test_write_read_round_trip_and_errors(nwg, tmp_path):
    g = nwg.Graph.rmat(12, 16, seed=3)
    p = str(tmp_path / "g.nwbin")
    g.write_nwbin(p)
    h = nwg.Graph.read(p, symmetric=True)
    a, b = g.csr(), h.csr()
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
    h.release()
    g.release()
    with pytest.raises(nwg.NwgError) as e:
        nwg.Graph.read(str(tmp_path / "missing.mtx"))
    assert e.value.code == nwg.NWG_EINVAL
    bad = tmp_path / "bad.bin"
    bad.write_bytes(b"\x00" * 100)
    with pytest.raises(nwg.NwgError):
        nwg.Graph.read(str(bad))
    trunc = tmp_path / "trunc.nwbin"
    trunc.write_bytes(open(os.path.join(HERE, "karate.u64.nwbin"), "rb").read()[:200])
    with pytest.raises(nwg.NwgError):
        nwg.Graph.read(str(trunc))
    mm = tmp_path / "short.mtx"
    mm.write_text("%%MatrixMarket matrix coordinate pattern general\n3 3 4\n1 2\n2 3\n")
    with pytest.raises(nwg.NwgError) as e:
        nwg.Graph.read(str(mm))
    assert "entry 3" in str(e.value)
