"""nwg_bfs_noalloc: the traversal for callers that may not allocate device
memory (cudaMalloc/cudaFree synchronise the device, so latency-bound
services and processes whose device memory belongs to their own allocator
forbid them).  The entry point keeps all its scratch in one static device
array; the caller owns inputs and outputs.

Checked through the C ABI against the registered-graph entry point nwg_bfs,
with the bar every parity test here uses: depths bit-exact and the reached
set identical (parent identity may differ where top-down claims race), the
parents passing BFSVerifier's rules -- on two calls in a row, since every
call reuses the same static scratch.  Named to be collected last.
"""
import numpy as np
import pytest

from oracle import graphgen as gg

pytestmark = pytest.mark.gpu

NULL = 0xFFFFFFFF


def _dev(torch, a):
    return torch.from_numpy(a.view(np.int64) if a.dtype == np.uint64 else a.view(np.int32)).cuda()


def test_noalloc_matches_registered_entry_point(nwg, port):
    import torch

    cases = []
    off, cols = gg.rmat(16, 16, seed=16)  # 65,536 vertices, ~1.8 M entries: inside the static limits
    cases.append((off, cols, None, None))
    rng = np.random.default_rng(3)
    n = 20000
    u = rng.integers(0, n, 150000).astype(np.uint64)
    v = rng.integers(0, n, 150000).astype(np.uint64)
    doff, dcols = gg.directed_csr(u, v, n)
    dioff, dicols = gg.transpose(doff, dcols, n)
    cases.append((doff, dcols, dioff, dicols))

    for off, cols, in_off, in_cols in cases:
        n = off.size - 1
        g = nwg.Graph.from_csr(off, cols, in_off, in_cols)
        off_d, col_d = _dev(torch, off), _dev(torch, cols)
        in_off_d = _dev(torch, in_off) if in_off is not None else None
        in_col_d = _dev(torch, in_cols) if in_cols is not None else None
        par_d = torch.empty(n, dtype=torch.int32, device="cuda")
        roots = gg.roots(off, 3, seed=5)
        for call in range(2):  # two calls in a row reuse the same static scratch
            for r in roots:
                r = int(r)
                want = nwg.bfs(g, g, r)
                nwg.bfs_noalloc(off_d, col_d, n, r, par_d, in_off_d, in_col_d)
                torch.cuda.synchronize()
                got = par_d.cpu().numpy().view(np.uint32)
                d_want = nwg.depths_from_parents(want, r)
                d_got = nwg.depths_from_parents(got, r)
                assert np.array_equal(d_got, d_want), f"call {call}, root {r}: depths differ"
                assert np.array_equal(got != NULL, want != NULL)
                assert port.verify(off, cols, r, got, in_off, in_cols)
        g.release()


def test_noalloc_rejects_graphs_over_the_limit(nwg):
    import torch

    n = (1 << 20) + 1
    off = torch.zeros(n + 1, dtype=torch.int64, device="cuda")
    col = torch.zeros(4, dtype=torch.int32, device="cuda")
    par = torch.empty(n, dtype=torch.int32, device="cuda")
    with pytest.raises(nwg.NwgError) as e:
        nwg.bfs_noalloc(off, col, n, 0, par)
    assert e.value.code == nwg.NWG_EINVAL
    assert "limit" in str(e.value)


def test_noalloc_rejects_entry_counts_over_the_limit_and_non_transposes(nwg):
    """Refusals that come before any launch: more CSR entries than the static
    scratch holds (read from out_off[n]), and an in-CSR whose entry count
    differs from the out-CSR's."""
    import torch

    big = (1 << 24) + 1
    off = torch.tensor([0, big, big], dtype=torch.int64, device="cuda")
    col = torch.zeros(4, dtype=torch.int32, device="cuda")
    par = torch.empty(2, dtype=torch.int32, device="cuda")
    with pytest.raises(nwg.NwgError) as e:
        nwg.bfs_noalloc(off, col, 2, 0, par)
    assert e.value.code == nwg.NWG_EINVAL and "limit" in str(e.value)
    off = torch.tensor([0, 1, 2], dtype=torch.int64, device="cuda")
    col = torch.tensor([1, 0, 0, 0], dtype=torch.int32, device="cuda")
    in_off = torch.tensor([0, 1, 3], dtype=torch.int64, device="cuda")
    in_col = torch.tensor([1, 0, 0, 0], dtype=torch.int32, device="cuda")
    with pytest.raises(nwg.NwgError) as e:
        nwg.bfs_noalloc(off, col, 2, 0, par, in_off, in_col)
    assert e.value.code == nwg.NWG_EINVAL and "transpose" in str(e.value)


@pytest.mark.parametrize("kind", ["uniform_at_n_limit", "rmat19"])
def test_noalloc_near_the_limits(nwg, port, kind):
    """Graphs at the static limits (2^20 vertices; just under 2^24 entries),
    where the frontier queues fill to their full sizes: depths equal the
    registered entry point's on two calls in a row."""
    import torch

    off, cols = gg.uniform(1 << 20, 15, seed=4) if kind == "uniform_at_n_limit" else gg.rmat(19, 16, seed=2)
    n = off.size - 1
    assert cols.size < (1 << 24)
    g = nwg.Graph.from_csr(off, cols)
    off_d, col_d = _dev(torch, off), _dev(torch, cols)
    par_d = torch.empty(n, dtype=torch.int32, device="cuda")
    for r in gg.roots(off, 2, seed=8):
        r = int(r)
        want = nwg.depths_from_parents(nwg.bfs(g, g, r), r)
        for _ in range(2):
            nwg.bfs_noalloc(off_d, col_d, n, r, par_d)
            torch.cuda.synchronize()
            got = par_d.cpu().numpy().view(np.uint32)
            assert np.array_equal(nwg.depths_from_parents(got, r), want)
            assert port.verify(off, cols, r, got)
    g.release()
