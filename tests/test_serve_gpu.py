"""Serving loop (nwg_server): each query's answer is the same alone and in
the mix.

An answer is the uint8 depth row of one (graph, root) single-source BFS
(255 = unreached), bit-exact against the oracle's serial BFS.  "Alone": a
server with one slot and batches of one, each query submitted and awaited
by itself.  "In the mix": the same queries replayed as a burst and as a
Poisson stream through a server with several slots, so queries are
coalesced into multi-source passes with other queries (same graph,
different roots, duplicates included) while other passes run on other
streams.  The tolerance is zero: depths are integers.
"""
import numpy as np
import pytest

from oracle import graphgen as gg

pytestmark = pytest.mark.gpu

NULL = 0xFFFFFFFF


def _u8(d):
    return np.where(d == NULL, 255, d).astype(np.uint8)


@pytest.fixture(scope="module")
def served(nwg):
    rng = np.random.default_rng(4)
    host = [gg.rmat(10, 16, seed=1), gg.rmat(12, 8, seed=2), gg.rmat(13, 24, seed=3), gg.grid(40, 30, 1, seed=4),
            gg.grid(64, 64, 1, seed=5), gg.uniform(3000, 12, seed=6)]
    # a directed graph (pull passes read the in-CSR)
    n = 2500
    u = rng.integers(0, n, 20000).astype(np.uint64)
    v = rng.integers(0, n, 20000).astype(np.uint64)
    doff, dcols = gg.directed_csr(u, v, n)
    host.append((doff, dcols) + gg.transpose(doff, dcols, n))
    graphs = [nwg.Graph.from_csr(*h) for h in host]
    pools = [gg.roots(h[0], 8, seed=i + 1) for i, h in enumerate(host)]
    yield host, graphs, pools
    for g in graphs:
        g.release()


def _queries(pools, count, seed):
    rng = np.random.default_rng(seed)
    gid = rng.integers(0, len(pools), count).astype(np.uint32)
    roots = np.array([pools[g][rng.integers(0, pools[g].size)] for g in gid], np.uint32)
    return gid, roots


def test_each_answer_same_alone_and_in_the_mix(nwg, port, served):
    host, graphs, pools = served
    gid, roots = _queries(pools, 400, seed=9)
    want = {}
    for g, r in set(zip(gid.tolist(), roots.tolist())):
        h = host[g]
        want[(g, r)] = _u8(port.depths(h[0], h[1], r))

    alone = nwg.Server(graphs, slots=1, max_batch=1)
    alone_out = []
    for g, r in zip(gid.tolist(), roots.tolist()):
        out = np.full(graphs[g].n, 7, np.uint8)
        alone.wait(alone.submit(g, r, out))
        assert np.array_equal(out, want[(g, r)]), f"alone: graph {g} root {r}"
        alone_out.append(out)
    alone.close()

    mix = nwg.Server(graphs, slots=4, max_batch=256)
    burst = np.zeros(gid.size)  # everything at once: the largest batches
    poisson = np.cumsum(np.random.default_rng(3).exponential(1e6 / 20000.0, gid.size))
    for arrival in (burst, poisson):
        outs = [np.full(graphs[g].n, 7, np.uint8) for g in gid]
        lat, bs, st = mix.run_trace(gid, roots, arrival, outs)
        assert st.failed == 0 and st.queries == gid.size
        for i, (g, r) in enumerate(zip(gid.tolist(), roots.tolist())):
            assert np.array_equal(outs[i], alone_out[i]), f"query {i}: graph {g} root {r} differs in the mix"
        assert np.all(lat > 0) and np.all(bs >= 1)
        assert st.p50_ms <= st.p99_ms <= st.max_ms
        assert st.batches >= 1 and abs(st.mean_batch - gid.size / st.batches) < 1e-9
    # the burst was coalesced and ran on several slots at once
    lat, bs, st = mix.run_trace(gid, roots, burst)
    assert bs.max() > 1 and st.mean_batch > 1.0
    assert st.peak_in_flight >= 2
    mix.close()


def test_admission_budget_bounds_state(nwg, served):
    host, graphs, pools = served
    gid, roots = _queries(pools, 300, seed=12)
    big = max(g.n for g in graphs)
    probe = nwg.Server(graphs, slots=1, budget_bytes=1 << 34)
    slot_bytes = probe.run_trace(gid[:1], roots[:1], [0.0])[2].slot_bytes
    probe.close()
    # two slots plus room for only a handful of queries: most wait for budget
    budget = 2 * slot_bytes + 8 * int(2.5 * big) + 4096
    s = nwg.Server(graphs, slots=2, budget_bytes=budget)
    outs = [np.zeros(graphs[g].n, np.uint8) for g in gid]
    lat, bs, st = s.run_trace(gid, roots, np.zeros(gid.size), outs)
    assert st.slots == 2 and st.failed == 0
    assert st.peak_state_bytes <= st.budget_bytes
    # a pass holds queries of one graph: the budget, not max_batch, bounded it
    qbytes = np.array([2 * graphs[g].n + (4 * graphs[g].n + 7) // 8 for g in gid], np.int64)
    assert np.all(bs.astype(np.int64) * qbytes <= st.budget_bytes)
    assert bs.max() < 256
    ref = nwg.Server(graphs, slots=1)
    for i in range(0, gid.size, 37):
        out = np.zeros(graphs[gid[i]].n, np.uint8)
        ref.wait(ref.submit(int(gid[i]), int(roots[i]), out))
        assert np.array_equal(out, outs[i])
    ref.close()
    s.close()


def test_server_argument_errors(nwg, served):
    _, graphs, _ = served
    s = nwg.Server(graphs, slots=1)
    with pytest.raises(nwg.NwgError) as e:
        s.submit(len(graphs), 0)
    assert e.value.code == nwg.NWG_EINVAL
    with pytest.raises(nwg.NwgError):
        s.submit(0, graphs[0].n)
    with pytest.raises(nwg.NwgError):
        s.run_trace([0, 0], [1, 2], [5.0, 1.0])  # arrivals must not decrease
    s.close()
    with pytest.raises(nwg.NwgError) as e:
        nwg.Server(graphs, budget_bytes=1 << 20)  # no slot fits
    assert "budget" in str(e.value)


def path_plus_rmat(path_n):
    """A path of path_n vertices beside an RMAT-10 graph (ids from path_n on)."""
    u = np.arange(path_n - 1, dtype=np.uint64)
    roff, rcols = gg.rmat(10, 16, seed=3)
    ru = np.repeat(np.arange(roff.size - 1, dtype=np.uint64), (roff[1:] - roff[:-1]).astype(np.int64))
    pu = np.concatenate([u, ru + np.uint64(path_n)])
    pv = np.concatenate([u + np.uint64(1), rcols.astype(np.uint64) + np.uint64(path_n)])
    return gg.csr_from_pairs(pu, pv, path_n + roff.size - 1)


def test_deep_query_fails_alone_and_uint16_answers_it(nwg, port):
    """A path graph of 600 vertices (depths up to 599) served beside RMAT
    graphs and beside a graph holding both a 400-vertex path and an RMAT
    component.  uint8 answers: only the queries whose depths reach 255 fail
    (NWG_EOVERFLOW); every other query, including those coalesced with a
    deep one into the same pass, is answered exactly.  uint16 answers:
    every query is answered exactly and none fails."""
    pn = 600
    u = np.arange(pn - 1, dtype=np.uint64)
    host = [gg.csr_from_pairs(u, u + np.uint64(1), pn), gg.rmat(11, 16, seed=8), gg.rmat(12, 8, seed=9),
            path_plus_rmat(400)]
    graphs = [nwg.Graph.from_csr(*h) for h in host]
    queries = [(0, 0), (0, 300), (0, 599), (3, 0), (3, 200), (3, None), (3, 399), (0, 450), (1, None), (2, None),
               (3, None), (0, 100), (1, None), (3, 150)]
    rng = np.random.default_rng(3)
    qs = []
    for gi, r in queries:
        if r is None:  # a root with out-edges in the RMAT part
            base = 400 if gi == 3 else 0
            r = base + int(gg.roots(host[gi][0][base:] - host[gi][0][base], 1, seed=int(rng.integers(1, 1000)))[0])
        qs.append((gi, r))
    want = [port.depths(host[gi][0], host[gi][1], r) for gi, r in qs]
    deep = [int(np.where(w == NULL, 0, w).max()) >= 255 for w in want]
    assert any(deep) and not all(deep)

    # uint8 answers: submitted together, so each graph's queries share passes
    srv = nwg.Server(graphs, slots=1, max_batch=256)
    outs, tickets = [], []
    for gi, r in qs:
        outs.append(np.zeros(host[gi][0].size - 1, np.uint8))
        tickets.append(srv.submit(gi, r, outs[-1]))
    for i, t in enumerate(tickets):
        if deep[i]:
            with pytest.raises(nwg.NwgError) as e:
                srv.wait(t)
            assert e.value.code == nwg.NWG_EOVERFLOW
        else:
            srv.wait(t)
            assert np.array_equal(outs[i], _u8(want[i])), qs[i]
    srv.close()

    # uint16 answers, replayed as a trace: all exact, none failed
    srv = nwg.Server(graphs, slots=2, max_batch=256, depth_bytes=2)
    gid = np.array([q[0] for q in qs], np.uint32)
    roots = np.array([q[1] for q in qs], np.uint32)
    outs = [np.zeros(host[gi][0].size - 1, np.uint16) for gi, _ in qs]
    _, bs, st = srv.run_trace(gid, roots, np.zeros(len(qs)), outs)
    assert st.failed == 0 and bs.max() > 1
    for i in range(len(qs)):
        assert np.array_equal(outs[i], np.where(want[i] == NULL, 0xFFFF, want[i]).astype(np.uint16)), qs[i]
    srv.close()
    for g in graphs:
        g.release()
