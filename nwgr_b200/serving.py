"""Serving workload: resident graphs from the ragged-batch distribution and
an open-loop Poisson stream of (graph, root) queries with Zipf popularity.

    graphs, pools = serving_graphs(nwg, 200)        # registered, resident in HBM
    server = nwg.Server(graphs, slots=8, budget_bytes=16 << 30)
    g, r, t = query_trace(pools, rate_qps=50_000, count=100_000, zipf_s=1.1)
    latency_ms, batch, stats = server.run_trace(g, r, t)

Graphs: vertex counts log-uniform on 2^10..2^18, half RMAT (edge factor
uniform 8..32, A/B/C/D .57/.19/.19/.05, permuted, symmetrized, deduplicated)
and half 2D grids with 1% random shortcuts -- the ragged-batch rules
(nwgr_b200.ragged.ragged_workload), generated on the device from seeds and
left registered.  Popularity: graph ranks are a seeded permutation, query
weights proportional to rank^-s.  Roots: uniform over a seeded pool of
vertices with out-degree > 0 per graph.
"""
from __future__ import annotations

import math

import numpy as np


def serving_graphs(nwg, num_graphs: int = 200, seed: int = 11, lo: int = 10, hi: int = 18, pool: int = 256):
    """Registered graphs (resident) and a root pool (uint32 array) per graph."""
    rng = np.random.default_rng(seed)
    graphs, pools = [], []
    for i in range(num_graphs):
        logn = rng.uniform(lo, hi)
        if i % 2 == 0:
            g = nwg.Graph.rmat(int(round(logn)), int(rng.integers(8, 33)), seed=seed * 100003 + i)
        else:
            n = int(2 ** logn)
            w = max(2, int(round(math.sqrt(n))))
            g = nwg.Graph.grid(w, max(2, n // w), 1, seed=seed * 100003 + i)
        graphs.append(g)
        pools.append(np.asarray(g.roots(pool, seed=seed * 7919 + i), np.uint32))
    return graphs, pools


def zipf_weights(num: int, s: float, seed: int) -> np.ndarray:
    """Query probability per graph: rank^-s over a seeded rank permutation."""
    ranks = np.random.default_rng(seed).permutation(num) + 1
    w = ranks.astype(np.float64) ** -s
    return w / w.sum()


def query_trace(pools, rate_qps: float, count: int, zipf_s: float = 1.1, seed: int = 5):
    """(graph ids, roots, arrival microseconds) of a Poisson stream."""
    rng = np.random.default_rng(seed)
    arrival = np.cumsum(rng.exponential(1e6 / rate_qps, count))
    arrival -= arrival[0]
    p = zipf_weights(len(pools), zipf_s, seed + 1)
    gid = rng.choice(len(pools), size=count, p=p).astype(np.uint32)
    pick = rng.integers(0, 1 << 62, count)
    roots = np.fromiter((pools[g][k % pools[g].size] for g, k in zip(gid, pick)), np.uint32, count)
    return gid, roots, arrival
