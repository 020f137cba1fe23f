"""TEST INFRASTRUCTURE ONLY (the oracle for the graph generators).

numpy restatement of the seeded synthetic graph generators that the CUDA
library implements in ``nwgr_b200/csrc/nwg_gen.cu``.  Tests build small graphs
here and check the device generator against them bit for bit.

NWGraph has no RMAT/uniform/grid generator (its only generator,
include/nwgraph/generators/configuration_model.hpp, does not compile), so the
definitions below are this project's; the CSR clean-up follows the
reference's own edge-list pipeline: symmetrize (both directions of every
undirected pair, as io/mmio.hpp:96-100 does for symmetric files), drop
self-loops (build.hpp:427-444 remove_self_loops), sort and deduplicate
(build.hpp:58-70 lexical_sort_by, build.hpp:344-355 uniq), then fill a CSR
with rows sorted by neighbour id (build.hpp:210-266 fill_directed).

Randomness is counter-based so every edge can be generated independently
(and identically) on the host and on the device:
  splitmix64(x)             Steele, Lea and Flood's SplitMix64 finaliser
  draw(seed, stream, idx) = splitmix64(splitmix64(seed) ^ (stream << 56) ^ idx)
  lemire(h, n)            = ((h >> 32) * n) >> 32      (uniform on [0, n), n < 2^32)
"""
from __future__ import annotations

import numpy as np

M64 = np.uint64(0xFFFFFFFFFFFFFFFF)
GOLDEN = np.uint64(0x9E3779B97F4A7C15)
MIX1 = np.uint64(0xBF58476D1CE4E5B9)
MIX2 = np.uint64(0x94D049BB133111EB)

STREAM_RMAT = 1
STREAM_PERM = 2
STREAM_UNIFORM = 3
STREAM_GRID = 4
STREAM_ROOTS = 5

DEFAULT_ROOT_SEED = 27491095  # bench/bfs.cpp:32 default --seed


def splitmix64(x):
    x = np.asarray(x, dtype=np.uint64)
    with np.errstate(over="ignore"):
        z = x + GOLDEN
        z = (z ^ (z >> np.uint64(30))) * MIX1
        z = (z ^ (z >> np.uint64(27))) * MIX2
    return z ^ (z >> np.uint64(31))


def seed_key(seed: int) -> np.uint64:
    return np.uint64(int(splitmix64(np.uint64(seed & 0xFFFFFFFFFFFFFFFF))))


def draw(seed: int, stream: int, idx):
    k = seed_key(seed) ^ np.uint64(stream << 56)
    return splitmix64(np.asarray(idx, dtype=np.uint64) ^ k)


def lemire(h, n: int):
    h = np.asarray(h, dtype=np.uint64)
    return ((h >> np.uint64(32)) * np.uint64(n)) >> np.uint64(32)


def rmat_thresholds(a: float, b: float, c: float):
    """32-bit integer thresholds of the cumulative quadrant probabilities.
    The device generator receives these integers, never the floats."""
    ta = int(a * 4294967296.0)
    tab = int((a + b) * 4294967296.0)
    tabc = int((a + b + c) * 4294967296.0)
    return ta, tab, tabc


def permute(x, scale: int, seed: int):
    """Bijection on [0, 2^scale): three rounds of (x*K + C) mod 2^s followed
    by x ^= x >> ceil(s/2)."""
    x = np.asarray(x, dtype=np.uint64)
    mask = np.uint64((1 << scale) - 1)
    sh = np.uint64((scale + 1) >> 1)
    for r in range(3):
        k = np.uint64(int(draw(seed, STREAM_PERM, 2 * r)) | 1)
        c = draw(seed, STREAM_PERM, 2 * r + 1)
        with np.errstate(over="ignore"):
            x = (x * k + c) & mask
        x = x ^ (x >> sh)
    return x


def rmat_edges(scale: int, edge_factor: int, seed: int, a=0.57, b=0.19, c=0.19, chunk=1 << 20):
    """Undirected RMAT endpoint pairs (before permutation), edge_factor * 2^scale of them."""
    n_edges = edge_factor << scale
    ta, tab, tabc = (np.uint64(t) for t in rmat_thresholds(a, b, c))
    words = (scale + 1) >> 1
    us, vs = [], []
    for e0 in range(0, n_edges, chunk):
        e = np.arange(e0, min(n_edges, e0 + chunk), dtype=np.uint64)
        u = np.zeros(e.shape, np.uint64)
        v = np.zeros(e.shape, np.uint64)
        for lvl in range(scale):
            w = draw(seed, STREAM_RMAT, e * np.uint64(words) + np.uint64(lvl >> 1))
            t = (w >> np.uint64(32)) if (lvl & 1) else (w & np.uint64(0xFFFFFFFF))
            ub = (t >= tab).astype(np.uint64)  # quadrants C, D set the source bit
            vb = (((t >= ta) & (t < tab)) | (t >= tabc)).astype(np.uint64)  # quadrants B, D
            u = (u << np.uint64(1)) | ub
            v = (v << np.uint64(1)) | vb
        us.append(u)
        vs.append(v)
    return np.concatenate(us), np.concatenate(vs)


def csr_from_pairs(u, v, n: int):
    """Symmetrize, drop self-loops, sort, dedup -> (offsets uint64[n+1], cols uint32[m])."""
    u = np.asarray(u, dtype=np.uint64)
    v = np.asarray(v, dtype=np.uint64)
    keep = u != v
    u, v = u[keep], v[keep]
    keys = np.concatenate([(u << np.uint64(32)) | v, (v << np.uint64(32)) | u])
    keys = np.unique(keys)  # sorted, deduplicated
    src = (keys >> np.uint64(32)).astype(np.int64)
    cols = (keys & np.uint64(0xFFFFFFFF)).astype(np.uint32)
    counts = np.bincount(src, minlength=n).astype(np.uint64)
    off = np.zeros(n + 1, dtype=np.uint64)
    np.cumsum(counts, out=off[1:])
    return off, cols


def rmat(scale: int, edge_factor: int = 16, seed: int = 1, a=0.57, b=0.19, c=0.19):
    u, v = rmat_edges(scale, edge_factor, seed, a, b, c)
    u = permute(u, scale, seed)
    v = permute(v, scale, seed)
    return csr_from_pairs(u, v, 1 << scale)


def uniform(n: int, avg_degree: int = 32, seed: int = 1):
    """n vertices, n*avg_degree/2 uniform random undirected pairs."""
    pairs = (n * avg_degree) // 2
    idx = np.arange(pairs, dtype=np.uint64)
    u = lemire(draw(seed, STREAM_UNIFORM, idx * np.uint64(2)), n)
    v = lemire(draw(seed, STREAM_UNIFORM, idx * np.uint64(2) + np.uint64(1)), n)
    return csr_from_pairs(u, v, n)


def grid(width: int, height: int, shortcut_pct: int = 1, seed: int = 1):
    """4-neighbour width x height grid (id = y*width + x) plus
    shortcut_pct% of the grid's edge count as uniform random long-range pairs."""
    n = width * height
    ids = np.arange(n, dtype=np.uint64).reshape(height, width)
    ru = ids[:, :-1].ravel()
    rv = ids[:, 1:].ravel()
    du = ids[:-1, :].ravel()
    dv = ids[1:, :].ravel()
    g_edges = ru.size + du.size
    s = (g_edges * shortcut_pct) // 100
    idx = np.arange(s, dtype=np.uint64)
    su = lemire(draw(seed, STREAM_GRID, idx * np.uint64(2)), n)
    sv = lemire(draw(seed, STREAM_GRID, idx * np.uint64(2) + np.uint64(1)), n)
    return csr_from_pairs(np.concatenate([ru, du, su]), np.concatenate([rv, dv, sv]), n)


def roots(off, count: int = 64, seed: int = DEFAULT_ROOT_SEED):
    """`count` roots uniform on [0, n) with out-degree > 0 (duplicates allowed,
    as in bench/common.hpp:123-136, but without its inclusive-n upper bound)."""
    off = np.asarray(off, dtype=np.uint64)
    n = off.size - 1
    deg = off[1:] - off[:-1]
    if count and not np.any(deg):
        raise ValueError("graph has no vertex with out-degree > 0")
    out = []
    k = 0
    while len(out) < count:
        batch = lemire(draw(seed, STREAM_ROOTS, np.arange(k, k + 1024, dtype=np.uint64)), n)
        for v in batch.tolist():
            if deg[v] > 0:
                out.append(v)
                if len(out) == count:
                    break
        k += 1024
    return np.asarray(out, dtype=np.uint32)


def transpose(off, cols, n: int):
    """In-edge CSR of a directed CSR (rows sorted)."""
    off = np.asarray(off, dtype=np.uint64)
    src = np.repeat(np.arange(n, dtype=np.uint64), (off[1:] - off[:-1]).astype(np.int64))
    keys = (cols.astype(np.uint64) << np.uint64(32)) | src
    keys.sort()
    t_src = (keys >> np.uint64(32)).astype(np.int64)
    t_cols = (keys & np.uint64(0xFFFFFFFF)).astype(np.uint32)
    counts = np.bincount(t_src, minlength=n).astype(np.uint64)
    t_off = np.zeros(n + 1, dtype=np.uint64)
    np.cumsum(counts, out=t_off[1:])
    return t_off, t_cols


def directed_csr(u, v, n: int):
    """Directed CSR (no symmetrization): drop self-loops, sort, dedup."""
    u = np.asarray(u, dtype=np.uint64)
    v = np.asarray(v, dtype=np.uint64)
    keep = u != v
    keys = np.unique((u[keep] << np.uint64(32)) | v[keep])
    src = (keys >> np.uint64(32)).astype(np.int64)
    cols = (keys & np.uint64(0xFFFFFFFF)).astype(np.uint32)
    counts = np.bincount(src, minlength=n).astype(np.uint64)
    off = np.zeros(n + 1, dtype=np.uint64)
    np.cumsum(counts, out=off[1:])
    return off, cols
