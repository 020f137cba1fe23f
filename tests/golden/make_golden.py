"""Generates tests/golden/fixtures.npz from the reference itself.

Run where the NWGraph sources exist (they are read, never copied):

    python tests/golden/make_golden.py [--reference PATH]   (default: $NWG_REFERENCE_ROOT, else a
    checkout named "reference" beside this repository)

For every MatrixMarket fixture in the reference's data/ directory the script
builds the edge set exactly as read_mm does (io/mmio.hpp:86-103,172-208:
1-based ids, symmetric files contribute both directions of each
off-diagonal entry, general files each entry as given, self-loops and
duplicates kept), stores it as an out-CSR plus its transpose (the in-CSR),
and records, for a few roots, what the reference's own nw::graph::bfs
(algorithms/bfs.hpp:160-311, compiled unmodified by oracle/ref_dobfs.cpp)
returns: the depths implied by its parents and whether its BFSVerifier
accepts them.  Two seeded RMAT graphs (scale 10 and 11, project generator)
are added the same way.  It also stores the direction trace of the C
restatement (oracle/dobfs_port.c) for each (graph, root).

The output pins the oracle: tests check that the C restatement reproduces
these depths on any machine, without the reference present.
"""
from __future__ import annotations

import argparse
import glob
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import graphgen as gg  # noqa: E402
from oracle import oracle as O  # noqa: E402


def csr_keep_all(u, v, n):
    """CSR with rows sorted by target, duplicates and self-loops kept."""
    order = np.lexsort((v, u))
    u, v = u[order], v[order]
    counts = np.bincount(u.astype(np.int64), minlength=n).astype(np.uint64)
    off = np.zeros(n + 1, np.uint64)
    np.cumsum(counts, out=off[1:])
    return off, v.astype(np.uint32)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=None, help="NWGraph source tree")
    ap.add_argument("--out", default=os.path.join(os.path.dirname(os.path.abspath(__file__)), "fixtures.npz"))
    args = ap.parse_args()
    args.reference = args.reference or O.REFERENCE_ROOT
    os.environ["NWG_REFERENCE_INCLUDE"] = os.path.join(args.reference, "include")
    O.REFERENCE_INCLUDE = os.environ["NWG_REFERENCE_INCLUDE"]
    ref = O.Reference()
    ref.set_threads(1)
    port = O.Port()

    graphs = []
    for path in sorted(glob.glob(os.path.join(args.reference, "data", "*.mtx"))):
        n, u, v = O.read_mtx(path)
        off, cols = csr_keep_all(u, v, n)
        in_off, in_cols = csr_keep_all(v, u, n)
        symmetric = np.array_equal(off, in_off) and np.array_equal(cols, in_cols)
        graphs.append((os.path.basename(path)[:-4], off, cols, None if symmetric else in_off,
                       None if symmetric else in_cols))
    for scale in (10, 11):
        off, cols = gg.rmat(scale, 16, seed=scale)
        graphs.append((f"rmat{scale}", off, cols, None, None))

    out = {}
    names = []
    for name, off, cols, in_off, in_cols in graphs:
        n = off.size - 1
        deg = off[1:] - off[:-1]
        roots = [r for r in (0, 1, 5) if r < n]
        if np.any(deg):
            roots += gg.roots(off, 3, seed=7).tolist()
        roots = sorted(set(roots))
        g = ref.graph(off, cols, in_off, in_cols)
        depth_rows, ok_rows, dirs, founds = [], [], [], []
        for r in roots:
            parents, _ = g.dobfs(r, 32, 15, 18)
            ok = g.verify(r, parents)
            d = port.depths_from_parents(parents, r)
            if d is None:
                raise SystemExit(f"{name} root {r}: reference parents are not a tree")
            serial = port.depths(off, cols, r)
            if not np.array_equal(d, serial):
                raise SystemExit(f"{name} root {r}: reference depths differ from a serial BFS")
            _, tr = port.dobfs(off, cols, r, in_off, in_cols)
            depth_rows.append(d)
            ok_rows.append(ok)
            dirs.append(tr["dir"].astype(np.uint8))
            founds.append(tr["found"].astype(np.uint64))
        g.close()
        names.append(name)
        out[f"{name}/off"] = off
        out[f"{name}/cols"] = cols
        if in_off is not None:
            out[f"{name}/in_off"] = in_off
            out[f"{name}/in_cols"] = in_cols
        out[f"{name}/roots"] = np.asarray(roots, np.uint32)
        out[f"{name}/depths"] = np.stack(depth_rows).astype(np.uint32)
        out[f"{name}/ref_verifier_ok"] = np.asarray(ok_rows, bool)
        for i, (dd, ff) in enumerate(zip(dirs, founds)):
            out[f"{name}/trace_dir/{i}"] = dd
            out[f"{name}/trace_found/{i}"] = ff
        print(f"{name:16s} n={n:6d} m={cols.size:7d} sym={in_off is None} roots={roots} verifier={ok_rows}")
    out["names"] = np.asarray(names)
    np.savez_compressed(args.out, **out)
    print("wrote", args.out, os.path.getsize(args.out), "bytes")


if __name__ == "__main__":
    main()
