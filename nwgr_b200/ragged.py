"""Ragged batches: many small graphs, (graph, root) traversals in one
persistent launch, parameters from an autotuner cached per graph-shape class.

    batch = RaggedBatch(graphs)            # packs the CSRs in HBM once
    tuner = Autotuner()                    # loads the JSON cache
    params = tuner.params_for(batch, items_by_graph)   # tunes unseen classes
    parents, offs, results, ms = batch.run(items_with_params, blocks_per_sm=params.blocks_per_sm)

Graph-shape class: (floor(log2 n), round(log2 average degree)) -- the two
quantities that set a traversal's level count, frontier sizes and hub
weight.  Per class the tuner chooses the top-down degree threshold
(warp_min: vertices at or above it are expanded in 256-edge chunks by a
whole warp) and the direction switch points alpha, beta (the reference's
defaults are 15 and 18; any choice gives the same depths, only the work
changes); per batch it chooses the resident blocks per SM of the persistent
launch.  Choices are timed on the device (CUDA events of the persistent
launch) over a sample of each class's items.

Cache: JSON at $NWG_AUTOTUNE_CACHE, else $XDG_CACHE_HOME/nwgr_b200/autotune.json
(~/.cache when XDG_CACHE_HOME is unset), keyed by GPU name and library
version.  Tuning results belong to the machine that measured them, so the
package ships none: a class the cache lacks is tuned on first use.
"""
from __future__ import annotations

import json
import math
import os
from dataclasses import dataclass

import numpy as np

from . import RaggedBatch, version



def default_cache_path() -> str:
    base = os.environ.get("XDG_CACHE_HOME") or os.path.join(os.path.expanduser("~"), ".cache")
    return os.path.join(base, "nwgr_b200", "autotune.json")


WARP_MIN = (32, 64, 128)
ALPHA = (15, 60)
BETA = (18, 36)
BLOCKS_PER_SM = (1, 2, 3)


def shape_class(n: int, m: int) -> str:
    d = max(1.0, m / max(1, n))
    return f"n{int(math.log2(max(1, n)))}_d{int(round(math.log2(d)))}"


@dataclass
class ClassParams:
    warp_min: int = 32
    alpha: int = 15
    beta: int = 18


def _device_key() -> str:
    try:
        import torch

        name = torch.cuda.get_device_name(0)
    except Exception:
        name = "unknown"
    return f"{name}|{version()}"


class Autotuner:
    def __init__(self, path: str | None = None):
        self.path = path or os.environ.get("NWG_AUTOTUNE_CACHE") or default_cache_path()
        self.key = _device_key()
        self.cache = {}
        try:
            with open(self.path) as f:
                self.cache = json.load(f)
        except (OSError, ValueError):
            self.cache = {}
        self.entry = self.cache.setdefault(self.key, {"classes": {}, "blocks_per_sm": None})

    def save(self) -> None:
        try:
            os.makedirs(os.path.dirname(os.path.abspath(self.path)), exist_ok=True)
            tmp = self.path + ".tmp"
            with open(tmp, "w") as f:
                json.dump(self.cache, f, indent=1, sort_keys=True)
            os.replace(tmp, self.path)
        except OSError:
            pass

    def class_params(self, cls: str) -> ClassParams | None:
        p = self.entry["classes"].get(cls)
        return ClassParams(**p) if p else None

    def _time(self, batch: RaggedBatch, items, bps: int, reps: int = 2) -> float:
        best = float("inf")
        for _ in range(reps):
            _, _, _, ms = batch.run(items, blocks_per_sm=bps)
            best = min(best, ms)
        return best

    def tune(self, batch: RaggedBatch, graph_mn, roots_by_graph, sample: int = 12, force: bool = False):
        """Tunes every class present in the batch that the cache lacks.
        graph_mn: per graph (n, m); roots_by_graph: per graph a list of roots.
        Returns {class: ClassParams} and the batch's blocks_per_sm."""
        classes = {}
        for g, (n, m) in enumerate(graph_mn):
            classes.setdefault(shape_class(n, m), []).append(g)
        out = {}
        for cls, gs in sorted(classes.items()):
            cached = self.class_params(cls)
            if cached and not force:
                out[cls] = cached
                continue
            pick = gs[:: max(1, len(gs) // sample)][:sample]
            base = [(g, int(r)) for g in pick for r in roots_by_graph[g]]
            best, best_t = ClassParams(), float("inf")
            for wm in WARP_MIN:
                for a in ALPHA:
                    for b in BETA:
                        t = self._time(batch, [(g, r, a, b, wm) for g, r in base], 2)
                        if t < best_t:
                            best, best_t = ClassParams(wm, a, b), t
            out[cls] = best
            self.entry["classes"][cls] = best.__dict__
        bps = self.entry.get("blocks_per_sm")
        if bps is None or force:
            items = self.items(graph_mn, roots_by_graph, out)
            times = {b: self._time(batch, items, b, 2) for b in BLOCKS_PER_SM}
            bps = min(times, key=times.get)
            self.entry["blocks_per_sm"] = bps
        self.save()
        return out, bps

    @staticmethod
    def items(graph_mn, roots_by_graph, params):
        items = []
        for g, (n, m) in enumerate(graph_mn):
            p = params.get(shape_class(n, m), ClassParams())
            items += [(g, int(r), p.alpha, p.beta, p.warp_min) for r in roots_by_graph[g]]
        return items


def ragged_workload(nwg, num_graphs: int = 1000, roots_per_graph: int = 4, seed: int = 1, lo: int = 10, hi: int = 18):
    """The ragged benchmark set: vertex counts log-uniform on 2^lo..2^hi,
    half RMAT (edge factor uniform 8..32, A/B/C/D .57/.19/.19/.05) and half
    2D grids with 1% random shortcuts, generated on the device from seeds;
    `roots_per_graph` seeded roots each (out-degree > 0).  Returns the host
    CSRs, (n, m) per graph, roots per graph and the kind of each graph."""
    rng = np.random.default_rng(seed)
    graphs, mn, roots, kinds = [], [], [], []
    for i in range(num_graphs):
        logn = rng.uniform(lo, hi)
        if i % 2 == 0:
            scale = int(round(logn))
            ef = int(rng.integers(8, 33))
            g = nwg.Graph.rmat(scale, ef, seed=seed * 100003 + i)
            kinds.append("rmat")
        else:
            n = int(2 ** logn)
            w = max(2, int(round(math.sqrt(n))))
            h = max(2, n // w)
            g = nwg.Graph.grid(w, h, 1, seed=seed * 100003 + i)
            kinds.append("grid")
        off, cols = g.csr()
        roots.append(g.roots(roots_per_graph, seed=seed * 7919 + i))
        g.release()
        graphs.append((off, cols))
        mn.append((off.size - 1, cols.size))
    return graphs, mn, roots, kinds
