"""Throughput of the B200 direction-optimizing BFS (one JSON line on stdout).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--graph rmat24|uniform24|grid4096|rmatS]
                    [--roots 64] [--impl nwg|reference]

Workload (default): RMAT scale 24, edge factor 16, A/B/C/D = .57/.19/.19/.05,
ids permuted, symmetrized, deduplicated, self-loops removed (uint32 columns,
uint64 offsets), generated on the device from a fixed seed; 64 roots drawn
uniformly among vertices with out-degree > 0 (seed 27491095).  One "step" is
the 64 single-source traversals.

Metric: GTEPS = (E_r / 2) / t per root, E_r = sum of out-degrees of the
vertices the root reaches (directed CSR entries, Graph500 convention),
harmonic mean over the roots; t = device time of the whole traversal
(initialisation of parents and bitmaps included, like the reference's bfs()
call) from CUDA events on the launching stream.  The L2 is flushed (256 MB
write) before every traversal, outside the events.

e2e: the same metric through the C ABI with host buffers: each step
registers the graph from pinned host CSR arrays (the upload), runs
nwg_bfs_roots over the 64 roots (two traversals in flight, each root's
parents copied to its own row of pinned host memory), and releases the
graph; per-root time = step time / 64.  The first --warmup steps are
untimed, like the device leg's.  per_call_gteps is the same with one
synchronous nwg_bfs call per root.

roofline: algorithmic bytes of a traversal B_r = 4 E_r + 8 n_r + 4 N
(every adjacency entry of the component, one offset per reached vertex,
the parent array) over its device time, against the measured HBM copy
bandwidth.

cpu_baseline / --impl reference: the reference's own nw::graph::bfs
(include/nwgraph/algorithms/bfs.hpp, compiled unmodified against the
project's TBB-compatible thread pool, oracle/_ref) on this host's cores,
timed like bench/common.hpp's time_op, on a bounded sample of the roots.

Further sections of the same JSON line (each skippable with --no-<name>):
  other        the other graphs of the single-source workload (of RMAT-24,
               uniform 2^24 with average degree 32, the 4096 x 4096 grid with
               1% shortcuts, those not named by --graph): GTEPS over the same 64 roots
               timed like the main line, roofline fraction, and the
               reference's bfs on the host for one root
  verifier     device BFSVerifier time per root, and the reference's
               verifier on the host for the first root
  batched      multi-source BFS on RMAT-22 with 64/256/1024 roots against 64
               back-to-back single-source traversals
  ragged       1000 small graphs x 4 roots in one persistent launch against
               one call per item
  serving      200 resident graphs, Poisson query rates 1k-200k/s, Zipf(1.1)
               popularity: queries/s and p50/p99 latency
  betweenness  brandes_bc over 64 sources on RMAT-22, beside the reference's
               on a 4-source sample
Profiling modes (one run inside the NVTX range nwg_profile, for ncu):
--profile-one (single-source, host-stepped), --profile-trav (single-source,
the persistent kernel), --profile-msbfs, --profile-bc.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

ROOT_SEED = 27491095
GRAPH_SEED = 1
PEAKS_FILE = os.path.join(ROOT, "MEASURED_PEAKS.json")
FALLBACK_HBM_GBS = 6650.0

# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) of one traversal
# (one launch of the persistent kernel k_trav) captured with ncu on a smaller
# graph of the same kind, and that graph's directed entries; scaled to a
# workload by its entries (profiles/k_trav_traffic_rmat22_uniform22.md).
TRAFFIC_CAPTURES = {"rmat": (179.8e6, 128306546), "uniform": (511.6e6, 134217204)}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--graph", default="rmat24")
    ap.add_argument("--roots", type=int, default=64)
    ap.add_argument("--impl", default="nwg", choices=["nwg", "reference"])
    ap.add_argument("--cpu-sample-roots", type=int, default=64,
                    help="roots of the cpu_baseline leg (each timed once)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-batched", action="store_true")
    ap.add_argument("--no-ragged", action="store_true")
    ap.add_argument("--no-serving", action="store_true")
    ap.add_argument("--no-verify", action="store_true")
    ap.add_argument("--no-bc", action="store_true")
    ap.add_argument("--no-other", action="store_true", help="skip the other graphs of the single-source workload")
    ap.add_argument("--profile-msbfs", action="store_true",
                    help="one multi-source pass on RMAT-22 (--ms-sources roots), levels driven from the host, in "
                         "NVTX range nwg_profile (for ncu)")
    ap.add_argument("--ms-sources", type=int, default=64, help="sources of the --profile-msbfs pass (at most 256)")
    ap.add_argument("--profile-bc", action="store_true",
                    help="betweenness from one source on RMAT-22 in NVTX range nwg_profile (for ncu)")
    ap.add_argument("--serve-slots", type=int, default=16)
    ap.add_argument("--profile-one", action="store_true",
                    help="after warm-up, run one host-stepped traversal (one kernel per step) inside an NVTX range "
                         "'nwg_profile' and exit (for ncu)")
    ap.add_argument("--trace-steps", type=int, default=0, metavar="R",
                    help="print the device-timed step trace (direction, frontier, discoveries, microseconds) of "
                         "the first R roots' traversals (L2 flushed before each) and exit")
    ap.add_argument("--profile-trav", action="store_true",
                    help="after warm-up, run one traversal as the persistent kernel k_trav inside an NVTX range "
                         "'nwg_profile' and exit (for ncu)")
    return ap.parse_args()


def graph_spec(name: str):
    if name == "rmat24":
        return {"kind": "rmat", "scale": 24, "edge_factor": 16}
    if name.startswith("rmat"):
        return {"kind": "rmat", "scale": int(name[4:]), "edge_factor": 16}
    if name == "uniform24":
        return {"kind": "uniform", "n": 1 << 24, "avg_degree": 32}
    if name.startswith("uniform"):
        return {"kind": "uniform", "n": 1 << int(name[7:]), "avg_degree": 32}
    if name == "grid4096":
        return {"kind": "grid", "width": 4096, "height": 4096, "shortcut_pct": 1}
    raise SystemExit(f"unknown graph {name}")


def make_graph(nwg, spec):
    if spec["kind"] == "rmat":
        return nwg.Graph.rmat(spec["scale"], spec["edge_factor"], seed=GRAPH_SEED)
    if spec["kind"] == "uniform":
        return nwg.Graph.uniform(spec["n"], spec["avg_degree"], seed=GRAPH_SEED)
    return nwg.Graph.grid(spec["width"], spec["height"], spec["shortcut_pct"], seed=GRAPH_SEED)


def workload_name(spec):
    if spec["kind"] == "rmat":
        return f"RMAT-{spec['scale']} ef{spec['edge_factor']} .57/.19/.19/.05 permuted symmetrized dedup"
    if spec["kind"] == "uniform":
        return f"uniform n={spec['n']} avg degree {spec['avg_degree']}"
    return f"grid {spec['width']}x{spec['height']} 4-neighbour + {spec['shortcut_pct']}% shortcuts"


def hmean(x):
    x = np.asarray(x, dtype=np.float64)
    return float(x.size / np.sum(1.0 / x))


def peaks():
    try:
        with open(PEAKS_FILE) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return FALLBACK_HBM_GBS, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.rows = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([c.strip() for c in line.split(",")])

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.3)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = [r for r in self.rows if len(r) >= 9]
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def max_over_ranks(values, dist=None, device="cpu"):
    """Element-wise maximum of a per-rank float64 vector over all ranks (the
    slowest rank's time per root); identity without a process group."""
    if dist is None:
        return np.asarray(values, np.float64)
    import torch

    t = torch.tensor(np.asarray(values, np.float64), device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return t.cpu().numpy()


def replica_gteps(e_r, per_root_ms, world):
    """Whole-job throughput of `world` replicas that each traverse the same
    roots: world x harmonic mean over roots of (E_r / 2) / t_r, t_r the
    slowest rank's time for root r."""
    gteps = (np.asarray(e_r, np.float64) / 2.0) / (np.asarray(per_root_ms, np.float64) * 1e-3) / 1e9
    return world * hmean(gteps), gteps


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def metric_name(args, n_roots):
    """The metric string both arms print (the reference arm's and this library's)."""
    return f"BFS GTEPS (harmonic mean over {n_roots} roots) @ {args.graph}"


def host_graph(spec):
    """The workload's CSR built on the host cores by the oracle's generator
    (oracle/graphgen_host.c): the same graph, bit for bit, as the device
    generator, without loading this library."""
    from oracle.oracle import HostGen

    h = HostGen()
    if spec["kind"] == "rmat":
        return h.rmat(spec["scale"], spec["edge_factor"], seed=GRAPH_SEED)
    if spec["kind"] == "uniform":
        return h.uniform(spec["n"], spec["avg_degree"], seed=GRAPH_SEED)
    return h.grid(spec["width"], spec["height"], spec["shortcut_pct"], seed=GRAPH_SEED)


def reference_roots_timed(rg, deg, roots, order):
    """Times the reference's bfs (bfs.hpp:160-311, oracle/_ref) once per
    entry of `order` (indices into roots), wall clock around each call like
    NWGraph's time_op (bench/common.hpp:155-167).  Returns per-root mean
    seconds and E_r / 2 for every root timed."""
    secs = {}
    edges = {}
    for i in order:
        parents, t = rg.dobfs(int(roots[i]), 32, 15, 18)
        secs.setdefault(i, []).append(t)
        if i not in edges:
            edges[i] = float(deg[parents != 0xFFFFFFFF].sum()) / 2.0
    idx = sorted(secs)
    return np.asarray([np.mean(secs[i]) for i in idx]), np.asarray([edges[i] for i in idx])


def run_reference_arm(args, spec, world, rank):
    """The reference's own CPU bfs on this host (rank 0 only).  The graph is
    built by the oracle's host generator, so this process loads no library
    of this repository's product; every one of the workload's roots is timed
    at least once inside the timed steps."""
    if rank != 0:
        return
    from oracle import graphgen as gg
    from oracle.oracle import Reference

    off, cols = host_graph(spec)
    roots = gg.roots(off, args.roots, seed=ROOT_SEED)
    deg = off[1:] - off[:-1]
    ref = Reference()
    rg = ref.graph(off, cols)
    threads = ref.threads()
    for step in range(args.warmup):  # one untimed traversal per warm-up step
        rg.dobfs(int(roots[step % roots.size]), 32, 15, 18, want_parents=False)
    per_step = max(1, -(-roots.size // max(1, args.steps)))  # the timed steps cover every root
    order = [k % roots.size for k in range(per_step * args.steps)]
    t0 = time.perf_counter()
    secs, edges = reference_roots_timed(rg, deg, roots, order)
    wall = time.perf_counter() - t0
    rg.close()
    v = hmean(edges / secs / 1e9)
    sample = (f"{per_step} roots per step, {len(order)} timed calls covering all {secs.size} of the "
              f"{roots.size} roots (per-root mean time), reference bfs.hpp on the project's TBB-compatible "
              f"pool, {threads} threads; graph from the oracle's host generator")
    line = {
        "impl": "reference", "metric": metric_name(args, roots.size), "value": v,
        "unit": "GTEPS", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * wall / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "uint32", "data": "synthetic (seeded host generator)",
        "config": {"workload": workload_name(spec), "n": int(off.size - 1), "m_directed": int(cols.size),
                   "roots": int(roots.size), "alpha": 15, "beta": 18, "timing": "host wall clock per call"},
        "cpu_baseline": {"value": v, "unit": "GTEPS", "cores": threads, "kind": "reference",
                         "ms_per_root_median": 1e3 * float(np.median(secs)),
                         "glibc_tunables": os.environ.get("GLIBC_TUNABLES", ""), "sample": sample},
        "e2e": {"value": v, "unit": "GTEPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def bench_batched(nwg, torch, scale=22, ks=(64, 256, 1024), reps=3):
    """Batched multi-source BFS (64 sources per 64-bit word) against 64
    back-to-back single-source traversals of the same roots, on RMAT-`scale`.
    Aggregate GTEPS = sum over roots of E_r / 2, over the device time of the
    whole batch (CUDA events); depths are checked equal on the host for a
    sample of roots."""
    g = nwg.Graph.rmat(scale, 16, seed=GRAPH_SEED)
    kmax = max(ks)
    roots = g.roots(kmax, seed=ROOT_SEED)
    stream = torch.cuda.Stream()
    par = torch.empty(g.n, dtype=torch.int32, device="cuda")
    ws = g.workspace()
    e_r = np.zeros(kmax)
    for i, r in enumerate(roots):  # E_r of every root (untimed)
        nwg.bfs_device(g, int(r), par)
        e_r[i] = g.component_edges(par)[0]
    # 64 back-to-back single-source traversals
    plain = []
    for rep in range(reps + 1):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stream):
            a.record(stream)
            for r in roots[:64]:
                ws.bfs_async(int(r), par, stream.cuda_stream)
            b.record(stream)
        stream.synchronize()
        if rep:
            plain.append(a.elapsed_time(b))
    plain_ms = float(np.median(plain))
    plain_gteps = float(e_r[:64].sum() / 2.0 / (plain_ms * 1e-3) / 1e9)
    ms = nwg.MsWorkspace(g)
    out = {"graph": f"RMAT-{scale} ef16", "plain64_ms": plain_ms, "plain64_gteps": plain_gteps, "msbfs": {}}
    for k in ks:
        depths = torch.empty((k, g.n), dtype=torch.uint8, device="cuda")
        times = []
        for rep in range(reps + 1):
            st = ms.run(roots[:k], depths, stream=stream.cuda_stream)
            if rep:
                times.append(st.device_ms)
        t = float(np.median(times))
        gteps = float(e_r[:k].sum() / 2.0 / (t * 1e-3) / 1e9)
        out["msbfs"][str(k)] = {"ms": t, "gteps": gteps, "vs_plain64": gteps / plain_gteps, "passes": st.passes,
                                "push_levels": st.push_levels, "pull_levels": st.pull_levels}
        if k == min(ks):  # depths equal to the single-source traversals for a sample of roots
            d = depths.cpu().numpy()
            ok = True
            for i in (0, k // 2, k - 1):
                nwg.bfs_device(g, int(roots[i]), par)
                dd = nwg.depths_from_parents(par.cpu().numpy().view(np.uint32), int(roots[i]))
                ok &= bool(np.array_equal(np.where(dd == 0xFFFFFFFF, 255, dd).astype(np.uint8), d[i]))
            out["depths_match_single_source_sample"] = ok
        del depths
    ms.close()
    ws.close()
    g.release()
    return out


def bench_ragged(nwg, torch, num_graphs=1000, reps=3):
    """Ragged batch: num_graphs graphs (n log-uniform on 2^10..2^18, half
    RMAT with edge factor 8..32, half 2D grids with 1% shortcuts), 4 roots
    each, all (graph, root) items in one persistent launch replayed as a CUDA
    graph, parameters from the autotuner (cached per graph-shape class).
    Compared with the same items as one nwg_bfs call each on separately
    registered graphs (device time of the calls summed)."""
    from nwgr_b200.ragged import Autotuner, ragged_workload

    t0 = time.perf_counter()
    graphs, mn, roots, kinds = ragged_workload(nwg, num_graphs)
    gen_s = time.perf_counter() - t0
    batch = nwg.RaggedBatch(graphs)
    tuner = Autotuner()
    t0 = time.perf_counter()
    params, bps = tuner.tune(batch, mn, roots)
    tune_s = time.perf_counter() - t0
    items = Autotuner.items(mn, roots, params)
    parents, offs, res, _ = batch.run(items, blocks_per_sm=bps)
    times = [batch.run(items, parents_dev=parents, blocks_per_sm=bps)[3] for _ in range(reps)]
    t = float(np.median(times))
    host = parents.cpu().numpy().view(np.uint32)
    e_total = 0.0
    for i, (g, r, *_rest) in enumerate(items):
        off = graphs[g][0]
        p = host[offs[i]:offs[i] + off.size - 1]
        e_total += float((off[1:] - off[:-1])[p != 0xFFFFFFFF].sum())
    per_call_ms = 0.0
    for g, (off, cols) in enumerate(graphs):
        G = nwg.Graph.from_csr(off, cols)
        for r in roots[g]:
            _, st = nwg.bfs(G, G, int(r), stats=True)
            per_call_ms += st.device_ms
        G.release()
    batch.release()
    return {"graphs": num_graphs, "items": len(items), "total_vertices": int(sum(n for n, _ in mn)),
            "total_entries": int(sum(m for _, m in mn)), "persistent_ms": t,
            "gteps": e_total / 2.0 / (t * 1e-3) / 1e9, "per_call_device_ms_sum": per_call_ms,
            "speedup_vs_per_call": per_call_ms / t, "blocks_per_sm": bps,
            "classes": len(params),
            "warp_min_per_class": {str(w): sum(1 for v in params.values() if v.warp_min == w)
                                   for w in sorted({v.warp_min for v in params.values()})},
            "generate_s": gen_s, "autotune_s": tune_s}


def profile_extension(args, torch):
    """Single runs of the multi-source pass or of betweenness for a profiler."""
    if args.profile_msbfs:
        os.environ["NWG_MS_STEPPED"] = "1"  # kernels launched one by one (ncu cannot enter conditional graphs)
    import nwgr_b200 as nwg

    g = nwg.Graph.rmat(22, 16, seed=GRAPH_SEED)
    roots = g.roots(max(64, args.ms_sources), seed=ROOT_SEED)
    if args.profile_msbfs:
        roots = roots[: args.ms_sources]
        ws = nwg.MsWorkspace(g)
        depths = torch.empty((roots.size, g.n), dtype=torch.uint8, device="cuda")
        ws.run(roots, depths)
        torch.cuda.synchronize()
        torch.cuda.nvtx.range_push("nwg_profile")
        st = ws.run(roots, depths)
        torch.cuda.synchronize()
        torch.cuda.nvtx.range_pop()
        print(json.dumps({"profile_msbfs": True, "levels": st.levels, "push": st.push_levels, "pull": st.pull_levels}))
        ws.close()
    else:
        nwg.betweenness(g, roots[:1], lanes=1)
        torch.cuda.synchronize()
        torch.cuda.nvtx.range_push("nwg_profile")
        _, st = nwg.betweenness(g, roots[:1], lanes=1)
        torch.cuda.synchronize()
        torch.cuda.nvtx.range_pop()
        print(json.dumps({"profile_bc": True, "levels": st.max_levels, "device_ms": st.device_ms}))
    g.release()


def bench_verifier(nwg, torch, g, roots, with_cpu):
    """Device BFSVerifier (nwg_verify) on the bench graph: device time of the
    check (its own top-down BFS plus the per-vertex parent checks) for the
    first roots' device parents, beside the reference's BFSVerifier
    (bfs.hpp:44-98, oracle/_ref) on the host for the first root."""
    par = torch.empty(g.n, dtype=torch.int32, device="cuda")
    out = {"roots": [], "device_ms": [], "valid": []}
    for r in roots[:4]:
        nwg.bfs_device(g, int(r), par)
        res = nwg.verify(g, int(r), par)
        out["roots"].append(int(r))
        out["device_ms"].append(float(res.device_ms))
        out["valid"].append(bool(res.valid))
    if with_cpu:
        from oracle.oracle import Reference

        off, cols = g.csr()
        nwg.bfs_device(g, int(roots[0]), par)
        host = par.cpu().numpy().view(np.uint32)
        ref = Reference()
        rg = ref.graph(off, cols)
        t0 = time.perf_counter()
        ok = rg.verify(int(roots[0]), host)
        out["reference_cpu_ms"] = 1e3 * (time.perf_counter() - t0)
        out["reference_valid"] = bool(ok)
        rg.close()
    return out


def bench_bc(nwg, scale=22, k=64, cpu_sample=4, with_cpu=True):
    """Approximate betweenness centrality (brandes_bc<float, double>) on
    RMAT-`scale` from k seeded sources: device time of nwg_bc, beside the
    reference's parallel brandes_bc on this host for the first cpu_sample
    sources (oracle/_ref, all host threads)."""
    g = nwg.Graph.rmat(scale, 16, seed=GRAPH_SEED)
    src = g.roots(k, seed=ROOT_SEED)
    nwg.betweenness(g, src[:4])  # warm-up
    times = []
    for _ in range(3):
        _, st = nwg.betweenness(g, src)
        times.append(st.device_ms)
    out = {"graph": f"RMAT-{scale} ef16", "sources": int(k), "device_ms": float(np.median(times)),
           "ms_per_source": float(np.median(times)) / k, "levels": int(st.max_levels), "lanes": int(st.lanes)}
    if with_cpu:
        from oracle.oracle import Reference

        off, cols = g.csr()
        ref = Reference()
        rg = ref.graph(off, cols)
        _, secs = rg.bc(src[:cpu_sample])
        rg.close()
        out["reference_cpu_ms_per_source"] = 1e3 * secs / cpu_sample
        out["reference_threads"] = ref.threads()
        out["speedup_per_source"] = out["reference_cpu_ms_per_source"] / out["ms_per_source"]
    g.release()
    return out


SERVE_RATES = (1000, 10000, 50000, 100000, 200000)


def bench_serving(nwg, num_graphs=200, rates=SERVE_RATES, seconds=1.5, slots=16, budget=16 << 30):
    """Serving: num_graphs resident graphs (the ragged distribution), an
    open-loop Poisson stream of (graph, root) queries per offered rate
    (`seconds` of arrivals, at least 2,000 queries), graph popularity
    Zipf(1.1), per-query-state budget 16 GiB, same-graph queries coalesced
    into multi-source passes, `slots` passes in flight.  Latency: scheduled
    arrival to the answer (uint8 depth row) in pinned host memory."""
    from nwgr_b200.serving import query_trace, serving_graphs

    t0 = time.perf_counter()
    graphs, pools = serving_graphs(nwg, num_graphs)
    gen_s = time.perf_counter() - t0
    csr_bytes = int(sum(8 * (g.n + 1) + 4 * g.m for g in graphs))
    server = nwg.Server(graphs, slots=slots, budget_bytes=budget)
    warm = query_trace(pools, 20000, 4000, seed=99)
    server.run_trace(*warm)
    out = []
    for rate in rates:
        count = int(max(2000, min(300000, rate * seconds)))
        gid, roots, arr = query_trace(pools, rate, count, seed=int(rate) % 1000003)
        _, bs, st = server.run_trace(gid, roots, arr)
        out.append({"offered_qps": rate, "queries": count, "qps": round(st.qps, 1), "p50_ms": round(st.p50_ms, 3),
                    "p99_ms": round(st.p99_ms, 3), "max_ms": round(st.max_ms, 3),
                    "mean_batch": round(st.mean_batch, 2), "failed": int(st.failed),
                    "peak_in_flight": int(st.peak_in_flight),
                    "overlap": round(st.batch_time_s / st.wall_s, 2) if st.wall_s > 0 else 0.0,
                    "peak_state_mb": round(st.peak_state_bytes / 1e6, 1)})
    info = {"slots": int(st.slots), "slot_bytes": int(st.slot_bytes), "state_budget_bytes": int(st.budget_bytes)}
    server.close()
    for g in graphs:
        g.release()
    return {"graphs": num_graphs, "csr_bytes": csr_bytes, "zipf_s": 1.1, "budget_bytes": budget, **info,
            "generate_s": gen_s, "rates": out}


def bench_other_graphs(nwg, torch, main_graph, hbm, with_cpu, n_roots=64, reps=3):
    """The other graphs of the single-source workload (RMAT-24, uniform 2^24
    at average degree 32, the 4096 x 4096 grid with 1% shortcuts), each
    timed like the main line: device time per traversal with the L2 flushed
    before it, GTEPS as the harmonic mean over `n_roots` roots, algorithmic
    bytes over time against the HBM peak; beside it the reference's bfs on
    the host for the first root."""
    out = {}
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    for name in ("rmat24", "uniform24", "grid4096"):
        if name == main_graph:
            continue
        spec = graph_spec(name)
        g = make_graph(nwg, spec)
        roots = g.roots(n_roots, seed=ROOT_SEED)
        ws = g.workspace()
        par = torch.empty(g.n, dtype=torch.int32, device="cuda")
        stream = torch.cuda.Stream()
        e_r, n_r = [], []
        for r in roots:
            with torch.cuda.stream(stream):
                ws.bfs_async(int(r), par, stream.cuda_stream)
            stream.synchronize()
            e, v = g.component_edges(par)
            e_r.append(e)
            n_r.append(v)
        e_r, n_r = np.asarray(e_r, np.float64), np.asarray(n_r, np.float64)
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in roots]
        times = []
        for rep in range(reps + 1):
            for i, r in enumerate(roots):
                with torch.cuda.stream(stream):
                    flush.fill_(i & 0xFF)
                    ev[i][0].record(stream)
                    ws.bfs_async(int(r), par, stream.cuda_stream)
                    ev[i][1].record(stream)
            stream.synchronize()
            if rep:  # the first pass over the roots is warm-up
                times.append([ev[i][0].elapsed_time(ev[i][1]) for i in range(len(roots))])
        t = np.mean(np.asarray(times), axis=0)
        gteps = (e_r / 2.0) / (t * 1e-3) / 1e9
        b_r = 4.0 * e_r + 8.0 * n_r + 4.0 * g.n
        achieved = float(np.mean(b_r / (t * 1e-3)) / 1e9)
        st = ws.stats()
        row = {"workload": workload_name(spec), "n": g.n, "m_directed": g.m, "roots": int(roots.size),
               "gteps": hmean(gteps), "ms_per_root_median": float(np.median(t)), "levels_last_root": int(st.levels),
               "roofline": {"achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm}}
        ws.close()
        if with_cpu:
            off, cols = g.csr()
            g.release()
            row["cpu_reference"] = cpu_baseline(off, cols, roots, 4, "after the device legs")
            del off, cols
        else:
            g.release()
        out[name] = row
    return out


def cpu_baseline(off, cols, roots, n_roots, when="before the device legs"):
    """The reference's bfs.hpp on the host cores over the first n_roots roots
    (each once; all of them by default, the roots the reference arm times)."""
    from oracle.oracle import Reference

    try:
        ref = Reference()
    except (FileNotFoundError, OSError) as e:
        return {"value": None, "unit": "GTEPS", "cores": 0, "kind": "reference", "sample": f"unavailable: {e}"}
    deg = off[1:] - off[:-1]
    rg = ref.graph(off, cols)
    rg.dobfs(int(roots[0]), 32, 15, 18, want_parents=False)  # warm the pool and pages
    k = min(int(n_roots), roots.size)
    secs, edges = reference_roots_timed(rg, deg, roots, list(range(k)))
    rg.close()
    return {"value": hmean(edges / secs / 1e9), "unit": "GTEPS", "cores": ref.threads(), "kind": "reference",
            "ms_per_root_median": 1e3 * float(np.median(secs)),
            "glibc_tunables": os.environ.get("GLIBC_TUNABLES", ""),
            "sample": f"the first {k} of the {roots.size} roots, once each, reference bfs.hpp on the project's "
                      f"TBB-compatible pool, wall clock around each call (time_op), {when}"}


MALLOC_THP = "glibc.malloc.hugetlb=1"


def reexec_with_malloc_thp(args):
    """Restarts this process (same PID, arguments and environment) with
    glibc's malloc asked to back its allocations with transparent huge
    pages.  The reference's bfs allocates its parent array, bitmaps and
    queues on every call; with 4 KB pages (THP in madvise mode, glibc's
    default) the same calls ran 1.47x slower on RMAT-24.  Both CPU legs
    (the reference arm and cpu_baseline) therefore run with it, the setting
    under which the reference is fastest."""
    if args.no_cpu and args.impl != "reference":
        return
    if args.profile_one or args.profile_trav or args.profile_msbfs or args.profile_bc or args.trace_steps:
        return
    cur = os.environ.get("GLIBC_TUNABLES", "")
    if MALLOC_THP in cur.split(":"):
        return
    env = dict(os.environ)
    env["GLIBC_TUNABLES"] = f"{cur}:{MALLOC_THP}" if cur else MALLOC_THP
    sys.stdout.flush()
    sys.stderr.flush()
    os.execve(sys.executable, [sys.executable, os.path.abspath(__file__)] + sys.argv[1:], env)


def main():
    args = parse()
    reexec_with_malloc_thp(args)
    spec = graph_spec(args.graph)
    world, rank, local = dist_setup(args)
    import torch

    if args.impl == "reference":
        if world > 1:
            torch.cuda.set_device(local)
        run_reference_arm(args, spec, world, rank)
        return

    torch.cuda.set_device(local)
    if args.profile_msbfs or args.profile_bc:
        profile_extension(args, torch)
        return
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=torch.device("cuda", local))
    import nwgr_b200 as nwg

    g = make_graph(nwg, spec)
    n, m = g.n, g.m
    roots = g.roots(args.roots, seed=ROOT_SEED)
    # the reference on the host cores first, in the same process state as the
    # reference arm (a fresh process holding only the graph): timed after the
    # GPU legs, the same calls ran up to 40% faster or slower from run to run
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu and not (args.profile_one or args.profile_trav or args.trace_steps):
        off, cols = g.csr()
        cpu = cpu_baseline(off, cols, roots, args.cpu_sample_roots)
        del off, cols
    stream = torch.cuda.Stream()
    ws = g.workspace()
    parents = torch.empty(n, dtype=torch.int32, device="cuda")
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")

    # per-root work (E_r, n_r) and launch counts from one untimed pass
    e_r, n_r, launches = [], [], []
    for r in roots:
        with torch.cuda.stream(stream):
            ws.bfs_async(int(r), parents, stream.cuda_stream)
        stream.synchronize()
        st = ws.stats()
        if st.status != 0:
            raise SystemExit(f"traversal from root {int(r)} reported status {st.status}")
        e, v = g.component_edges(parents)
        e_r.append(e)
        n_r.append(v)
        launches.append(st.kernel_launches)  # counted on the device
    e_r = np.asarray(e_r, np.float64)
    n_r = np.asarray(n_r, np.float64)

    if args.trace_steps:
        # per-step device time from the traversal's own %globaltimer stamps
        # (each step ends at the decision that follows it)
        out = []
        for r in roots[: args.trace_steps]:
            with torch.cuda.stream(stream):
                flush.fill_(2)
                ws.bfs_async(int(r), parents, stream.cuda_stream)
            stream.synchronize()
            st = ws.stats()
            tr = st.trace()
            us = st.step_ns() / 1e3
            out.append({"root": int(r), "status": int(st.status), "first_decide_us": round(int(st.first_decide_ns) / 1e3, 1),
                        "steps_us_total": round(float(us.sum()), 1),
                        "steps": [["BU" if tr["dir"][j] else "TD", int(tr["frontier"][j]), int(tr["found"][j]),
                                   round(float(us[j]), 1)] for j in range(len(us))]})
        print(json.dumps({"trace_steps": True, "workload": workload_name(spec), "roots": out}))
        return

    if args.profile_trav:
        # one traversal = one launch of the persistent kernel, after an L2 flush
        with torch.cuda.stream(stream):
            flush.fill_(1)
            torch.cuda.nvtx.range_push("nwg_profile")
            ws.bfs_async(int(roots[0]), parents, stream.cuda_stream)
            torch.cuda.nvtx.range_pop()
        stream.synchronize()
        st = ws.stats()
        print(json.dumps({"profile_trav": True, "root": int(roots[0]), "n": n, "m": m, "steps": st.steps,
                          "status": st.status, "kernel_launches": st.kernel_launches}))
        return

    if args.profile_one:
        # the step kernels launched one at a time from the host (per-step
        # figures; the persistent kernel runs all steps in one launch)
        nwg.bfs_stepped(g, int(roots[0]), parents)
        torch.cuda.synchronize()
        torch.cuda.nvtx.range_push("nwg_profile")
        st = nwg.bfs_stepped(g, int(roots[0]), parents)
        torch.cuda.synchronize()
        torch.cuda.nvtx.range_pop()
        print(json.dumps({"profile_one": True, "root": int(roots[0]), "n": n, "m": m, "steps": st.steps,
                          "trace_dir": st.trace()["dir"].tolist()}))
        return

    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in roots]

    def one_step(record):
        for i, r in enumerate(roots):
            with torch.cuda.stream(stream):
                flush.fill_(i & 0xFF)
                ev[i][0].record(stream)
                ws.bfs_async(int(r), parents, stream.cuda_stream)
                ev[i][1].record(stream)
        stream.synchronize()
        if record is not None:
            record.append([ev[i][0].elapsed_time(ev[i][1]) for i in range(len(roots))])

    for _ in range(args.warmup):
        one_step(None)
    clocks = ClockSampler(local)
    clocks.start()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    rec = []
    for _ in range(args.steps):
        one_step(rec)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    clk = clocks.stop()

    per_root_ms = max_over_ranks(np.mean(np.asarray(rec), axis=0), dist, "cuda")  # mean over steps, per root
    value, gteps = replica_gteps(e_r, per_root_ms, world)
    hbm, hbm_kind = peaks()
    b_r = 4.0 * e_r + 8.0 * n_r + 4.0 * n
    achieved_gbs = float(np.mean(b_r / (per_root_ms * 1e-3)) / 1e9)
    traffic = None
    if spec["kind"] in TRAFFIC_CAPTURES:
        cap_bytes, cap_m = TRAFFIC_CAPTURES[spec["kind"]]
        traffic = cap_bytes * m / cap_m

    # e2e through the C ABI with host buffers
    e2e = None
    if not args.no_e2e:
        off, cols = g.csr()
        off_p = torch.from_numpy(off.view(np.int64)).pin_memory()
        col_p = torch.from_numpy(cols.view(np.int32)).pin_memory()
        par_h = torch.empty(n, dtype=torch.int32).pin_memory()
        rows_h = torch.empty((len(roots), n), dtype=torch.int32).pin_memory()  # one parents row per root
        rows_np = rows_h.numpy().view(np.uint32)
        roots_u = np.asarray(roots, dtype=np.uint32)
        h2d = off.nbytes + cols.nbytes
        e2e_vals, ups, steps_s, roots_s, calls = [], [], [], [], []
        for step in range(args.warmup + args.steps):  # the first `warmup` steps are untimed
            t0 = time.perf_counter()
            ge = nwg.Graph.from_csr(off_p.numpy().view(np.uint64), col_p.numpy().view(np.uint32))
            up = time.perf_counter() - t0
            nwg.bfs_roots(ge, roots_u, parents_out=rows_np)
            total = time.perf_counter() - t0
            if step == 0:  # untimed: one nwg_bfs call per root, for the per-call figure
                for r in roots:
                    t1 = time.perf_counter()
                    nwg.bfs(ge, ge, int(r), parents_out=par_h.numpy().view(np.uint32))
                    calls.append(time.perf_counter() - t1)
            ge.release()
            if step >= args.warmup:
                # each root's share of the step: the upload and every traversal
                # and parents copy of the step, divided evenly over the roots
                e2e_vals.append(hmean((e_r / 2.0) / (total / len(roots)) / 1e9))
                ups.append(up)
                steps_s.append(total)
                roots_s.append(total - up)
        for i in (0, len(roots) - 1):  # the rows are the traversals of their roots
            if int(np.count_nonzero(rows_np[i] != 0xFFFFFFFF)) != int(n_r[i]) or rows_np[i][roots_u[i]] != roots_u[i]:
                raise RuntimeError("e2e: nwg_bfs_roots row %d is not the traversal of its root" % i)
        per_call = float(hmean((e_r / 2.0) / (np.asarray(calls) + float(np.median(ups)) / len(roots)) / 1e9))
        # the copies alone, for the split of the call time: one parent array
        # device -> pinned host, and the CSR host -> device
        d2h_s, h2d_s = [], []
        for _ in range(5):
            ta = time.perf_counter()
            par_h.copy_(parents)
            torch.cuda.synchronize()
            d2h_s.append(time.perf_counter() - ta)
        off_d = torch.empty(off.size, dtype=torch.int64, device="cuda")
        col_d = torch.empty(cols.size, dtype=torch.int32, device="cuda")
        for _ in range(2):
            ta = time.perf_counter()
            off_d.copy_(off_p)
            col_d.copy_(col_p)
            torch.cuda.synchronize()
            h2d_s.append(time.perf_counter() - ta)
        del off_d, col_d
        e2e = {"value": float(np.mean(e2e_vals)) * world, "unit": "GTEPS", "h2d_bytes_per_step": int(h2d),
               "d2h_bytes_per_step": int(4 * n * len(roots)),
               "upload_s_median": float(np.median(ups)), "upload_gbs": h2d / float(np.median(ups)) / 1e9,
               "h2d_copy_gbs": h2d / min(h2d_s) / 1e9, "d2h_copy_gbs": 4.0 * n / min(d2h_s) / 1e9,
               "d2h_copy_ms": 1e3 * min(d2h_s), "step_ms_median": 1e3 * float(np.median(steps_s)),
               "steps_gteps": [round(float(x) * world, 1) for x in e2e_vals],
               "steps_upload_ms": [round(1e3 * x, 2) for x in ups],
               "steps_roots_ms": [round(1e3 * x, 2) for x in roots_s],
               "per_call_gteps": per_call * world, "call_ms_median": 1e3 * float(np.median(calls)),
               "note": "per step: upload CSR from pinned host memory (registration), nwg_bfs_roots over the "
                       "64 roots (two traversals in flight, each root's parents copied to its own pinned host "
                       "row), release; each root is charged step time / 64; per_call_gteps: the same with one "
                       "synchronous nwg_bfs call per root; *_copy_gbs: the same bytes copied alone (one parent "
                       "array, one CSR)"}
    verifier = None
    if not args.no_verify:
        verifier = bench_verifier(nwg, torch, g, roots, rank == 0 and not args.no_cpu)
    other = None
    if not args.no_other and rank == 0:
        if ws is not None:
            ws.close()
            g.release()
            ws, g = None, None
        other = bench_other_graphs(nwg, torch, args.graph, hbm, not args.no_cpu)
    batched = None
    if not args.no_batched:
        if ws is not None:
            ws.close()
            g.release()
            ws, g = None, None
        batched = bench_batched(nwg, torch)
    ragged = None
    if not args.no_ragged:
        if ws is not None:
            ws.close()
            g.release()
            ws, g = None, None
        ragged = bench_ragged(nwg, torch)
    serving = None
    if not args.no_serving:
        if ws is not None:
            ws.close()
            g.release()
            ws, g = None, None
        serving = bench_serving(nwg, slots=args.serve_slots)
    bc = None
    if not args.no_bc:
        if ws is not None:
            ws.close()
            g.release()
            ws, g = None, None
        bc = bench_bc(nwg, with_cpu=rank == 0 and not args.no_cpu)

    if rank == 0:
        line = {
            "metric": metric_name(args, len(roots)),
            "value": value, "unit": "GTEPS", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": float(np.sum(per_root_ms)), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "uint32", "data": "synthetic (seeded device generator)",
            "config": {"workload": workload_name(spec), "n": n, "m_directed": m, "roots": len(roots),
                       "alpha": 15, "beta": 18, "timing": "device time (CUDA events per traversal)",
                       "l2": "flushed (256 MB write) before every traversal",
                       "parallelism": f"replicas x{world}" if world > 1 else "1 GPU"},
            "gteps_min": float(np.min(gteps)), "gteps_max": float(np.max(gteps)),
            "ms_per_root_median": float(np.median(per_root_ms)), "wall_s_timed": wall,
            "roofline": {"bound": "hbm", "achieved": achieved_gbs, "peak": hbm, "unit": "GB/s",
                         "frac": achieved_gbs / hbm, "peak_kind": hbm_kind,
                         "kernel": "k_trav: one cooperative launch per traversal (init, decisions, top-down, "
                                   "pull and bitmap-to-queue steps, solo levels)",
                         "algorithmic_bytes_per_launch_mean": float(np.mean(b_r)),
                         "traffic": traffic,
                         "traffic_note": "ncu DRAM bytes of one traversal of the same graph kind at scale 22, "
                                         "scaled by directed entries" if traffic else None},
            "gpu_launches": int(np.sum(launches)) * args.steps,
            # the driver keeps the last ~1.6 KB of the line: the batched
            # result (the extension's target) goes last
            "clocks": clk, "e2e": e2e, "cpu_baseline": cpu, "other_graphs": other, "verifier": verifier,
            "betweenness": bc, "serving": serving, "ragged": ragged, "batched": batched,
        }
        print(json.dumps(line), flush=True)
    if ws is not None:
        ws.close()
    if g is not None:
        g.release()
    if dist:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
