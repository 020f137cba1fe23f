"""CPU checks of bench.py's host logic, including the multi-rank path as
world-size-2 gloo ranks (the GPU run uses NCCL; the reduction is the same)."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402


def test_harmonic_mean_and_replica_throughput():
    assert bench.hmean([1.0, 1.0]) == pytest.approx(1.0)
    assert bench.hmean([1.0, 3.0]) == pytest.approx(1.5)
    e_r = np.array([2e9, 2e9])
    v, g = bench.replica_gteps(e_r, np.array([1.0, 2.0]), 1)
    assert np.allclose(g, [1000.0, 500.0])
    assert v == pytest.approx(bench.hmean([1000.0, 500.0]))
    v4, _ = bench.replica_gteps(e_r, np.array([1.0, 2.0]), 4)
    assert v4 == pytest.approx(4 * v)


def test_graph_specs():
    assert bench.graph_spec("rmat24") == {"kind": "rmat", "scale": 24, "edge_factor": 16}
    assert bench.graph_spec("rmat18")["scale"] == 18
    assert bench.graph_spec("uniform24")["n"] == 1 << 24
    assert bench.graph_spec("grid4096")["width"] == 4096
    with pytest.raises(SystemExit):
        bench.graph_spec("nope")


def test_both_arms_name_the_same_metric(monkeypatch):
    """The reference arm and this library's arm print one metric string for
    the same workload and root count, so their values can be divided."""
    monkeypatch.setattr(sys, "argv", ["bench.py"])
    args = bench.parse()
    assert args.roots == 64 and args.graph == "rmat24" and args.warmup >= 3
    assert bench.metric_name(args, args.roots) == "BFS GTEPS (harmonic mean over 64 roots) @ rmat24"
    monkeypatch.setattr(sys, "argv", ["bench.py", "--impl", "reference"])
    ref = bench.parse()
    assert bench.metric_name(ref, ref.roots) == bench.metric_name(args, args.roots)


def _rank(rank, world, port, q):
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        local = np.array([1.0 + rank, 5.0 - 3 * rank, 2.0])  # rank 0: [1,5,2]; rank 1: [2,2,2]
        q.put((rank, bench.max_over_ranks(local, dist, "cpu").tolist()))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_gloo_world2():
    import multiprocessing as mp
    import socket

    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = dict(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert out[0] == out[1] == [2.0, 5.0, 2.0]
