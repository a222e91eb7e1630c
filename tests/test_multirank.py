"""Host logic of the multi-GPU benchmark path with two gloo ranks on CPU: every rank reports its own
time, the job time is the slowest rank's, and the value aggregates all ranks' steps."""
import os
import socket

import pytest


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import torch
    import torch.distributed as dist

    import bench

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        local_ms = 100.0 * (rank + 1)  # rank 1 is the slow one
        job_ms = bench.reduce_max(local_ms, "cpu")
        value = bench.job_value(world, 10, job_ms)
        out.put((rank, job_ms, value))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_rank_max_timing_and_aggregate_value():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs)
    res = sorted(q.get(timeout=5) for _ in range(2))
    for rank, job_ms, value in res:
        assert job_ms == pytest.approx(200.0)
        assert value == pytest.approx(2 * 10 / 0.2)


def test_single_process_helpers():
    import bench

    assert bench.reduce_max(3.5, "cpu") == 3.5
    assert bench.job_value(1, 20, 500.0) == pytest.approx(40.0)


def test_shard_patterns_covers_every_pattern_once_and_balances():
    """Longest-processing-time-first sharding of a config-5-like ensemble (256 patterns)."""
    import numpy as np

    from fresco_b200.ensemble import pattern_cost, shard_patterns

    rng = np.random.default_rng(5)
    N = np.exp(rng.uniform(np.log(1000), np.log(200000), 256)).astype(int)
    side = rng.choice([64, 128, 256, 512], 256)
    costs = [pattern_cost(n, s + 1) for n, s in zip(N, side)]
    for ws in [1, 2, 3, 8]:
        parts = shard_patterns(costs, ws)
        assert len(parts) == ws
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(256))
        loads = [sum(costs[i] for i in p) for p in parts]
        assert max(loads) <= sum(costs) / ws + max(costs) + 1e-6
    with pytest.raises(ValueError):
        shard_patterns(costs, 0)


def _gather_worker(rank, world, port, out):
    import torch.distributed as dist

    from fresco_b200.ensemble import gather_results, shard_patterns

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        costs = [float(7 * i % 11 + 1) for i in range(23)]
        mine = shard_patterns(costs, world)[rank]
        local = [{"pattern": i, "energy": 0.5 * i, "rank": rank} for i in mine]
        merged = gather_results(local, mine)
        out.put((rank, [(r["pattern"], r["energy"]) for r in merged], sorted({r["rank"] for r in merged})))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_rank_ensemble_gather():
    """Each rank keeps its own shard of patterns; the final gather gives every rank all results in order."""
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_gather_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=180)
    assert all(p.exitcode == 0 for p in procs)
    res = sorted(q.get(timeout=5) for _ in range(2))
    for rank, merged, ranks in res:
        assert merged == [(i, 0.5 * i) for i in range(23)]
        assert ranks == [0, 1]
