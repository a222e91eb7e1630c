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
