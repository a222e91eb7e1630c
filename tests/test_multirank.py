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


def _shard_worker(rank, world, port, out):
    import numpy as np
    import torch
    import torch.distributed as dist

    from fresco_b200.shard import shard_totals
    from oracle import oracle as O

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        x, _, Sk, V, L = O.stealthy_nuwu_inputs(900, 9, 8, ndim=2, seed=12)
        radii = 0.5 + np.random.default_rng(13).random(900)
        cut = [0, 350, 900]  # uneven slabs
        pts = x.reshape(-1, 2)[cut[rank] : cut[rank + 1]].ravel()
        r_loc = radii[cut[rank] : cut[rank + 1]]
        n_total, ws = shard_totals(r_loc, 2)  # all-reduce over the gloo group
        ref = O.NUwU(radii, 9, Sk, V, L)
        c_loc = (np.pi * r_loc * r_loc) ** 2 * (n_total / ws)  # nuwu.hpp:125-149 over the whole pattern
        rho = ref.rho_active(pts, c_loc)
        t = torch.from_numpy(np.stack([rho.real, rho.imag]))
        dist.all_reduce(t)  # the one exchange per evaluation
        phi, g = ref.finish_active(t[0].numpy() + 1j * t[1].numpy(), pts, c_loc, n_total)
        gathered = [None] * world
        dist.all_gather_object(gathered, g)
        out.put((rank, n_total, ws, phi, np.concatenate(gathered)))
    finally:
        dist.destroy_process_group()


def test_two_rank_sharded_pattern_totals_and_loss():
    """One NUwU pattern split into two uneven slabs over two gloo ranks: the point and weight totals
    reach every rank, and the rank-local rho summed by one all-reduce gives every rank the whole
    pattern's loss and each rank its points' share of the gradient (oracle arithmetic standing in for
    the device steps of fresco_b200.ShardedNUwU)."""
    import numpy as np
    import torch.multiprocessing as mp

    from fresco_b200.shard import weight_factor_sum
    from oracle import oracle as O

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_shard_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=180)
    assert all(p.exitcode == 0 for p in procs)
    res = sorted((q.get(timeout=5) for _ in range(2)), key=lambda t: t[0])
    x, _, Sk, V, L = O.stealthy_nuwu_inputs(900, 9, 8, ndim=2, seed=12)
    radii = 0.5 + np.random.default_rng(13).random(900)
    e_ref, g_ref = O.NUwU(radii, 9, Sk, V, L).get_energy_gradient(x)
    for rank, n_total, ws, phi, g in res:
        assert n_total == 900
        assert ws == pytest.approx(weight_factor_sum(radii, 2), rel=1e-14)
        assert phi == pytest.approx(e_ref, rel=1e-11)
        assert np.linalg.norm(g - g_ref) <= 1e-11 * np.linalg.norm(g_ref)


def _halo_columns(p, L0, nc):
    """Column (cell along axis 0) of each point: the expression the device kernels use."""
    import numpy as np

    u = p[:, 0] - np.floor(p[:, 0] / L0) * L0
    return np.clip((u * (nc / L0)).astype(np.int64), 0, nc - 1)


def _halo_worker(rank, world, port, out):
    """The halo exchange of ShardedInversePower(halo=True) restated on the host over gloo: column marks
    and exports travel through gather_varying; each rank's share (own points' gradients, pairs whose
    lower index is its own) must add up to the whole pattern's repulsion."""
    import numpy as np
    import torch
    import torch.distributed as dist

    from fresco_b200.shard import gather_varying, spatial_order
    from oracle import oracle as O

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        rng = np.random.default_rng(4)
        n, L = 600, np.ones(2)
        x = rng.random((n, 2))
        radii = (0.5 / np.sqrt(np.pi * n)) * (1 + 0.2 * (rng.random(n) - 0.5))
        p = spatial_order(x.ravel(), L)
        x, radii = x[p], radii[p]
        rcut = 2 * radii.max()
        nc = int(min(np.floor(L[0] / (rcut * (1 + 1e-9))), np.floor(np.sqrt(n))))
        lo, hi = n * rank // world, n * (rank + 1) // world
        own = x[lo:hi]
        col = _halo_columns(own, L[0], nc)
        marks = np.zeros(nc, dtype=np.float64)
        marks[col] = 1.0
        allm, counts = gather_varying(torch.tensor(marks), None)
        assert counts == [nc] * world
        allm = allm.numpy().reshape(world, nc) > 0
        near = allm | np.roll(allm, 1, axis=1) | np.roll(allm, -1, axis=1)  # columns next to each rank's
        need = near[[q for q in range(world) if q != rank]].any(axis=0)
        reach = near[rank]
        sel = need[col]
        exp = np.concatenate([own[sel], (lo + np.nonzero(sel)[0])[:, None].astype(np.float64)], axis=1)
        recv, rc = gather_varying(torch.tensor(exp.ravel()), None)
        recv = recv.numpy().reshape(-1, 3)
        skip = sum(rc[:rank]) // 3
        others = np.concatenate([recv[:skip], recv[skip + rc[rank] // 3:]])
        halo = others[reach[_halo_columns(others[:, :2], L[0], nc)]]
        pts = np.concatenate([own, halo[:, :2]])
        gidx = np.concatenate([np.arange(lo, hi), halo[:, 2].astype(np.int64)])
        # own points' pairs over own + halo points (O(n^2) on this small case)
        i, j = np.triu_indices(len(pts), k=1)
        dr = pts[i] - pts[j]
        dr -= np.round(dr / L) * L
        r2 = np.sum(dr * dr, axis=1)
        rs = radii[gidx[i]] + radii[gidx[j]]
        m = r2 < rs * rs
        r = np.sqrt(r2[m])
        f = (1 - r / rs[m]) ** 2
        low = np.minimum(gidx[i][m], gidx[j][m])
        e = float(np.sum((f / 2)[(low >= lo) & (low < hi)]))
        gij = -f / ((r - rs[m]) * r)
        g = np.zeros_like(pts)
        np.add.at(g, i[m], -dr[m] * gij[:, None])
        np.add.at(g, j[m], dr[m] * gij[:, None])
        et = torch.tensor([e], dtype=torch.float64)
        dist.all_reduce(et)
        e_ref, g_ref = O.InversePower(2.0, 1.0, radii, L).get_energy_gradient(x.ravel())
        out.put((rank, float(et[0]), e_ref, float(np.max(np.abs(g[:hi - lo].ravel() - g_ref[2 * lo:2 * hi])) /
                                                    np.max(np.abs(g_ref))),
                 int(sel.sum()), len(halo)))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_rank_halo_exchange_logic():
    """Two gloo ranks run the halo exchange's host-side restatement: the energies add up to the whole
    pattern's, each rank's gradients are exact, and only the points near the slab ends travel."""
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_halo_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=180)
    assert all(p.exitcode == 0 for p in procs)
    res = sorted(q.get(timeout=5) for _ in range(2))
    for rank, e, e_ref, gerr, exported, halo in res:
        assert e_ref > 0 and abs(e - e_ref) <= 1e-12 * e_ref
        assert gerr <= 1e-12
        assert 0 < exported < 200 and 0 < halo < 300
