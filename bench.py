"""Benchmark: NUwU loss+gradient evaluations per second on B200.

Workload (one "step" = one NUwU ``get_energy_gradient``): 2D NUwU with
N = 1,048,576 seeded uniform points in [0, 2 pi)^2, a 1025 x 1025 mode grid
(K = 512; the reference supports only odd grids), target S0(k) = 0 for
0 < |k| <= 256 with weight 1, unconstrained elsewhere, L = 2 pi, eps = 1e-6,
in the FP32 spread/FFT/interpolation form with FP64 reductions.  Synthetic
seeded inputs stand in for data (the reference uses none).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Under torchrun (N > 1) every rank evaluates its own independent pattern (the
batched-ensemble sharding: no data-path collective), timing is the max over
ranks and ``value`` aggregates all ranks.  The ``sharded_pattern`` section
splits one config-2 pattern over the ranks instead (one all-reduce of rho at
the active modes per evaluation).  ``--impl reference`` times the
reference's own CPU implementation (its C++ compiled unchanged against the
FINUFFT-API shim backed by the CPU ES-kernel NUFFT restatement) on rank 0.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "NUwU loss+grad evals/s, 2D N=1M: FP32 vs FP64 on B200 at ≤1e-5 grad rel err"
N_POINTS = 1 << 20
K_MODES = 512
K_CONSTRAINED = 256
EPS = 1e-6
# eps whose kernel width (w = 6) the FP32 form needs for a 1e-5 relative gradient error
EPS_FP32_BOUND = 1e-5
L2_FLUSH_BYTES = 256 << 20

WORKLOAD = (
    "2D NUwU loss+grad: N=1048576 seeded uniform points in [0,2pi)^2, 1025x1025 modes (K=512), "
    "S0=0 & V=1 on 0<|k|<=256, L=2pi, eps=1e-6"
)


def stealthy_inputs(n_points, K, kmax, seed, box=2 * np.pi):
    """Seeded uniform points in [0, box)^2, radii 1, S0 = 0 and V = 1 on 0 < |k| <= kmax of the
    (2K+1)^2 mode grid."""
    rng = np.random.default_rng(seed)
    L = np.full(2, float(box))
    x = (rng.random((n_points, 2)) * L).ravel()
    kv = np.arange(-K, K + 1)
    kx, ky = np.meshgrid(kv, kv, indexing="ij")
    kmag = np.sqrt(kx.astype(np.float64) ** 2 + ky.astype(np.float64) ** 2)
    V = ((kmag <= kmax) & (kmag > 0)).astype(np.float64)
    return x, np.ones(n_points), np.zeros_like(V), V, L


def inputs(seed):
    return stealthy_inputs(N_POINTS, K_MODES, K_CONSTRAINED, seed)


ENSEMBLE_PATTERNS = 256
ENSEMBLE_WORKLOAD = (
    "batched 2D NUwU ensemble: 256 seeded patterns, N log-uniform in [1000, 200000], k-grid side uniform in "
    "{64,128,256,512} (K = side/2, odd (side+1)^2 modes), stealthy disc S0=0 & V=1 on 0<|k|<=side/8, "
    "L=2pi, eps=1e-6, FP32 spread/FFT/interp"
)


def ensemble_inputs(seed=5, n_patterns=ENSEMBLE_PATTERNS):
    """Per-pattern (x, radii, K, Sk, V) of the batched-ensemble workload."""
    rng = np.random.default_rng(seed)
    N = np.exp(rng.uniform(np.log(1000), np.log(200000), n_patterns)).astype(np.int64)
    side = rng.choice([64, 128, 256, 512], n_patterns)
    pats = []
    for p in range(n_patterns):
        K = int(side[p]) // 2
        x, r, Sk, V, L = stealthy_inputs(int(N[p]), K, int(side[p]) // 8, seed=1000 + p)
        pats.append((x, r, K, Sk.ravel(), V.ravel()))
    return pats, np.full(2, 2 * np.pi)


def ensemble_report(args, dev, ws, rank):
    """Batched ensemble: the rank's cost-model shard of the 256 patterns as one NUwUEnsemble (FP32),
    evaluations of every pattern per second (device-timed graph replays, max over ranks) and
    per-pattern device LBFGS steps; at one GPU also the same patterns as 256 separate NUwU
    potentials evaluated one after another (graph replay each)."""
    import torch

    from fresco_b200 import EnsembleLBFGS, NUwU, NUwUEnsemble
    from fresco_b200.ensemble import pattern_cost, shard_patterns

    pats, L = ensemble_inputs()
    costs = [pattern_cost(len(x) // 2, 2 * K + 1) for x, _, K, _, _ in pats]
    mine = shard_patterns(costs, ws)[rank]
    sel = [pats[i] for i in mine]
    ens = NUwUEnsemble([r for _, r, _, _, _ in sel], [K for _, _, K, _, _ in sel], [s for _, _, _, s, _ in sel],
                       [v for _, _, _, _, v in sel], L, eps=EPS, precision="fp32")
    xs = [x for x, _, _, _, _ in sel]
    t0 = time.perf_counter()
    ens.tune(xs)
    tune_s = time.perf_counter() - t0
    dx = torch.tensor(ens.concat(xs), device=dev)
    dg = torch.empty_like(dx)
    de = torch.empty(ens.n_patterns, dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev)
    for _ in range(max(3, args.warmup)):
        ens.get_energies_gradient_device(dx, dg, de, stream.cuda_stream)
    torch.cuda.synchronize()
    n = max(5, args.steps // 2)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    for _ in range(n):  # the points (154 MB) and grids exceed L2: no flush needed between steps
        ens.get_energies_gradient_device(dx, dg, de, stream.cuda_stream)
    b.record(stream)
    torch.cuda.synchronize()
    ms = reduce_max(a.elapsed_time(b) / n, dev)
    total_points = sum(len(x) // 2 for x, _, _, _, _ in pats)
    out = {"workload": ENSEMBLE_WORKLOAD, "patterns": len(pats), "points": int(total_points),
           "pattern_evals_per_s": round(len(pats) / (ms * 1e-3), 1), "ms_per_ensemble_eval": round(ms, 4),
           "points_per_s": round(total_points / (ms * 1e-3), 1), "tune_s": round(tune_s, 2),
           "setup": ens.describe()}
    # device LBFGS (M = 4) for every pattern: one graph launch per step (host clock around steps())
    opt = EnsembleLBFGS(xs, ens, M=4, tol=1e-12)
    opt.steps(3)
    nst = max(10, args.steps // 2)
    _, _, f0, _, it0, _, _ = opt.state(False)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    opt.steps(nst)
    lb_s = reduce_max(time.perf_counter() - t0, dev)
    _, _, f1, _, it1, _, _ = opt.state(False)
    out["lbfgs"] = {"steps_per_s": round(nst / lb_s, 2), "pattern_iterations_per_s":
                    round(reduce_sum(float(np.sum(it1 - it0)), dev) / lb_s, 1),
                    "patterns_lower_energy": int(reduce_sum(float(np.sum(f1 < f0)), dev)), "M": 4,
                    "timing": "host wall clock around the graph launches of steps(), max over ranks"}
    # run(niter): the whole minimisation as ONE graph launch (a conditional WHILE node repeats the step
    # while a pattern is still iterating)
    n_run = max(10, args.steps // 2)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    used = opt.run(n_run)
    run_s = reduce_max(time.perf_counter() - t0, dev)
    _, _, _, _, it2, _, _ = opt.state(False)
    out["lbfgs"]["run_one_launch"] = {
        "niter": n_run, "steps": int(used), "steps_per_s": round(used / run_s, 2),
        "pattern_iterations_per_s": round(reduce_sum(float(np.sum(it2 - it1)), dev) / run_s, 1),
        "timing": "host wall clock around run(), one graph launch, max over ranks"}
    del opt
    if ws == 1 and not args.no_ensemble_loop:
        # the same patterns as separate potentials, one after another on one stream
        pots = [NUwU(r, K, s, v, L, eps=EPS, precision="fp32") for _, r, K, s, v in pats]
        bufs = [(torch.tensor(x, device=dev), torch.empty(len(x), dtype=torch.float64, device=dev),
                 torch.empty((), dtype=torch.float64, device=dev)) for x, _, _, _, _ in pats]
        for _ in range(2):
            for pot, (px, pg, pe) in zip(pots, bufs):
                pot.energy_gradient_device(px, pg, pe)
        torch.cuda.synchronize()
        a.record(stream)
        for _ in range(3):
            for pot, (px, pg, pe) in zip(pots, bufs):
                pot.energy_gradient_device(px, pg, pe)
        b.record(stream)
        torch.cuda.synchronize()
        ms_loop = a.elapsed_time(b) / 3
        out["separate_potentials"] = {"pattern_evals_per_s": round(len(pats) / (ms_loop * 1e-3), 1),
                                      "ms_per_ensemble_eval": round(ms_loop, 4)}
        del pots, bufs
    del ens
    return out


def sharded_report(args, dev, ws, rank):
    """One config-2 pattern (seed 2, N = 2^20) split into equal index slabs over the job's ranks
    (fresco_b200.ShardedNUwU, FP32): per evaluation every rank computes rho of its slab at the
    active modes, one NCCL all-reduce sums them, every rank finishes the loss and its slab's
    gradient.  Device-timed, max over ranks; whole-pattern evaluations per second.  With one rank
    it is the single-GPU cost of the sharded path (cuFFT transforms; no collective)."""
    import torch

    from fresco_b200 import ShardedNUwU

    x, radii, Sk, V, L = inputs(seed=2)
    a, b = rank * N_POINTS // ws, (rank + 1) * N_POINTS // ws
    sh = ShardedNUwU(radii[a:b], K_MODES, Sk, V, L, eps=EPS, precision="fp32")
    dx = torch.tensor(x[2 * a : 2 * b], device=dev)
    stream = torch.cuda.current_stream(dev)

    def one_eval():
        r = sh.reduce(sh.rho(dx))
        return sh.finish(r)

    for _ in range(max(3, args.warmup)):
        e, _ = one_eval()
    torch.cuda.synchronize()
    if ws > 1:
        torch.distributed.barrier()
    n = max(5, args.steps)
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0.record(stream)
    for _ in range(n):
        e, _ = one_eval()
    t1.record(stream)
    torch.cuda.synchronize()
    ms = reduce_max(t0.elapsed_time(t1) / n, dev)
    out = {"workload": "the config-2 NUwU pattern (seed 2) split into equal point slabs, one per rank",
           "ranks": ws, "points_per_rank": int(b - a), "evals_per_s": round(1000.0 / ms, 2),
           "ms_per_eval": round(ms, 5), "allreduce_bytes_per_eval": int(16 * sh.n_rho),
           "energy": float(e.item()), "transforms": "cuFFT (pruned column passes)",
           "timing": "CUDA events on the launch stream, max over ranks"}
    if ws == 1:
        # LBFGS over the sharded pattern: the device LBFGS with its dot products and the shard's rho
        # passed through the exchange hook (a no-op with one rank); one process only, so that a
        # multi-rank job takes no collective here that its other sections do not
        from fresco_b200 import ShardedLBFGS

        opt = ShardedLBFGS(x[2 * a : 2 * b], sh, M=4, tol=0.0)
        opt.run(3)
        torch.cuda.synchronize()
        from fresco_b200._lib import check as _check, lib as _clib

        n_it = max(20, args.steps)
        t_0 = time.perf_counter()
        _check(_clib.fresco_optimizer_run(opt._opt._h, n_it))  # the iterations only, as the lbfgs section
        torch.cuda.synchronize()
        dt = time.perf_counter() - t_0
        res = opt.get_result()
        out["lbfgs"] = {"iterations_per_s": round(n_it / dt, 2), "iterations": n_it, "evals": int(res.nfev),
                        "energy": float(res.energy), "exchange_calls": int(opt.reducer.calls), "M": 4,
                        "timing": "host wall clock around the C-level run loop, one rank"}
    # config 2's repulsion over spatial slabs with the halo exchange: the points in spatial order, one
    # equal slab per rank; each rank evaluates its own points' pairs against its halo
    from fresco_b200.shard import ShardedInversePower, spatial_order

    rr = np.full(N_POINTS, 0.25 / np.sqrt(N_POINTS) * 2 * np.pi)
    xs = x.reshape(-1, 2)[spatial_order(x, L)].ravel()
    rep = ShardedInversePower(2.0, 1.0, rr, L, a, b, halo=True)
    dxs = torch.tensor(xs[2 * a : 2 * b], device=dev)
    gs = torch.empty_like(dxs)
    es = torch.zeros((), dtype=torch.float64, device=dev)
    for _ in range(3):
        rep.energy_gradient_device(dxs, grad=gs, out=es)
    torch.cuda.synchronize()
    if ws > 1:
        torch.distributed.barrier()
    n_h = max(5, args.steps)
    t_0 = time.perf_counter()
    for _ in range(n_h):
        rep.energy_gradient_device(dxs, grad=gs, out=es)
    torch.cuda.synchronize()
    dt_h = reduce_max(time.perf_counter() - t_0, dev)
    rep.exchange.check()
    exported, halo = rep.halo_stats()
    out["halo_repulsion"] = {
        "workload": "config-2 repulsion (N=2^20, diameter 0.5/sqrt(N) 2 pi), points in spatial order, one equal "
                    "slab per rank", "evals_per_s": round(n_h / dt_h, 2), "energy": float(es.item()),
        "exported_points": exported, "halo_points": halo, "exchange_bytes_per_eval": int(24 * exported),
        "setup": rep.describe(),
        "timing": "host wall clock around the evaluations (each reads the exchange sizes back), max over ranks"}
    del rep
    return out


def other_configs_report(args, dev):
    """Device-timed loss+gradient evaluations per second of the other configurations' potentials on
    this GPU (each input exceeds the 126 MB L2 or is evaluated back to back; no flush): config 3 3D
    NUwU (N = 2^21, 129^3 modes, radial S0 and V) FP32 and FP64, config 4 UwU on 4096^2 and UwNU on
    2048^2 against 100,000 k-points FP32 and FP64, config 1 NUwU (N = 4096, 65^2 modes) FP64."""
    import torch

    from fresco_b200 import NUwU, UwNU, UwU

    def rate(pot, x):
        xd = torch.tensor(x, device=dev)
        g = torch.empty_like(xd)
        e = torch.zeros((), dtype=torch.float64, device=dev)
        for _ in range(3):
            pot.energy_gradient_device(xd, grad=g, out=e)
        torch.cuda.synchronize()
        n = max(5, args.steps // 2)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(n):
            pot.energy_gradient_device(xd, grad=g, out=e)
        b.record()
        torch.cuda.synchronize()
        ms = a.elapsed_time(b) / n
        return {"evals_per_s": round(1000.0 / ms, 2), "ms_per_eval": round(ms, 4)}

    out = {}
    rng = np.random.default_rng(3)
    n3, k3 = 1 << 21, 64
    x3 = rng.random(3 * n3) * 2 * np.pi
    kv = np.arange(-k3, k3 + 1)
    kz, ky, kx = np.meshgrid(kv, kv, kv, indexing="ij")
    mag = np.sqrt(kx ** 2 + ky ** 2 + kz ** 2).ravel().astype(np.float64)
    sk3, v3 = 1.0 - np.exp(-((mag / 16.0) ** 2)), np.where(mag > 0, 1.0 / (1.0 + mag), 0.0)
    out["config3_nuwu3d"] = {"workload": "3D NUwU, N=2097152 uniform in [0,2pi)^3, 129^3 modes, "
                             "S0=1-exp(-(|k|/16)^2), V=1/(1+|k|), V(0)=0, eps=1e-6"}
    for prec in ("fp32", "fp64"):
        out["config3_nuwu3d"][prec] = rate(NUwU(np.ones(n3), k3, sk3, v3, np.full(3, 2 * np.pi), eps=EPS,
                                                precision=prec), x3)
    del x3, sk3, v3, mag, kx, ky, kz
    rng = np.random.default_rng(4)
    g4 = 4096
    xg = rng.random(g4 * g4)
    k = np.arange(g4) - g4 // 2
    m4 = np.sqrt(k[:, None] ** 2 + k[None, :] ** 2)
    v4 = ((m4 <= 64) & (m4 > 0)).astype(np.float64)
    out["config4_uwu"] = {"workload": "UwU on a 4096^2 grid, x uniform in [0,1], S0=0 & V=1 on 0<|k|<=64"}
    for prec in ("fp32", "fp64"):
        out["config4_uwu"][prec] = rate(UwU(np.array([g4, g4]), 64, np.zeros_like(v4), v4, np.ones(2),
                                            precision=prec), xg)
    # config 4's optimiser: modified FIRE with the reference's defaults on the FP32 UwU, host-driven
    # iterations and the graph form (the whole run(niter) loop as one CUDA graph launch)
    from fresco_b200._lib import check as _check, lib as _clib
    from fresco_b200.optimize import ModifiedFire_Graph, ModifiedFireCPP

    fire = {"workload": "modified FIRE (reference defaults, tol=0) on the FP32 UwU above",
            "timing": "host wall clock around the C-level run loop"}
    n_fire = max(20, args.steps)
    for name, cls in (("ModifiedFireCPP", ModifiedFireCPP), ("ModifiedFire_Graph", ModifiedFire_Graph)):
        opt = cls(xg, UwU(np.array([g4, g4]), 64, np.zeros_like(v4), v4, np.ones(2), precision="fp32"), tol=0.0)
        opt.run(3)  # initial evaluation, graph capture, warm-up iterations
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        _check(_clib.fresco_optimizer_run(opt._h, n_fire))
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        res = opt.get_result()
        fire[name] = {"iterations_per_s": round(n_fire / dt, 2), "ms_per_iteration": round(1e3 * dt / n_fire, 4),
                      "evals": int(res.nfev), "energy": float(res.energy)}
        del opt
    out["config4_uwu_fire"] = fire
    del xg, m4, v4
    rng = np.random.default_rng(4)
    gu, mk = 2048, 100_000
    xu = rng.random(gu * gu)
    r = 512 * np.sqrt(rng.random(mk))
    t = 2 * np.pi * rng.random(mk)
    kp = (np.stack([r * np.cos(t), r * np.sin(t)], axis=1) / gu).ravel()
    sku = np.zeros(mk)
    sku[rng.choice(mk, 64, replace=False)] = float(np.sum(xu))
    out["config4_uwnu"] = {"workload": "UwNU on a 2048^2 grid against 100,000 k-points uniform in |k|<=512, "
                                       "S0 = sum(x) at 64 peaks, V=1, eps=1e-6"}
    for prec in ("fp32", "fp64"):
        out["config4_uwnu"][prec] = rate(UwNU(np.array([gu, gu]), kp, sku, np.ones(mk), np.ones(2), eps=EPS,
                                              precision=prec), xu)
    # NUwNU with many k-points: the type-3 NUFFT path (points x k-points >= 2^22 pairs)
    from fresco_b200 import NUwNU

    rng = np.random.default_rng(6)
    n6, m6 = 1 << 16, 100_000
    x6 = rng.random(2 * n6)
    k6 = ((rng.random((m6, 2)) * 2 - 1) * 64.0).ravel()
    s6 = rng.random(m6) * n6 * (rng.random(m6) < 0.3)
    out["nuwnu_type3"] = {"workload": "NUwNU, N=65536 points uniform in [0,1)^2 (L=1), 100,000 k-points uniform in "
                                      "[-64,64]^2, S0 random, V=1, type-3 NUFFT both ways"}
    for prec, eps in (("fp32", EPS), ("fp64", 1e-12)):
        pot6 = NUwNU(np.ones(n6), k6, s6, np.ones(m6), np.ones(2), eps=eps, precision=prec)
        out["nuwnu_type3"][prec] = rate(pot6, x6)
        out["nuwnu_type3"][prec]["eps"] = eps
        out["nuwnu_type3"]["setup"] = pot6.describe()
        del pot6
    x1, r1, sk1, v1, l1 = stealthy_inputs(4096, 32, 16, seed=1)
    out["config1_nuwu"] = {"workload": "2D NUwU, N=4096, 65^2 modes, S0=0 & V=1 on 0<|k|<=16, eps=1e-12",
                           "fp64": rate(NUwU(r1, 32, sk1.ravel(), v1.ravel(), l1, eps=1e-12, precision="fp64"), x1)}
    out["timing"] = "CUDA events around back-to-back evaluations on one GPU (graph replay), after 3 warm-ups"
    return out


def config2_lbfgs500_report(x, radii, Sk, V, L, n_iter=500):
    """Config 2 as stated: NUwU + harmonic repulsion (a = 2, stiffness 1, diameter 0.5/sqrt(N) 2 pi)
    minimised by LBFGS with the reference defaults (M = 4) for 500 iterations from the seeded start, in
    the FP32 spread/FFT/interpolation form and in the plain FP64 form (both at the headline's eps 1e-6),
    and in the FP64 form at eps 1e-12 (the accuracy reference).  Host wall clock around the C-level run
    loop: every iteration waits for its line-search evaluations, as the reference's does."""
    import torch

    from fresco_b200 import CombinedPotential, InversePower, NUwU
    from fresco_b200._lib import check as _check, lib as _clib
    from fresco_b200.optimize import LBFGS_CPP

    rr = np.full(len(radii), 0.25 / np.sqrt(len(radii)) * 2 * np.pi)
    out = {"workload": "config 2: the headline NUwU pattern + harmonic repulsion, LBFGS M=4 (reference "
                       "defaults), 500 iterations from the seeded start",
           "timing": "host wall clock around the C-level run loop, one GPU"}
    for name, prec, eps in (("fp32", "fp32", EPS), ("fp64", "fp64", EPS), ("fp64_eps1e-12", "fp64", 1e-12)):
        comb = CombinedPotential()
        comb.add_potential(NUwU(radii, K_MODES, Sk, V, L, eps=eps, precision=prec))
        comb.add_potential(InversePower(2.0, 1.0, rr, np.asarray(L, float), use_cell_lists=True))
        opt = LBFGS_CPP(x, comb, tol=0.0, nsteps=n_iter + 10)
        e0 = float(comb.get_energy(x))  # an optimiser that has not iterated reports 0, like the reference
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        _check(_clib.fresco_optimizer_run(opt._h, n_iter))
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        res = opt.get_result()
        out[name] = {"eps": eps, "iterations": int(res.nsteps), "evals": int(res.nfev),
                     "iterations_per_s": round(n_iter / dt, 2), "seconds": round(dt, 3),
                     "energy_initial": e0, "energy_final": float(res.energy), "rms_final": float(res.rms)}
        del opt, comb
    out["fp32_final_energy_rel_diff_vs_fp64_eps1e-12"] = abs(out["fp32"]["energy_final"] -
                                                             out["fp64_eps1e-12"]["energy_final"]) / abs(
        out["fp64_eps1e-12"]["energy_final"])
    return out


ONLY_WORKLOADS = ("nuwu2d_fp32", "nuwu2d_fp64", "repulsion", "lbfgs", "nuwu3d_fp32", "nuwu3d_fp64", "uwu_fp32",
                  "uwnu_fp32", "nuwnu_type3_fp32", "ensemble")


def run_only(args):
    """One workload of this file, evaluated --warmup + --steps times on one GPU with nothing else around it
    (the command that the ncu captures under profiles/ profile), then one line with its mean time."""
    import torch

    from fresco_b200 import CombinedPotential, InversePower, NUwNU, NUwU, UwNU, UwU
    from fresco_b200.optimize import LBFGS_CPP

    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    name = args.only
    x, radii, Sk, V, L = inputs(seed=2)
    rr = np.full(N_POINTS, 0.25 / np.sqrt(N_POINTS) * 2 * np.pi)
    if name in ("nuwu2d_fp32", "nuwu2d_fp64"):
        pot = NUwU(radii, K_MODES, Sk, V, L, eps=EPS, precision=name[-4:])
    elif name == "repulsion":
        pot = InversePower(2.0, 1.0, rr, np.asarray(L, float), use_cell_lists=True)
    elif name == "lbfgs":
        pot = CombinedPotential()
        pot.add_potential(NUwU(radii, K_MODES, Sk, V, L, eps=EPS, precision="fp32"))
        pot.add_potential(InversePower(2.0, 1.0, rr, np.asarray(L, float), use_cell_lists=True))
        opt = LBFGS_CPP(x, pot, tol=0.0)
        opt.run(args.warmup)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        opt.run(args.steps)
        torch.cuda.synchronize()
        print(json.dumps({"only": name, "ms_per_iteration": 1e3 * (time.perf_counter() - t0) / args.steps}))
        return
    elif name.startswith("nuwu3d"):
        rng = np.random.default_rng(3)
        n3, k3 = 1 << 21, 64
        x = rng.random(3 * n3) * 2 * np.pi
        kv = np.arange(-k3, k3 + 1)
        kz, ky, kx = np.meshgrid(kv, kv, kv, indexing="ij")
        mag = np.sqrt(kx ** 2 + ky ** 2 + kz ** 2).ravel().astype(np.float64)
        pot = NUwU(np.ones(n3), k3, 1.0 - np.exp(-((mag / 16.0) ** 2)), np.where(mag > 0, 1.0 / (1.0 + mag), 0.0),
                   np.full(3, 2 * np.pi), eps=EPS, precision=name[-4:])
    elif name == "uwu_fp32":
        rng = np.random.default_rng(4)
        g4 = 4096
        x = rng.random(g4 * g4)
        k = np.arange(g4) - g4 // 2
        m4 = np.sqrt(k[:, None] ** 2 + k[None, :] ** 2)
        v4 = ((m4 <= 64) & (m4 > 0)).astype(np.float64)
        pot = UwU(np.array([g4, g4]), 64, np.zeros_like(v4), v4, np.ones(2), precision="fp32")
    elif name == "uwnu_fp32":
        rng = np.random.default_rng(4)
        gu, mk = 2048, 100_000
        x = rng.random(gu * gu)
        r = 512 * np.sqrt(rng.random(mk))
        t = 2 * np.pi * rng.random(mk)
        kp = (np.stack([r * np.cos(t), r * np.sin(t)], axis=1) / gu).ravel()
        sku = np.zeros(mk)
        sku[rng.choice(mk, 64, replace=False)] = float(np.sum(x))
        pot = UwNU(np.array([gu, gu]), kp, sku, np.ones(mk), np.ones(2), eps=EPS, precision="fp32")
    elif name == "nuwnu_type3_fp32":
        rng = np.random.default_rng(6)
        n6, m6 = 1 << 16, 100_000
        x = rng.random(2 * n6)
        k6 = ((rng.random((m6, 2)) * 2 - 1) * 64.0).ravel()
        s6 = rng.random(m6) * n6 * (rng.random(m6) < 0.3)
        pot = NUwNU(np.ones(n6), k6, s6, np.ones(m6), np.ones(2), eps=EPS, precision="fp32")
    elif name == "ensemble":
        from fresco_b200 import NUwUEnsemble

        pats, Le = ensemble_inputs()
        ens = NUwUEnsemble([r for _, r, _, _, _ in pats], [K for _, _, K, _, _ in pats],
                           [s for _, _, _, s, _ in pats], [v for _, _, _, _, v in pats], Le, eps=EPS,
                           precision="fp32")
        xs = [p[0] for p in pats]
        dx = torch.tensor(ens.concat(xs), device=dev)
        dg = torch.empty_like(dx)
        de = torch.empty(ens.n_patterns, dtype=torch.float64, device=dev)
        stream = torch.cuda.current_stream(dev).cuda_stream
        for _ in range(args.warmup):
            ens.get_energies_gradient_device(dx, dg, de, stream)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            ens.get_energies_gradient_device(dx, dg, de, stream)
        torch.cuda.synchronize()
        print(json.dumps({"only": name, "ms_per_eval": 1e3 * (time.perf_counter() - t0) / args.steps}))
        return
    else:
        raise SystemExit(f"--only: unknown workload {name!r} (one of {', '.join(ONLY_WORKLOADS)})")
    xt = torch.tensor(x, device=dev)
    g = torch.empty_like(xt)
    e = torch.zeros((), dtype=torch.float64, device=dev)
    for _ in range(args.warmup):
        pot.energy_gradient_device(xt, g, e)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        pot.energy_gradient_device(xt, g, e)
    torch.cuda.synchronize()
    print(json.dumps({"only": name, "ms_per_eval": 1e3 * (time.perf_counter() - t0) / args.steps,
                      "setup": pot.describe()}))


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


class Clocks:
    """Samples nvidia-smi clocks/throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.dev = device_index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.dev}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        rows = []
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        smax = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": reasons, "samples": len(rows)}


def algorithmic_bytes(geom_nf, n_active, N, s_r, s_c, s_w, d=2, d_f=2):
    """Per-eval algorithmic bytes of the loss-and-gradient path (each array read or written once) and the
    per-stage figures: points N, fine grid G = nf^2, real/complex/weight sizes s_r, s_c, s_w."""
    G = geom_nf * geom_nf
    n_modes = (2 * K_MODES + 1) ** 2
    b_points = N * (4 * d * s_r + 12)
    b_grid = G * s_c * (3 + 4 * d_f)
    b_modes = n_modes * (s_c + 2 * s_w)
    per_kernel = {
        # read x (d doubles), write the sorted record (cell, d fractions, index)
        "sort": N * (8 * d + 4 + d * s_r + 4),
        # read the sorted record, write the real fine grid
        "spread": N * (4 + d * s_r + s_r) + G * s_r,
        # real-to-complex FFT: read G reals, write G/2 complex
        "fft_type1": G * s_r + (G // 2) * s_c,
        # active modes: read rho + coefficients (idx + 4 doubles), write the packed field
        "modes": n_active * (s_c + 4 + 32 + s_c),
        # complex FFT of the packed field
        "fft_type2": 2 * G * s_c,
        # read the sorted record and the packed grid, write the gradient
        "interp": N * (4 + d * s_r + s_r + 4 + 8 * d) + G * s_c,
    }
    return b_points + b_grid + b_modes, per_kernel


def reduce_max(value, device):
    """Max of a per-rank scalar over all ranks (the job time is the slowest rank's)."""
    import torch

    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    try:
        import torch.distributed as dist

        if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
    except ImportError:
        pass
    return float(t.item())


def reduce_sum(value, device):
    """Sum of a per-rank scalar over all ranks."""
    import torch

    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    try:
        import torch.distributed as dist

        if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
            dist.all_reduce(t, op=dist.ReduceOp.SUM)
    except ImportError:
        pass
    return float(t.item())


def job_value(world_size, steps, job_ms):
    """Whole-job throughput: every rank's steps over the slowest rank's time."""
    return world_size * steps / (job_ms / 1000.0)


def run_ours(args):
    import torch

    ws, rank, local = dist_env()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if ws > 1:
        import torch.distributed as dist
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    import fresco_b200
    from fresco_b200 import NUwU

    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    hbm_peak = float(peaks.get("hbm_gbs", 6650.0))
    peak_src = "measured" if "hbm_gbs" in peaks else "fallback"

    x, radii, Sk, V, L = inputs(seed=2 + rank)
    pot32 = NUwU(radii, K_MODES, Sk, V, L, eps=EPS, precision="fp32")
    desc = pot32.describe()
    nf = int(desc.split("nf=")[1].split("x")[0])
    n_active = int(desc.split("active_modes=")[1].split()[0])
    xt = torch.tensor(x, device=dev)
    g = torch.empty_like(xt)
    e = torch.zeros((), dtype=torch.float64, device=dev)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream(dev)

    def timed_loop(pot, steps, warmup, record_stages=False):
        for _ in range(warmup):
            pot.energy_gradient_device(xt, g, e)
        torch.cuda.synchronize()
        if ws > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()
        if record_stages:
            pot.set_timing(True)
        total = 0.0
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
        for i in range(steps):
            flush.fill_(float(i))  # write > L2 between timed steps
            evs[i][0].record(stream)
            pot.energy_gradient_device(xt, g, e)
            evs[i][1].record(stream)
        torch.cuda.synchronize()
        for a, b in evs:
            total += a.elapsed_time(b)
        if ws > 1:
            torch.distributed.barrier()
        stages = pot.get_timing() if record_stages else {}
        if record_stages:
            pot.set_timing(False)
        return total, stages

    clocks = Clocks(local)
    clocks.start()
    t32_ms, _ = timed_loop(pot32, args.steps, args.warmup)
    clk = clocks.stop()
    e32 = float(e.item())
    g32 = g.clone()
    # per-stage breakdown (CUDA events between stages; runs the launches without graph replay)
    _, stages = timed_loop(pot32, min(args.steps, 10), 1, record_stages=True)

    # slowest rank decides the job time
    t_job_ms = reduce_max(t32_ms, dev)
    ms_per_step = t_job_ms / args.steps
    value = job_value(ws, args.steps, t_job_ms)

    # FP64 form (same eps) and the FP64 reference gradient (eps = 1e-12)
    pot64 = NUwU(radii, K_MODES, Sk, V, L, eps=EPS, precision="fp64")
    t64_ms, _ = timed_loop(pot64, max(3, args.steps // 2), 2)
    ms64 = t64_ms / max(3, args.steps // 2)
    g64 = g.clone()
    # the FP32 form with the kernel width its 1e-5 gradient bound needs (eps = 1e-5: w = 6)
    pot32w = NUwU(radii, K_MODES, Sk, V, L, eps=EPS_FP32_BOUND, precision="fp32")
    t32w_ms, _ = timed_loop(pot32w, args.steps, args.warmup)
    ms32w = reduce_max(t32w_ms, dev) / args.steps
    e32w = float(e.item())
    g32w = g.clone()
    desc32w = pot32w.describe()
    del pot32w
    potref = NUwU(radii, K_MODES, Sk, V, L, eps=1e-12, precision="fp64")
    potref.energy_gradient_device(xt, g, e)
    torch.cuda.synchronize()
    eref = float(e.item())
    gref = g.clone()
    err32 = float(torch.linalg.norm(g32 - gref) / torch.linalg.norm(gref))
    err64 = float(torch.linalg.norm(g64 - gref) / torch.linalg.norm(gref))
    err32w = float(torch.linalg.norm(g32w - gref) / torch.linalg.norm(gref))
    eerr32 = abs(e32 - eref) / abs(eref)
    fp32_bound = {"eps": EPS_FP32_BOUND, "w": int(desc32w.split(" w=")[1].split()[0]),
                  "evals_per_s": round(ws * 1000.0 / ms32w, 2), "ms_per_step": round(ms32w, 5),
                  "over_fp64": round(ms64 / ms32w, 3), "grad_rel_err": err32w,
                  "energy_rel_err": abs(e32w - eref) / abs(eref),
                  "note": "FP32 form at the kernel width chosen for the 1e-5 gradient bound, against the "
                          "FP64 form at eps=1e-6 (w=7); errors against the FP64 form at eps=1e-12"}
    del potref

    # config 2's full potential: NUwU (FP32 form) + cell-list harmonic repulsion (a = 2, eps = 1,
    # diameter 0.5/sqrt(N) 2 pi), device-timed like the headline; then LBFGS (M = 4) iterations on it,
    # host-timed around the synchronous run() (each iteration waits for its line-search evaluations)
    from fresco_b200 import CombinedPotential, InversePower
    from fresco_b200.optimize import LBFGS_CPP

    rep = InversePower(2.0, 1.0, np.full(N_POINTS, 0.25 / np.sqrt(N_POINTS) * 2 * np.pi), np.asarray(L, float))
    comb = CombinedPotential()
    comb.add_potential(pot32)
    comb.add_potential(rep)
    n_comb = max(3, args.steps // 2)
    tc_ms, _ = timed_loop(comb, n_comb, 3)
    comb_evals = 1000.0 / (reduce_max(tc_ms, dev) / n_comb)
    opt = LBFGS_CPP(x, comb, M=4)
    for _ in range(3):
        opt.one_iteration()
    torch.cuda.synchronize()
    e_start = float(opt.get_result().energy)
    from fresco_b200._lib import check as _check, lib as _clib

    n_it = max(30, args.steps)
    t0 = time.perf_counter()
    _check(_clib.fresco_optimizer_run(opt._h, n_it))  # the iterations only (run() also copies the result out)
    torch.cuda.synchronize()
    lbfgs_s = reduce_max(time.perf_counter() - t0, dev)
    res = opt.get_result()
    lbfgs = {"iterations_per_s": round(n_it / lbfgs_s, 2), "evals": int(res.nfev), "iterations": int(res.nsteps),
             "energy_after_warmup": e_start, "energy": float(res.energy), "M": 4,
             "timing": "host wall clock around the C-level run loop, per GPU"}
    del opt
    # the same LBFGS with its whole iteration on the device: one CUDA graph launch per evaluation
    from fresco_b200.optimize import LBFGS_Graph

    gopt = LBFGS_Graph(x, comb, M=4)
    gopt.run(3)  # initial evaluation, graph capture, warm-up iterations
    _, _, _, _, it0, nf0, _ = gopt.state(False)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    gopt.run(n_it)
    torch.cuda.synchronize()
    graph_s = reduce_max(time.perf_counter() - t0, dev)
    _, _, f1, _, it1, nf1, _ = gopt.state(False)
    lbfgs["graph_captured"] = {"iterations_per_s": round(float(it1[0] - it0[0]) / graph_s, 2),
                               "iterations": int(it1[0] - it0[0]), "evals": int(nf1[0] - nf0[0]),
                               "energy": float(f1[0]),
                               "timing": "host wall clock around run(), graph launches, per GPU"}
    del gopt

    # end to end through the public API: page-locked host x in, page-locked host gradient out
    x_host = torch.tensor(x).pin_memory().numpy()
    g_host = torch.empty(x.size, dtype=torch.float64).pin_memory().numpy()
    for _ in range(2):
        pot32.get_energy_gradient(x_host, out=g_host)
    torch.cuda.synchronize()
    ne2e = max(5, args.steps)
    t0 = time.perf_counter()
    for _ in range(ne2e):
        eh, gh = pot32.get_energy_gradient(x_host, out=g_host)
    e2e_s = (time.perf_counter() - t0) / ne2e
    e2e_value = ws / reduce_max(e2e_s, dev)
    # the host link's own floor for this call: the same bytes copied alone (pinned, CUDA events)
    xd_link = torch.empty(x.size, dtype=torch.float64, device=dev)
    x_pin, g_pin = torch.from_numpy(x_host), torch.from_numpy(g_host)
    link = {}
    for name, dst, src in (("h2d_gbs", xd_link, x_pin), ("d2h_gbs", g_pin, xd_link)):
        for _ in range(2):
            dst.copy_(src, non_blocking=True)
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(5):
            dst.copy_(src, non_blocking=True)
        b.record(stream)
        torch.cuda.synchronize()
        link[name] = round(5 * x.nbytes / (a.elapsed_time(b) * 1e-3) / 1e9, 2)
    link_ms = x.nbytes / (link["h2d_gbs"] * 1e9) * 1e3 + (x.nbytes + 8) / (link["d2h_gbs"] * 1e9) * 1e3
    del xd_link

    # roofline: per-stage device times from CUDA events on the launch stream
    # d_f = 1: the two gradient fields are interpolated as one Hermitian-packed complex field
    b_eval, per_kernel = algorithmic_bytes(nf, n_active, N_POINTS, 4, 8, 8, d_f=1)
    stage_ms = {k: v[0] / max(v[1], 1) for k, v in stages.items()}
    top = max(stage_ms, key=stage_ms.get) if stage_ms else "spread"
    top_ms = stage_ms.get(top, ms_per_step)
    achieved = per_kernel.get(top, b_eval) / (top_ms * 1e-3) / 1e9
    traffic = None
    capture = None
    try:  # DRAM bytes per launch from an ncu capture of this workload (profiles/traffic.txt: "stage bytes")
        with open(os.path.join(ROOT, "profiles", "traffic.txt")) as fh:
            text = fh.read()
        prof = {ln.split()[0]: int(ln.split()[1]) for ln in text.splitlines() if ln.strip() and not ln.startswith("#")}
        traffic = prof.get(top)
        import re

        m = re.search(r"commit ([0-9a-f]{7,40})", text)
        capture = m.group(1) if m else None
        # a stage re-captured later is named in the header as "(<stage>: <kernel> at commit <sha>)"
        m = re.search(r"\(" + top + r": \S+ at commit ([0-9a-f]{7,40})\)", text)
        capture = m.group(1) if m else capture
    except (OSError, ValueError, IndexError):
        pass
    roofline = {"kernel": top, "bound": "hbm", "achieved": round(achieved, 1), "peak": hbm_peak, "unit": "GB/s",
                "frac": round(achieved / hbm_peak, 4), "traffic": traffic, "peak_source": peak_src,
                "algorithmic_bytes": per_kernel.get(top),
                "traffic_source": f"ncu capture at commit {capture} (profiles/traffic.txt)" if capture else None}
    try:  # the stage's own limiter: L1/shared-memory pipe use from the same kind of ncu capture
        with open(os.path.join(ROOT, "profiles", "l1tex.txt")) as fh:
            l1 = {ln.split()[0]: ln.split()[1:] for ln in fh if ln.strip() and not ln.startswith("#")}
        if top in l1:
            roofline["l1tex"] = {"frac": round(float(l1[top][0]) / 100.0, 3),
                                 "shared_wavefronts": int(l1[top][1]),
                                 "source": "ncu l1tex__throughput.avg.pct_of_peak_sustained_active "
                                           f"(profiles/l1tex.txt, capture at commit {capture})"}
    except (OSError, ValueError, IndexError):
        pass
    eval_achieved = b_eval / (ms_per_step * 1e-3) / 1e9
    roofline_eval = {"bound": "hbm", "algorithmic_bytes": b_eval, "achieved": round(eval_achieved, 1),
                     "peak": hbm_peak, "unit": "GB/s", "frac": round(eval_achieved / hbm_peak, 4)}

    lbfgs500 = None if (args.no_lbfgs500 or ws > 1) else config2_lbfgs500_report(x, radii, Sk, V, L)

    ensemble = None if args.no_ensemble else ensemble_report(args, dev, ws, rank)
    sharded = None
    if not args.no_sharded:
        try:  # an error that every rank meets alike (set-up, memory) is reported instead of ending the run
            sharded = sharded_report(args, dev, ws, rank)
        except Exception as exc:  # noqa: BLE001
            sharded = {"error": f"{type(exc).__name__}: {exc}"[:300]}
    others = None if (args.no_other_configs or ws > 1) else other_configs_report(args, dev)

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu:
        cpu = cpu_baseline(x, radii, Sk, V, L, samples=args.cpu_samples)

    # kernels of ours per eval: sort count, sort scatter, spread, band row r2c, band modes, band row c2c, interp
    launches = 7 * args.steps
    out = {
        "metric": METRIC,
        "value": round(value, 2),
        "unit": "evals/s",
        "n_gpus": ws,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(ms_per_step, 5),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic (seeded uniform points, rank r uses seed 2+r)",
        "config": {"workload": WORKLOAD, "precision": "fp32 spread/FFT/interp, fp64 loss reduction",
                   "setup": desc, "l2": "flushed between timed steps (256 MiB write)",
                   "parallelism": f"independent pattern per GPU x{ws}"},
        "e2e": {"value": round(e2e_value, 2), "unit": "evals/s", "h2d_bytes_per_step": int(x.nbytes),
                "d2h_bytes_per_step": int(x.nbytes + 8), "host_link": link,
                "copy_floor_ms": round(link_ms, 4),
                "copy_plus_device_ms": round(link_ms + ms_per_step, 4), "ms_per_step": round(1e3 / e2e_value, 4)},
        "gpu_launches": launches,
        "roofline": roofline,
        "roofline_eval": roofline_eval,
        "stages_ms": {k: round(v, 4) for k, v in stage_ms.items()},
        "fp64": {"evals_per_s": round(ws * 1000.0 / ms64, 2), "ms_per_step": round(ms64, 5),
                 "fp32_over_fp64": round(ms64 / ms_per_step, 3)},
        "fp32_width_for_bound": fp32_bound,
        "nuwu_plus_repulsion": {"evals_per_s_per_gpu": round(comb_evals, 2)},
        "lbfgs": lbfgs,
        "config2_lbfgs500": lbfgs500,
        "ensemble": ensemble,
        "sharded_pattern": sharded,
        "other_configs": others,
        "accuracy": {"grad_rel_err_fp32": err32, "grad_rel_err_fp64_eps1e-6": err64, "energy_rel_err_fp32": eerr32,
                     "oracle": "GPU FP64 form at eps=1e-12 (parity-tested against exact sums)"},
        "clocks": clk,
        "cpu_baseline": cpu,
    }
    if rank == 0:
        print(json.dumps(out), flush=True)
    del pot32, pot64
    if ws > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()


CPU_WARMUP = 3


def timed_cpu_evals(p, x, samples, warmup=CPU_WARMUP):
    """Per-evaluation wall times (s) of `samples` get_energy_gradient calls after `warmup` untimed ones."""
    for _ in range(warmup):
        p.get_energy_gradient(x)
    times = []
    for _ in range(samples):
        t0 = time.perf_counter()
        p.get_energy_gradient(x)
        times.append(time.perf_counter() - t0)
    return times


def cpu_baseline(x, radii, Sk, V, L, samples=20):
    """The reference's CPU path on this host (oracle/_ref, ES-kernel NUFFT shim, all cores): median of
    `samples` evaluations after 3 warm-ups."""
    try:
        from oracle import refimpl as R

        if not R.available():
            return {"value": None, "unit": "evals/s", "cores": 0, "kind": "reference", "sample": "oracle/_ref missing"}
        R.set_mode(R.ES)
        cores = R.host_cores()
        R.set_threads(cores)
        p = R.NUwU(radii, K_MODES, Sk, V, L, eps=EPS)
        times = timed_cpu_evals(p, x, samples)
        med = statistics.median(times)
        return {"value": round(1.0 / med, 4), "unit": "evals/s", "cores": cores, "kind": "reference",
                "sample": f"median of {samples} evals of the full workload after {CPU_WARMUP} warm-ups "
                          f"(min {min(times) * 1e3:.1f} ms, max {max(times) * 1e3:.1f} ms); reference nuwu.hpp "
                          "compiled unchanged against the FINUFFT-API shim (CPU ES-kernel NUFFT restatement, "
                          "FP64, eps=1e-6), not FINUFFT itself"}
    except Exception as ex:  # the baseline is reported, never fatal
        return {"value": None, "unit": "evals/s", "cores": 0, "kind": "reference", "sample": f"failed: {ex}"}


def run_reference(args):
    ws, rank, _ = dist_env()
    if rank != 0:
        return
    from oracle import refimpl as R

    if not R.available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libfresco_ref.so not built"}))
        return
    R.set_mode(R.ES)
    cores = R.host_cores()
    R.set_threads(cores)
    x, radii, Sk, V, L = inputs(seed=2)
    p = R.NUwU(radii, K_MODES, Sk, V, L, eps=EPS)
    warm = max(CPU_WARMUP, args.warmup)
    times = timed_cpu_evals(p, x, args.steps, warm)
    med = statistics.median(times)
    value = 1.0 / med
    sample = (f"median of {args.steps} full evals of the workload after {warm} warm-ups (mean "
              f"{1e3 * sum(times) / len(times):.1f} ms); reference nuwu.hpp compiled unchanged against the "
              f"FINUFFT-API shim: CPU ES-kernel NUFFT restatement, FP64, eps=1e-6; FINUFFT itself is not "
              f"installable here")
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": round(value, 4), "unit": "evals/s", "n_gpus": ws,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(1000 * med, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded uniform points, seed 2)",
        "config": {"workload": WORKLOAD, "precision": "fp64 (reference)", "parallelism": f"{cores} host threads"},
        "cpu_baseline": {"value": round(value, 4), "unit": "evals/s", "cores": cores, "kind": "reference",
                         "sample": sample},
        "e2e": {"value": round(value, 4), "unit": "evals/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cpu-samples", type=int, default=20)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-ensemble", action="store_true", help="skip the batched-ensemble section")
    ap.add_argument("--no-lbfgs500", action="store_true", help="skip config 2's 500-iteration LBFGS runs")
    ap.add_argument("--no-sharded", action="store_true", help="skip the sharded single-pattern section")
    ap.add_argument("--no-other-configs", action="store_true",
                    help="skip the throughput of the other configurations' potentials")
    ap.add_argument("--no-ensemble-loop", action="store_true",
                    help="skip timing the ensemble's patterns as separate potentials")
    ap.add_argument("--only", default=None, choices=ONLY_WORKLOADS,
                    help="run one workload alone (warmup + steps evaluations; the profiling command)")
    args = ap.parse_args()
    if args.warmup < 3 and args.impl == "ours":
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    elif args.only:
        run_only(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
