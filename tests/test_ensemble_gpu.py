"""Batched NUwU ensembles against the single-pattern potentials, the oracle's exact sums and the
single-pattern LBFGS (whose own parity with the reference's lbfgs.cpp is tested in test_optimize_gpu.py)."""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

# (N, K, kmax, polydisperse radii): mixed point counts and mode grids, several patterns per grid
SPECS = [(40, 8, 4, False), (3000, 8, 5, True), (700, 16, 8, False), (20000, 16, 6, False), (5000, 32, 12, True),
         (150, 32, 10, False), (9000, 4, 2, False), (60000, 64, 20, False),
         # 512^2 and 1024^2 fine grids: the batched band transforms (per-pattern active bands differ)
         (4000, 128, 30, False), (500, 128, 16, True), (30000, 256, 64, False), (2000, 256, 40, False)]


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(np.asarray(b)), 1e-300))


def patterns(specs, L, seed=0):
    xs, radii, Ks, Sks, Vs = [], [], [], [], []
    for i, (N, K, kmax, poly) in enumerate(specs):
        x, r, Sk, V, _ = O.stealthy_nuwu_inputs(N, K, kmax, ndim=2, seed=seed + i, L=L)
        if poly:
            r = 0.5 + np.random.default_rng(seed + 100 + i).random(N)
        xs.append(x)
        radii.append(r)
        Ks.append(K)
        Sks.append(Sk.ravel())
        Vs.append(V.ravel())
    return xs, radii, Ks, Sks, Vs


@pytest.mark.parametrize("precision,eps,tol", [("fp64", 1e-12, 1e-10), ("fp32", 1e-6, 2e-5)])
@pytest.mark.parametrize("split", [0.0, 1e30, "tune", 160, 320])
def test_ensemble_matches_single_patterns(precision, eps, tol, split):
    """Every pattern's energy and gradient equal the single-pattern NUwU (FP64 at eps 1e-12 as the
    reference value), with all patterns tiled, all direct, the tuned split and subproblem size, and
    all patterns tiled in subproblems of at most 160 or 320 points (an int split)."""
    from fresco_b200 import NUwU, NUwUEnsemble

    L = np.full(2, 2 * np.pi)
    xs, radii, Ks, Sks, Vs = patterns(SPECS, L, seed=3)
    ens = NUwUEnsemble(radii, Ks, Sks, Vs, L, eps=eps, precision=precision)
    assert ens.describe().count("fft=band") == 2, ens.describe()
    if split == "tune":
        ens.tune(xs)
        assert "subproblem<=" in ens.describe()
    elif isinstance(split, int):
        ens.set_split(0.0)
        ens.set_subproblem_cap(split)
        assert ens.describe().count(f"subproblem<={split}") == ens.describe().count("[")
    else:
        ens.set_split(split)
    e, g = ens.get_energies_gradient(xs)
    e_only = ens.get_energies(xs)
    for p in range(len(SPECS)):
        ref = NUwU(radii[p], Ks[p], Sks[p], Vs[p], L, eps=1e-12)
        e0, g0 = ref.get_energy_gradient(xs[p])
        gp = ens.split(g)[p]
        assert abs(e[p] - e0) <= tol * abs(e0), (p, e[p], e0)
        assert abs(e_only[p] - e0) <= tol * abs(e0), p
        assert rel(gp, g0) < tol, (p, rel(gp, g0))
    # repeated calls replay a captured graph and give the same numbers
    e2, g2 = ens.get_energies_gradient(xs)
    e3, g3 = ens.get_energies_gradient(xs)
    assert rel(e3, e) < 1e-6 and rel(g3, g) < 1e-5
    assert np.all(np.isfinite(e2)) and np.all(ens.status() == 0)


def test_ensemble_against_exact_sums():
    """Small patterns against the oracle's exact FP64 direct sums (nuwu.hpp formulas)."""
    from fresco_b200 import NUwUEnsemble

    L = np.ones(2)
    specs = [(60, 6, 3, False), (250, 6, 4, True), (120, 10, 5, False)]
    xs, radii, Ks, Sks, Vs = patterns(specs, L, seed=11)
    ens = NUwUEnsemble(radii, Ks, Sks, Vs, L, eps=1e-12)
    e, g = ens.get_energies_gradient(xs)
    for p in range(len(specs)):
        e0, g0 = O.NUwU(radii[p], Ks[p], Sks[p], Vs[p], L).get_energy_gradient(xs[p])
        assert abs(e[p] - e0) <= 1e-10 * abs(e0)
        assert rel(ens.split(g)[p], g0) < 1e-10


def test_ensemble_device_buffers_and_layout_errors():
    import torch

    from fresco_b200 import NUwUEnsemble

    L = np.ones(2)
    xs, radii, Ks, Sks, Vs = patterns(SPECS[:4], L, seed=5)
    ens = NUwUEnsemble(radii, Ks, Sks, Vs, L, eps=1e-6, precision="fp32")
    e, g = ens.get_energies_gradient(xs)
    dx = torch.from_numpy(ens.concat(xs)).cuda()
    dg = torch.empty_like(dx)
    de = torch.empty(ens.n_patterns, dtype=torch.float64, device="cuda")
    for _ in range(3):  # direct, captured, replayed
        ens.get_energies_gradient_device(dx, dg, de, torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    assert rel(de.cpu().numpy(), e) < 1e-6
    assert rel(dg.cpu().numpy(), g) < 1e-5
    with pytest.raises(ValueError):
        ens.set_subproblem_cap(100)
    with pytest.raises(ValueError):
        ens.get_energies_gradient(np.zeros(ens.ndof + 2))
    with pytest.raises(ValueError):
        NUwUEnsemble([np.ones(3)], 2, [np.zeros(25)], [np.ones(25)], np.ones(3))  # 3D box


def test_nonfinite_pattern_is_isolated():
    from fresco_b200 import NUwUEnsemble

    L = np.ones(2)
    xs, radii, Ks, Sks, Vs = patterns(SPECS[:5], L, seed=7)
    ens = NUwUEnsemble(radii, Ks, Sks, Vs, L, eps=1e-9)
    e_ok, g_ok = ens.get_energies_gradient(xs)
    bad = [x.copy() for x in xs]
    bad[2][5] = np.nan
    e, g = ens.get_energies_gradient(bad)
    st = ens.status()
    assert np.isnan(e[2]) and np.all(np.isnan(ens.split(g)[2]))
    assert st[2] & 1 and st[0] == 0 and st[1] == 0
    for p in [0, 1, 3, 4]:
        assert abs(e[p] - e_ok[p]) <= 1e-12 * abs(e_ok[p])
        assert rel(ens.split(g)[p], ens.split(g_ok)[p]) < 1e-12
    e, _ = ens.get_energies_gradient(xs)
    assert np.all(np.isfinite(e))


@pytest.mark.parametrize("kw", [dict(), dict(maxstep=0.5, maxErise=1e-12), dict(maxstep=0.05, rel_energy=True,
                                                                              maxErise=1e-9)])
def test_ensemble_lbfgs_matches_single_lbfgs(kw):
    """Per pattern, run(niter) gives the trajectory of LBFGS_CPP(x0_p, NUwU_p).run(niter): same
    iterations and evaluations, coordinates and energy within 1e-8."""
    from fresco_b200 import EnsembleLBFGS, NUwU, NUwUEnsemble
    from fresco_b200.optimize import LBFGS_CPP

    L = np.ones(2)
    specs = [(300, 8, 4, False), (1200, 8, 5, True), (500, 16, 7, False), (80, 4, 2, False)]
    xs, radii, Ks, Sks, Vs = patterns(specs, L, seed=21)
    ens = NUwUEnsemble(radii, Ks, Sks, Vs, L, eps=1e-12)
    opt = EnsembleLBFGS(xs, ens, M=4, tol=1e-10, **kw)
    used = opt.run(12)
    res = opt.get_results()
    # run() is one graph launch whose loop checks the patterns after every step: it stops with the
    # last pattern, whose evaluations are its initial one plus one per step
    assert used == max(r.nfev for r in res) - 1
    for p in range(len(specs)):
        single = LBFGS_CPP(xs[p], NUwU(radii[p], Ks[p], Sks[p], Vs[p], L, eps=1e-12), M=4, tol=1e-10, **kw)
        single.run(12)
        r0 = single.get_result()
        assert res[p].nsteps == r0.nsteps, p
        assert res[p].nfev == r0.nfev, p
        assert abs(res[p].energy - r0.energy) <= 1e-8 * abs(r0.energy), p
        assert rel(res[p].coords, r0.coords) < 1e-8, p
        assert rel(res[p].grad, r0.grad) < 1e-6, p
    # a second run continues every pattern
    opt.run(3)
    assert all(r.nsteps == 15 or r.success for r in opt.get_results())


def test_ensemble_lbfgs_fp32_decreases_every_loss():
    """A config-5-like mix in FP32: tuned split, fixed step count, every loss goes down."""
    from fresco_b200 import EnsembleLBFGS, NUwUEnsemble

    rng = np.random.default_rng(5)
    L = np.ones(2)
    specs = []
    for _ in range(12):
        side = int(rng.choice([64, 128]))
        specs.append((int(np.exp(rng.uniform(np.log(1000), np.log(20000)))), side // 2, side // 8, False))
    xs, radii, Ks, Sks, Vs = patterns(specs, L, seed=40)
    ens = NUwUEnsemble(radii, Ks, Sks, Vs, L, eps=1e-6, precision="fp32")
    ens.tune(xs)
    e0 = ens.get_energies(xs)
    opt = EnsembleLBFGS(xs, ens, M=4, tol=1e-12)
    opt.steps(10)
    res = opt.get_results()
    for p, r in enumerate(res):
        assert r.energy < e0[p], (p, r.energy, e0[p])
        assert 1 <= r.nsteps <= 10 and r.nfev == 11
