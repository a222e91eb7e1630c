"""Generates the golden fixtures in tests/golden/ from the reference's own C++.

Run in a checkout where the reference tree is available::

    make -C oracle REF=<reference root>
    python tests/golden/make_golden.py

Every value comes from ``oracle/_ref/libfresco_ref.so``: the reference's
source/fresco/{nuwu,uwu,uwnu,nuwnu}.hpp, inversepower_potential.hpp + cell
lists, combine_potentials.hpp, source/lbfgs.cpp and source/modified_fire.cpp
compiled unchanged, with every transform evaluated as an exact FP64 direct
sum (the shim's EXACT mode), i.e. the reference's arithmetic with FINUFFT's
error removed.  Inputs are seeded and stored next to the outputs.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import oracle as O  # noqa: E402
from oracle import refimpl as R  # noqa: E402


def save(name, **arrays):
    path = os.path.join(HERE, name + ".npz")
    np.savez_compressed(path, **arrays)
    print(name, {k: np.asarray(v).shape for k, v in arrays.items()})


def kgrid(K, ndim):
    kv = np.arange(-K, K + 1)
    grids = np.meshgrid(*([kv] * ndim), indexing="ij")
    return np.sqrt(sum(g.astype(np.float64) ** 2 for g in grids))


def main():
    R.set_mode(R.EXACT)
    R.set_threads(min(8, os.cpu_count() or 1))

    # NUwU 2D at the CPU-runnable size: N=4096 uniform in [0, 2pi)^2, 65x65
    # modes (K=32), S0=0 on 0<|k|<=16.
    x, radii, Sk, V, L = O.stealthy_nuwu_inputs(4096, 32, 16, ndim=2, seed=1)
    p = R.NUwU(radii, 32, Sk, V, L)
    e, g = p.get_energy_gradient(x)
    save("nuwu_2d_n4096", x=x, radii=radii, K=32, Sk=Sk, V=V, L=L, energy=e, energy_only=p.get_energy(x), grad=g)

    # NUwU 2D, non-uniform radii, random asymmetric targets, L = 1 (example convention)
    rng = np.random.default_rng(7)
    N, K = 700, 10
    x = rng.random(2 * N) * 1.3 - 0.15
    radii = 0.5 + rng.random(N)
    V = rng.random((2 * K + 1) ** 2) * (rng.random((2 * K + 1) ** 2) < 0.6)
    Sk = rng.random((2 * K + 1) ** 2) * (rng.random((2 * K + 1) ** 2) < 0.5)
    L = np.ones(2)
    p = R.NUwU(radii, K, Sk, V, L)
    e, g = p.get_energy_gradient(x)
    save("nuwu_2d_asym", x=x, radii=radii, K=K, Sk=Sk, V=V, L=L, energy=e, energy_only=p.get_energy(x), grad=g)

    # NUwU 3D with the smooth radial target S0 = 1 - exp(-(|k|/2)^2), V = 1/(1+|k|), V(0) = 0
    rng = np.random.default_rng(3)
    N, K = 600, 4
    x = rng.random(3 * N) * 2 * np.pi
    km = kgrid(K, 3)
    Sk = (1.0 - np.exp(-((km / 2.0) ** 2))).ravel()
    V = (1.0 / (1.0 + km)).ravel()
    V[km.ravel() == 0] = 0.0
    radii = np.ones(N)
    L = np.full(3, 2 * np.pi)
    p = R.NUwU(radii, K, Sk, V, L)
    e, g = p.get_energy_gradient(x)
    save("nuwu_3d_radial", x=x, radii=radii, K=K, Sk=Sk, V=V, L=L, energy=e, energy_only=p.get_energy(x), grad=g)

    # UwU 2D: intensity grid 32x24 in [0,1], S0 = 0 on |k|<=6, V(0) = 0 (centred layout).
    # One OpenMP thread: the reference sums rhotot inside an unsynchronised
    # `omp parallel for` (uwu.hpp:128-133, 158-163), a data race with more threads.
    R.set_threads(1)
    rng = np.random.default_rng(4)
    shape = (32, 24)
    xg = rng.random(shape)
    ky = np.fft.fftshift(np.fft.fftfreq(shape[0], 1.0 / shape[0]))
    kx = np.fft.fftshift(np.fft.fftfreq(shape[1], 1.0 / shape[1]))
    km = np.sqrt(ky[:, None] ** 2 + kx[None, :] ** 2)
    V = (km <= 6).astype(np.float64)
    V[km == 0] = 0.0
    Sk = np.zeros(shape)
    p = R.UwU(np.array(shape), 6, Sk, V, np.ones(2))
    e, g = p.get_energy_gradient(xg.ravel())
    save("uwu_2d", x=xg.ravel(), N=np.array(shape), Sk=Sk, V=V, L=np.ones(2), energy=e,
         energy_only=p.get_energy(xg.ravel()), grad=g)

    R.set_threads(min(8, os.cpu_count() or 1))

    # UwNU 2D: 32x32 grid, 60 k-points uniform in the disc |k| <= 8 cycles, K = k/32 with L = 1,
    # S0 = sum(x0) at 4 peaks, 0 elsewhere
    rng = np.random.default_rng(5)
    shape = (32, 32)
    xg = rng.random(shape).ravel()
    nk = 60
    r = 8.0 * np.sqrt(rng.random(nk))
    th = rng.random(nk) * 2 * np.pi
    kpts = np.stack([r * np.cos(th), r * np.sin(th)], axis=1) / 32.0
    Sk = np.zeros(nk)
    Sk[rng.choice(nk, 4, replace=False)] = xg.sum()
    V = np.ones(nk)
    p = R.UwNU(np.array(shape), kpts, Sk, V, np.ones(2))
    e, g = p.get_energy_gradient(xg)
    save("uwnu_2d", x=xg, N=np.array(shape), K=kpts.ravel(), Sk=Sk, V=V, L=np.ones(2), energy=e, grad=g)

    # NUwNU 2D: 1500 points, 5 peaks at |k| = 40 (examples/NUwNU.ipynb layout), non-uniform radii
    rng = np.random.default_rng(6)
    N = 1500
    x = rng.random(2 * N)
    th = np.arange(5) / 5 * np.pi
    kpts = np.stack([np.cos(th), np.sin(th)], axis=1) * 40.0
    Sk = np.ones(5) * N
    V = np.ones(5)
    radii = 0.8 + 0.4 * rng.random(N)
    p = R.NUwNU(radii, kpts.ravel(), Sk, V, np.ones(2))
    e, g = p.get_energy_gradient(x)
    save("nuwnu_2d", x=x, radii=radii, K=kpts.ravel(), Sk=Sk, V=V, L=np.ones(2), energy=e,
         energy_only=p.get_energy(x), grad=g)

    # Harmonic repulsion (a=2) with cell lists, 2D and 3D, periodic box
    R.set_threads(1)
    for ndim, N, box, rad in [(2, 2000, 10.0, 0.12), (3, 1500, 6.0, 0.25)]:
        rng = np.random.default_rng(10 + ndim)
        x = rng.random(ndim * N) * box
        radii = rad * (0.8 + 0.4 * rng.random(N))
        p = R.InversePower(2.0, 1.0, radii, np.full(ndim, box), use_cell_lists=True, ncellx_scale=1.0)
        e, g = p.get_energy_gradient(x)
        save(f"harmonic_{ndim}d", x=x, radii=radii, boxv=np.full(ndim, box), a=2.0, eps=1.0, energy=e, grad=g)

    # Combined: NUwU + harmonic repulsion, then 15 LBFGS iterations (M=10) of the reference optimiser
    R.set_threads(min(8, os.cpu_count() or 1))
    x, radii, Sk, V, L = O.stealthy_nuwu_inputs(256, 8, 5, ndim=2, seed=12)
    rep_radii = np.full(256, 0.5 / np.sqrt(256) * 2 * np.pi / 2)
    nu = R.NUwU(radii, 8, Sk, V, L)
    R.set_threads(1)
    rep = R.InversePower(2.0, 1.0, rep_radii, L, use_cell_lists=True, ncellx_scale=1.0)
    comb = R.CombinedPotential()
    comb.add_potential(nu)
    comb.add_potential(rep)
    e0, g0 = comb.get_energy_gradient(x)
    opt = R.LBFGS(x, comb, tol=1e-12, M=10)
    traj_e, traj_rms, traj_nfev = [], [], []
    for _ in range(15):
        opt.one_iteration()
        st = opt.state()
        traj_e.append(st["energy"])
        traj_rms.append(st["rms"])
        traj_nfev.append(st["nfev"])
    st = opt.state()
    save("lbfgs_combined_2d", x=x, radii=radii, rep_radii=rep_radii, K=8, Sk=Sk, V=V, L=L, energy0=e0, grad0=g0,
         traj_energy=np.array(traj_e), traj_rms=np.array(traj_rms), traj_nfev=np.array(traj_nfev),
         x_final=st["coords"], H0=st["H0"])

    # FIRE on UwU (12x12 grid), 25 iterations with the reference defaults (one
    # thread, see the UwU race above)
    R.set_threads(1)
    rng = np.random.default_rng(13)
    shape = (12, 12)
    xg = rng.random(shape).ravel()
    kv = np.fft.fftshift(np.fft.fftfreq(12, 1.0 / 12))
    km = np.sqrt(kv[:, None] ** 2 + kv[None, :] ** 2)
    V = (km <= 3).astype(np.float64)
    V[km == 0] = 0
    Sk = np.zeros(shape)
    pu = R.UwU(np.array(shape), 3, Sk, V, np.ones(2))
    fire = R.ModifiedFire(xg, pu)
    traj_e, traj_rms = [], []
    for _ in range(25):
        fire.run(1)  # run() initialises f and g first; one_iteration() alone does not (modified_fire.hpp:160-178)
        st = fire.state()
        traj_e.append(st["energy"])
        traj_rms.append(st["rms"])
    st = fire.state()
    save("fire_uwu_2d", x=xg, N=np.array(shape), Sk=Sk, V=V, L=np.ones(2), traj_energy=np.array(traj_e),
         traj_rms=np.array(traj_rms), x_final=st["coords"], nfev=st["nfev"])


if __name__ == "__main__":
    main()
