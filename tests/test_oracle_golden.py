"""The numpy oracle against golden vectors produced by the reference's own C++ (CPU only)."""
import os

import numpy as np
import pytest

from oracle import oracle as O

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load(name):
    return dict(np.load(os.path.join(GOLDEN, name + ".npz")))


def rel(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.mark.parametrize("name", ["nuwu_2d_n4096", "nuwu_2d_asym", "nuwu_3d_radial"])
def test_nuwu_golden(name):
    d = load(name)
    p = O.NUwU(d["radii"], float(d["K"]), d["Sk"], d["V"], d["L"])
    e, g = p.get_energy_gradient(d["x"])
    assert rel(e, d["energy"]) < 1e-12
    assert rel(g, d["grad"]) < 1e-12
    assert rel(p.get_energy(d["x"]), d["energy_only"]) < 1e-12


def test_uwu_golden():
    d = load("uwu_2d")
    p = O.UwU(d["N"], 6, d["Sk"], d["V"], d["L"])
    e, g = p.get_energy_gradient(d["x"])
    assert rel(e, d["energy"]) < 1e-12
    assert rel(g, d["grad"]) < 1e-12
    assert rel(p.get_energy(d["x"]), d["energy_only"]) < 1e-12


def test_uwnu_golden():
    d = load("uwnu_2d")
    p = O.UwNU(d["N"], d["K"], d["Sk"], d["V"], d["L"])
    e, g = p.get_energy_gradient(d["x"])
    assert rel(e, d["energy"]) < 1e-12
    assert rel(g, d["grad"]) < 1e-12


def test_nuwnu_golden():
    d = load("nuwnu_2d")
    p = O.NUwNU(d["radii"], d["K"], d["Sk"], d["V"], d["L"])
    e, g = p.get_energy_gradient(d["x"])
    assert rel(e, d["energy"]) < 1e-12
    assert rel(g, d["grad"]) < 1e-11
    assert rel(p.get_energy(d["x"]), d["energy_only"]) < 1e-12


@pytest.mark.parametrize("ndim", [2, 3])
def test_harmonic_golden(ndim):
    d = load(f"harmonic_{ndim}d")
    p = O.InversePower(float(d["a"]), float(d["eps"]), d["radii"], d["boxv"])
    e, g = p.get_energy_gradient(d["x"])
    assert rel(e, d["energy"]) < 1e-12
    assert rel(g, d["grad"]) < 1e-12


def test_inversepower_known_answers():
    """cpp_tests/source/test_inversepower.cpp:23-42 (pow 2.5, three particles)."""
    x = np.array([0.1, 0.2, 0.3, 0.44, 0.55, 1.66, 0.88, 1.1, 3.32])
    radii = np.array([0.91, 1.1, 1.13])
    per = O.InversePower(2.5, 1.0, radii, np.ones(3), method="periodic")
    cart = O.InversePower(2.5, 1.0, radii, np.ones(3), method="cartesian")
    assert abs(per.get_energy(x) - 0.60660574285698954) < 1e-10
    assert abs(cart.get_energy(x) - 0.023173380132354017) < 1e-10
    for pot in (per, cart):
        e, g = pot.get_energy_gradient(x)
        h = 1e-6
        for i in range(6):
            xp, xm = x.copy(), x.copy()
            xp[i] += h
            xm[i] -= h
            assert abs((pot.get_energy(xp) - pot.get_energy(xm)) / (2 * h) - g[i]) < 1e-6


def test_lbfgs_trajectory_golden():
    d = load("lbfgs_combined_2d")
    nu = O.NUwU(d["radii"], float(d["K"]), d["Sk"], d["V"], d["L"])
    rep = O.InversePower(2.0, 1.0, d["rep_radii"], d["L"])
    comb = O.CombinedPotential()
    comb.add_potential(nu)
    comb.add_potential(rep)
    e0, g0 = comb.get_energy_gradient(d["x"])
    assert rel(e0, d["energy0"]) < 1e-12 and rel(g0, d["grad0"]) < 1e-12
    opt = O.LBFGS(d["x"], comb, tol=1e-12, M=10)
    for i in range(len(d["traj_energy"])):
        opt.one_iteration()
        assert rel(opt.f, d["traj_energy"][i]) < 1e-9, i
        assert opt.nfev == d["traj_nfev"][i]
    assert rel(opt.x, d["x_final"]) < 1e-9
    assert rel(opt.H0, d["H0"]) < 1e-7


def test_fire_trajectory_golden():
    d = load("fire_uwu_2d")
    p = O.UwU(d["N"], 3, d["Sk"], d["V"], d["L"])
    opt = O.ModifiedFire(d["x"], p)
    for i in range(len(d["traj_energy"])):
        opt.run(1)
        assert rel(opt.f, d["traj_energy"][i]) < 1e-10, i
        assert rel(opt.rms, d["traj_rms"][i]) < 1e-10, i
    assert rel(opt.x, d["x_final"]) < 1e-10
    assert opt.nfev == int(d["nfev"])


def test_fire_one_iteration_without_run_keeps_zero_state():
    """The reference FIRE steps from f = 0, g = 0 when one_iteration() precedes run()."""
    d = load("fire_uwu_2d")
    p = O.UwU(d["N"], 3, d["Sk"], d["V"], d["L"])
    opt = O.ModifiedFire(d["x"], p)
    for _ in range(3):
        opt.one_iteration()
    assert opt.f == 0.0 and opt.rms == 1e10 and opt.nfev == 3
    assert np.array_equal(opt.x, d["x"])


def test_radial_profile_small_case():
    """The oracle's radial_profile against a hand count (centre at index shape/2, R = shape/2).  The
    reference drops its last bin, meant to be the one beyond R: on a 4 x 4 grid no cell lies beyond R,
    so the last real bin (r = 2) is dropped; on 8 x 8 the corners lie beyond R and r = 0..4 remain."""
    for n, kept in [(4, 2), (8, 5)]:
        data = np.arange(float(n * n)).reshape(n, n)
        q, prof = O.radial_profile(data, center=[n // 2, n // 2])
        idx = np.indices((n, n))
        r = np.sqrt((idx[0] - n // 2) ** 2 + (idx[1] - n // 2) ** 2).astype(int)
        expect = [data[r == k].mean() for k in range(kept)]
        np.testing.assert_array_equal(q, np.arange(kept))
        np.testing.assert_allclose(prof, expect)


def test_active_mode_sums_equal_full_sums():
    """The oracle's active-mode NUwU/UwNU sums (used at full sizes) equal its full exact sums when V is
    sparse, and the k-d tree pair search gives the O(N^2) repulsion."""
    rng = np.random.default_rng(21)
    for ndim, N, K in [(2, 300, 9), (3, 120, 3)]:
        x, radii, Sk, V, L = O.stealthy_nuwu_inputs(N, K, K, ndim=ndim, seed=ndim)
        radii = 0.5 + rng.random(N)
        V = V * (rng.random(V.shape) < 0.2) * rng.random(V.shape)
        Sk = rng.random(V.shape) * (rng.random(V.shape) < 0.5)
        ref = O.NUwU(radii, K, Sk, V, L)
        e, g = ref.get_energy_gradient(x)
        ea, ga = ref.get_energy_gradient_active(x, chunk=77)
        assert abs(ea - e) <= 1e-12 * abs(e)
        assert np.linalg.norm(ga - g) <= 1e-12 * np.linalg.norm(g)
    shape = np.array([12, 10])
    M = 40
    Kp = rng.random(M * 2) * 4 - 2
    V = rng.random(M) * (rng.random(M) < 0.5)
    Sk = rng.random(M) * (rng.random(M) < 0.5)
    grid = rng.random(int(np.prod(shape)))
    ref = O.UwNU(shape, Kp, Sk, V, np.array([1.0, 1.3]))
    e, g = ref.get_energy_gradient(grid)
    ea, ga = ref.get_energy_gradient_active(grid)
    assert abs(ea - e) <= 1e-12 * abs(e)
    assert np.linalg.norm(ga - g) <= 1e-12 * np.linalg.norm(g)
    for ndim in (2, 3):
        box = np.full(ndim, 2.0)
        pts = rng.random(300 * ndim) * 2.0
        rad = 0.08 + 0.04 * rng.random(300)
        ip = O.InversePower(2.0, 1.0, rad, box, use_cell_lists=True)
        e, g = ip.get_energy_gradient(pts)
        et, gt = ip.get_energy_gradient_tree(pts)
        assert e > 0 and abs(et - e) <= 1e-12 * e
        assert np.linalg.norm(gt - g) <= 1e-12 * np.linalg.norm(g)
