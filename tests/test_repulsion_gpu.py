"""Device soft-sphere repulsion against the oracle, the golden vectors and the reference's known answers."""
import os

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(np.asarray(b)), 1e-300))


@pytest.mark.parametrize("ndim", [2, 3])
def test_harmonic_golden(ndim):
    from fresco_b200 import InversePower

    d = dict(np.load(os.path.join(GOLDEN, f"harmonic_{ndim}d.npz")))
    p = InversePower(float(d["a"]), float(d["eps"]), d["radii"], d["boxv"], use_cell_lists=True)
    assert "cells=" in p.describe()
    e, g = p.get_energy_gradient(d["x"])
    assert rel(e, d["energy"]) < 1e-12
    assert rel(g, d["grad"]) < 1e-12
    assert rel(p.get_energy(d["x"]), d["energy"]) < 1e-12


def test_known_answers_small_box():
    """cpp_tests/source/test_inversepower.cpp:41-42: three particles, pow 2.5 (all-pairs path)."""
    from fresco_b200 import InversePower
    from fresco_b200.potentials import Distance

    x = np.array([0.1, 0.2, 0.3, 0.44, 0.55, 1.66, 0.88, 1.1, 3.32])
    radii = np.array([0.91, 1.1, 1.13])
    per = InversePower(2.5, 1.0, radii, np.ones(3), method=Distance.PERIODIC)
    cart = InversePower(2.5, 1.0, radii, np.ones(3), method=Distance.CARTESIAN)
    assert abs(per.get_energy(x) - 0.60660574285698954) < 1e-10
    assert abs(cart.get_energy(x) - 0.023173380132354017) < 1e-10
    for pot, ref in [(per, O.InversePower(2.5, 1.0, radii, np.ones(3), method="periodic")),
                     (cart, O.InversePower(2.5, 1.0, radii, np.ones(3), method="cartesian"))]:
        e, g = pot.get_energy_gradient(x)
        e0, g0 = ref.get_energy_gradient(x)
        assert abs(e - e0) < 1e-12
        assert rel(g, g0) < 1e-12


@pytest.mark.parametrize("N,box,a,equal", [(5000, 20.0, 2.0, False), (3000, 12.0, 2.5, False), (200, 2.0, 2.0, False),
                                           (20000, 40.0, 2.0, True), (4096, 3.0, 2.0, True)])
def test_random_configurations(N, box, a, equal):
    """Polydisperse radii (gathered per pair) and equal radii (one value), dense and dilute."""
    from fresco_b200 import InversePower

    rng = np.random.default_rng(N)
    x = rng.random(2 * N) * box * 1.5 - 0.25 * box  # some points outside the box
    radii = np.full(N, 0.17) if equal else 0.2 * (0.7 + 0.6 * rng.random(N))
    if equal and box < 10:
        radii = np.full(N, 0.25 / np.sqrt(N) * box)  # the benchmark's packing
    p = InversePower(a, 1.0, radii, np.full(2, box), use_cell_lists=True)
    e, g = p.get_energy_gradient(x)
    e0, g0 = O.InversePower(a, 1.0, radii, np.full(2, box)).get_energy_gradient(x)
    assert rel(e, e0) < 1e-12
    assert rel(g, g0) < 1e-12


def test_nonfinite_gives_nan():
    from fresco_b200 import InversePower

    rng = np.random.default_rng(1)
    x = rng.random(2000) * 10
    p = InversePower(2.0, 1.0, np.full(1000, 0.2), np.full(2, 10.0), use_cell_lists=True)
    x[0] = np.inf
    e, g = p.get_energy_gradient(x)
    assert np.isnan(e) and np.all(np.isnan(g))
    assert p.status() & 1
    x[0] = 1.0
    e, g = p.get_energy_gradient(x)
    assert np.isfinite(e) and p.status() == 0


def test_combined_nuwu_plus_repulsion():
    from fresco_b200 import CombinedPotential, InversePower, NUwU

    d = dict(np.load(os.path.join(GOLDEN, "lbfgs_combined_2d.npz")))
    nu = NUwU(d["radii"], float(d["K"]), d["Sk"], d["V"], d["L"], eps=1e-13)
    rep = InversePower(2.0, 1.0, d["rep_radii"], d["L"], use_cell_lists=True)
    comb = CombinedPotential()
    comb.add_potential(nu)
    comb.add_potential(rep)
    e, g = comb.get_energy_gradient(d["x"])
    assert rel(e, d["energy0"]) < 1e-10
    assert rel(g, d["grad0"]) < 1e-10
    assert rel(comb.get_energy(d["x"]), d["energy0"]) < 1e-10
