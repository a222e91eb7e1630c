"""UwNU and NUwNU on the device against golden vectors (reference C++) and the oracle."""
import os

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(np.asarray(b)), 1e-300))


@pytest.mark.parametrize("prec,eps,tol", [("fp64", 1e-12, 1e-10), ("fp32", 1e-6, 1e-5)])
def test_uwnu_golden(prec, eps, tol):
    from fresco_b200 import UwNU

    d = dict(np.load(os.path.join(GOLDEN, "uwnu_2d.npz")))
    p = UwNU(d["N"], d["K"], d["Sk"], d["V"], d["L"], eps=eps, precision=prec)
    e, g = p.get_energy_gradient(d["x"])
    assert rel(e, d["energy"]) < tol
    assert rel(g, d["grad"]) < tol
    assert rel(p.get_energy(d["x"]), d["energy"]) < tol


@pytest.mark.parametrize("shape,nk,kmax", [((48,), 30, 10.0), ((31, 40), 80, 9.0), ((12, 10, 14), 40, 3.0)])
def test_uwnu_shapes(shape, nk, kmax):
    from fresco_b200 import UwNU

    rng = np.random.default_rng(nk)
    ndim = len(shape)
    x = rng.random(int(np.prod(shape)))
    L = 0.5 + rng.random(ndim)
    K = (rng.random((nk, ndim)) - 0.5) * 2 * kmax / np.asarray(shape) * L  # |k~| up to ~ kmax cycles
    Sk = rng.random(nk) * (rng.random(nk) < 0.5) * 10
    V = rng.random(nk)
    ref = O.UwNU(np.array(shape), K, Sk, V, L)
    e0, g0 = ref.get_energy_gradient(x)
    for prec, eps, tol in [("fp64", 1e-12, 1e-10), ("fp32", 1e-6, 2e-5)]:
        p = UwNU(np.array(shape), K, Sk, V, L, eps=eps, precision=prec)
        e, g = p.get_energy_gradient(x)
        assert rel(e, e0) < tol, prec
        assert rel(g, g0) < tol, prec


def test_nuwnu_golden():
    from fresco_b200 import NUwNU

    d = dict(np.load(os.path.join(GOLDEN, "nuwnu_2d.npz")))
    p = NUwNU(d["radii"], d["K"], d["Sk"], d["V"], d["L"])
    e, g = p.get_energy_gradient(d["x"])
    assert rel(e, d["energy"]) < 1e-12
    assert rel(g, d["grad"]) < 1e-11
    assert rel(p.get_energy(d["x"]), d["energy_only"]) < 1e-12


@pytest.mark.parametrize("ndim,N,nk", [(1, 500, 7), (2, 3000, 40), (3, 2000, 600)])
def test_nuwnu_random(ndim, N, nk):
    from fresco_b200 import NUwNU

    rng = np.random.default_rng(ndim)
    x = rng.random(ndim * N) * 1.4 - 0.2
    radii = 0.5 + rng.random(N)
    K = (rng.random(nk * ndim) - 0.5) * 60
    Sk = rng.random(nk) * N * (rng.random(nk) < 0.5)
    V = rng.random(nk)
    L = 0.7 + rng.random(ndim)
    ref = O.NUwNU(radii, K, Sk, V, L)
    e0, g0 = ref.get_energy_gradient(x)
    p = NUwNU(radii, K, Sk, V, L)
    e, g = p.get_energy_gradient(x)
    assert rel(e, e0) < 1e-11
    assert rel(g, g0) < 1e-10
