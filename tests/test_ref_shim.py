"""The reference's C++ built against the FINUFFT/FFTW shim (oracle/_ref): exact mode reproduces the
golden vectors it generated, and the ES-kernel NUFFT restatement meets its tolerance (CPU only)."""
import numpy as np
import pytest

from oracle import oracle as O
from oracle import refimpl as R

pytestmark = pytest.mark.skipif(not R.available(), reason="oracle/_ref not built")


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b)))


@pytest.mark.parametrize("ndim,N,K", [(1, 2000, 60), (2, 3000, 24), (3, 1500, 8)])
@pytest.mark.parametrize("eps,tol", [(1e-6, 5e-6), (1e-12, 1e-10)])
def test_es_nufft_meets_tolerance(ndim, N, K, eps, tol):
    x, radii, Sk, V, L = O.stealthy_nuwu_inputs(N, K, K - 2, ndim=ndim, seed=ndim + 20)
    R.set_mode(R.EXACT)
    e0, g0 = R.NUwU(radii, K, Sk, V, L, eps=eps).get_energy_gradient(x)
    R.set_mode(R.ES)
    try:
        e1, g1 = R.NUwU(radii, K, Sk, V, L, eps=eps).get_energy_gradient(x)
    finally:
        R.set_mode(R.AUTO)
    assert abs(e1 - e0) <= tol * abs(e0)
    assert rel(g1, g0) <= tol


def test_exact_mode_matches_oracle_uwu_fft_sizes():
    """Odd and composite grid sizes through the FFTW shim (mixed radix, generic prime radices)."""
    rng = np.random.default_rng(2)
    R.set_mode(R.EXACT)
    R.set_threads(1)  # uwu.hpp:158-163 sums rhotot racily under OpenMP
    for shape in [(21, 14), (25, 49), (16, 13)]:
        xg = rng.random(shape).ravel()
        Sk = rng.random(shape)
        V = rng.random(shape)
        a = O.UwU(np.array(shape), 3, Sk, V, np.ones(2))
        b = R.UwU(np.array(shape), 3, Sk, V, np.ones(2))
        ea, ga = a.get_energy_gradient(xg)
        eb, gb = b.get_energy_gradient(xg)
        assert abs(ea - eb) <= 1e-12 * abs(ea)
        assert rel(gb, ga) <= 1e-12
