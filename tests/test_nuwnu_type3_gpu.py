"""NUwNU through the type-3 NUFFT (many k-points) against exact sums.

The reference evaluates NUwNU with FINUFFT type 3 in both directions (source/fresco/nuwnu.hpp:77-78,
165-166, 231-282).  The device uses a type-3 NUFFT when points x k-points reach 2^22 pairs, and exact
direct sums below that.  The oracle here is the reference's own nuwnu.hpp compiled in oracle/_ref
against exact direct sums (or the numpy restatement when that build is absent); the tolerances are
those of the other parity tests: 1e-10 for FP64 at eps 1e-12, 1e-5 for FP32 at eps 1e-6."""
import numpy as np
import pytest

from oracle import oracle as O
from oracle import refimpl as R

pytestmark = pytest.mark.gpu

PRECISIONS = [("fp64", 1e-12, 1e-10), ("fp32", 1e-6, 1e-5)]


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(np.asarray(b)), 1e-300))


def _inputs(ndim, N, M, kmax, seed, L=1.0):
    rng = np.random.default_rng(seed)
    Lv = np.full(ndim, float(L))
    x = (rng.random((N, ndim)) * Lv).ravel()
    radii = 0.5 + rng.random(N)
    K = ((rng.random((M, ndim)) * 2 - 1) * kmax).ravel()
    Sk = rng.random(M) * N * (rng.random(M) < 0.3)
    V = rng.random(M)
    return x, radii, K, Sk, V, Lv


def _reference(radii, K, Sk, V, L):
    if R.available():
        R.set_mode(R.EXACT)
        R.set_threads(R.host_cores())
        return R.NUwNU(radii, K, Sk, V, L, eps=1e-12)
    return O.NUwNU(radii, K, Sk, V, L)


@pytest.fixture(scope="module")
def case2d():
    x, radii, K, Sk, V, L = _inputs(2, 2000, 100_000, 60.0, seed=3)
    e_ref, g_ref = _reference(radii, K, Sk, V, L).get_energy_gradient(x)
    return x, radii, K, Sk, V, L, e_ref, g_ref


@pytest.mark.parametrize("prec,eps,tol", PRECISIONS)
def test_type3_2d_1e5_kpoints(case2d, prec, eps, tol):
    """2D, N = 2000 points, M = 10^5 k-points uniform in [-60, 60]^2, S0 and V random."""
    from fresco_b200 import NUwNU

    x, radii, K, Sk, V, L, e_ref, g_ref = case2d
    pot = NUwNU(radii, K, Sk, V, L, eps=eps, precision=prec)
    assert "type3" in pot.describe()
    for _ in range(3):  # direct launches, graph capture, graph replay
        e, g = pot.get_energy_gradient(x)
        assert abs(e - e_ref) <= tol * abs(e_ref), (e, e_ref)
        assert rel(g, g_ref) <= tol
    assert abs(pot.get_energy(x) - e_ref) <= tol * abs(e_ref)
    assert pot.status() == 0  # in particular not 16: the type-3 path served every evaluation


@pytest.mark.parametrize("prec,eps,tol", PRECISIONS)
@pytest.mark.parametrize("ndim,N,M,kmax,L", [(1, 3000, 4000, 400.0, 0.8), (3, 600, 20000, 12.0, 1.3)])
def test_type3_1d_3d(prec, eps, tol, ndim, N, M, kmax, L):
    from fresco_b200 import NUwNU

    x, radii, K, Sk, V, Lv = _inputs(ndim, N, M, kmax, seed=ndim + 10, L=L)
    e_ref, g_ref = _reference(radii, K, Sk, V, Lv).get_energy_gradient(x)
    pot = NUwNU(radii, K, Sk, V, Lv, eps=eps, precision=prec)
    assert "type3" in pot.describe()
    e, g = pot.get_energy_gradient(x)
    assert abs(e - e_ref) <= tol * abs(e_ref), (e, e_ref)
    assert rel(g, g_ref) <= tol
    assert pot.status() == 0  # the type-3 path, not the exact fallback (status bit 16)


def test_type3_exact_gradient_mode(case2d):
    """The exact-derivative convention (c_j 2 pi / L times the reference's value) through type 3."""
    from fresco_b200 import NUwNU

    x, radii, K, Sk, V, L, e_ref, g_ref = case2d
    pot = NUwNU(radii, K, Sk, V, L, eps=1e-12)
    pot.set_gradient_mode("exact")
    _, g = pot.get_energy_gradient(x)
    c = O.point_weights(radii, 2)
    assert rel(g, g_ref * np.repeat(c, 2) * 2 * np.pi / L[0]) < 1e-10


@pytest.mark.parametrize("L,fallback_far", [(1.3, True), (1.0, False)])
def test_type3_points_outside_the_plans_window_use_exact_sums(L, fallback_far):
    """The reference's map x = (p - round(p/L) + L) 2 pi / L drifts by 2 pi (L - 1) / L per box a point
    moves away (none for L = 1).  Points more than a box length outside the box are then beyond the plans'
    window: that evaluation runs the exact sums (status bit 16), with the same results.  A NaN
    coordinate gives a NaN energy."""
    from fresco_b200 import NUwNU

    x, radii, K, Sk, V, Lv = _inputs(2, 1200, 5000, 30.0, seed=7, L=L)
    pot = NUwNU(radii, K, Sk, V, Lv, eps=1e-12)
    assert "type3" in pot.describe()
    ref = _reference(radii, K, Sk, V, Lv)
    far = x.copy()
    far[::7] += 5.0 * L  # five boxes away
    for pts, fallback in ((x, False), (far, fallback_far), (x, False)):
        e_ref, g_ref = ref.get_energy_gradient(pts)
        e, g = pot.get_energy_gradient(pts)
        assert abs(e - e_ref) <= 1e-10 * abs(e_ref)
        assert rel(g, g_ref) <= 1e-10
        assert bool(pot.status() & 16) == fallback
    bad = x.copy()
    bad[5] = np.nan
    e, g = pot.get_energy_gradient(bad)
    assert np.isnan(e) and np.isnan(g).all()
    assert pot.status() & 1
    e, _ = pot.get_energy_gradient(x)
    assert np.isfinite(e)
