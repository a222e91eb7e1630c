"""NUwU on the device against the oracle (exact FP64 direct sums of the reference's formulas)."""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

# (precision, eps, relative tolerance on energy and on the gradient's 2-norm)
PRECISIONS = [("fp64", 1e-12, 1e-10), ("fp32", 1e-6, 1e-5)]


def _inputs(ndim, N, K, kmax, seed, L=None, random_weights=False, radii_spread=True):
    x, radii, Sk, V, L = O.stealthy_nuwu_inputs(N, K, kmax, ndim=ndim, seed=seed, L=L)
    rng = np.random.default_rng(seed + 100)
    if radii_spread:
        radii = 0.5 + rng.random(N)
    if random_weights:
        V = rng.random(V.shape) * (rng.random(V.shape) < 0.7)
        Sk = rng.random(Sk.shape) * 2.0 * (rng.random(Sk.shape) < 0.5)
    return x, radii, Sk, V, L


def _check(pot, ref, x, tol):
    e_ref, g_ref = ref.get_energy_gradient(x)
    e, g = pot.get_energy_gradient(x)
    assert abs(e - e_ref) <= tol * abs(e_ref), (e, e_ref)
    err = np.linalg.norm(g - g_ref) / np.linalg.norm(g_ref)
    assert err <= tol, err
    e2 = pot.get_energy(x)
    assert abs(e2 - ref.get_energy(x)) <= tol * abs(e_ref)
    assert pot.status() == 0


@pytest.mark.parametrize("prec,eps,tol", PRECISIONS)
# K = 3 gives 14-cell fine grids at w = 7, not a multiple of four cells: the FP32 spreads fall back
# from the thread-per-point kernels to the phased 2D and warp-per-point 3D kernels
@pytest.mark.parametrize("ndim,N,K,kmax", [(2, 400, 10, 8), (3, 150, 4, 3), (1, 120, 24, 18), (2, 300, 3, 3),
                                           (3, 200, 3, 2)])
def test_nuwu_stealthy(prec, eps, tol, ndim, N, K, kmax):
    from fresco_b200 import NUwU

    x, radii, Sk, V, L = _inputs(ndim, N, K, kmax, seed=ndim)
    ref = O.NUwU(radii, K, Sk, V, L)
    pot = NUwU(radii, K, Sk, V, L, eps=eps, precision=prec)
    _check(pot, ref, x, tol)


@pytest.mark.parametrize("prec,eps,tol", PRECISIONS)
@pytest.mark.parametrize("ndim", [2, 3])
def test_nuwu_asymmetric_targets(prec, eps, tol, ndim):
    """V and S0 with no k <-> -k symmetry and S0 != 0 entries (exercises the Hermitian packing)."""
    from fresco_b200 import NUwU

    N, K = (300, 7) if ndim == 2 else (120, 3)
    x, radii, Sk, V, L = _inputs(ndim, N, K, K, seed=11 + ndim, random_weights=True)
    ref = O.NUwU(radii, K, Sk, V, L)
    pot = NUwU(radii, K, Sk, V, L, eps=eps, precision=prec)
    _check(pot, ref, x, tol)


@pytest.mark.parametrize("prec,eps,tol", PRECISIONS)
@pytest.mark.parametrize("K,kmax,random_weights,band", [(128, 80, False, True), (128, 100, True, True),
                                                        (64, 40, True, False), (128, 128, True, False)])
def test_nuwu_2d_band_transforms(prec, eps, tol, K, kmax, random_weights, band):
    """Power-of-two fine grids of 512 and more take the band transforms (register FFTs over
    |k_x| <= kmax); a 256 grid, or a band as wide as the grid allows, falls back to the cuFFT passes."""
    from fresco_b200 import NUwU

    N = 1500
    x, radii, Sk, V, L = _inputs(2, N, K, kmax, seed=K + kmax, random_weights=random_weights)
    if random_weights:  # keep the asymmetric targets inside the band
        n = 2 * K + 1
        k = np.arange(n) - K
        inside = (np.abs(k)[None, :] <= kmax) & (np.abs(k)[:, None] <= kmax)
        V = np.where(inside.reshape(V.shape), V, 0.0)
    ref = O.NUwU(radii, K, Sk, V, L)
    pot = NUwU(radii, K, Sk, V, L, eps=eps, precision=prec)
    assert ("fft=band" in pot.describe()) == band, pot.describe()
    _check(pot, ref, x, tol)


@pytest.mark.parametrize("prec,eps,tol", PRECISIONS)
def test_nuwu_2d_clustered_points_wide_weights(prec, eps, tol):
    """Most points in one corner of the box, so their bins hold several subproblems (at most 640
    points each) that add to the same fine-grid cells, with weights spanning about four decades
    (radii 0.05..3): the FP32 spread accumulates each subproblem in fixed point scaled by its own
    largest weight."""
    from fresco_b200 import NUwU

    N = 6000
    x, _, Sk, V, L = _inputs(2, N, 64, 40, seed=31, random_weights=True)
    rng = np.random.default_rng(31)
    pts = rng.random((N, 2)) * np.asarray(L)[None, :]
    pts[:4500] = pts[:4500] * 0.06  # 4500 points in a square of side 0.06 L: a few 64-cell bins
    x = pts.ravel()
    radii = 0.05 + 2.95 * rng.random(N) ** 3
    ref = O.NUwU(radii, 64, Sk, V, L)
    pot = NUwU(radii, 64, Sk, V, L, eps=eps, precision=prec)
    _check(pot, ref, x, tol)


@pytest.mark.parametrize("prec,eps,tol", PRECISIONS)
def test_nuwu_3d_clustered_points_wide_weights(prec, eps, tol):
    """The 3D form of the clustered test: 3000 of 4000 points in a corner cube of side 0.1 L (bins
    split into several subproblems on a 32^3 fine grid of 16 x 16 x 8-cell tiles), radii 0.05..3."""
    from fresco_b200 import NUwU

    N = 4000
    _, _, Sk, V, L = _inputs(3, N, 8, 6, seed=32, random_weights=True)
    rng = np.random.default_rng(32)
    pts = rng.random((N, 3)) * np.asarray(L)[None, :]
    pts[:3000] = pts[:3000] * 0.1
    radii = 0.05 + 2.95 * rng.random(N) ** 3
    ref = O.NUwU(radii, 8, Sk, V, L)
    pot = NUwU(radii, 8, Sk, V, L, eps=eps, precision=prec)
    _check(pot, ref, pts.ravel(), tol)


@pytest.mark.parametrize("L", [1.0, 2 * np.pi, 3.7])
def test_nuwu_box_map_quirk(L):
    """Points inside and outside the box under the reference's coordinate map (nuwu.hpp:216-250)."""
    from fresco_b200 import NUwU

    rng = np.random.default_rng(5)
    N, K = 200, 6
    x, radii, Sk, V, Lv = _inputs(2, N, K, 5, seed=5, L=np.full(2, L))
    x = x + rng.normal(scale=L, size=x.shape)  # points far outside [0, L)
    ref = O.NUwU(radii, K, Sk, V, Lv)
    pot = NUwU(radii, K, Sk, V, Lv, eps=1e-12)
    _check(pot, ref, x, 1e-10)


def test_nuwu_nonfinite_input():
    from fresco_b200 import NUwU

    x, radii, Sk, V, L = _inputs(2, 50, 4, 3, seed=9)
    pot = NUwU(radii, 4, Sk, V, L)
    x[7] = np.nan
    e, g = pot.get_energy_gradient(x)
    assert np.isnan(e) and np.all(np.isnan(g))
    assert pot.status() & 1
    x[7] = 0.3
    e, g = pot.get_energy_gradient(x)
    assert np.isfinite(e) and np.all(np.isfinite(g))
    assert pot.status() == 0


def test_nuwu_no_active_modes_and_empty_weights():
    from fresco_b200 import NUwU

    x, radii, Sk, V, L = _inputs(2, 30, 3, 2, seed=4)
    pot = NUwU(radii, 3, Sk, np.zeros_like(V), L)
    e, g = pot.get_energy_gradient(x)
    assert e == 0.0 and np.all(g == 0.0)


def test_nuwu_device_path_matches_host_path():
    import torch

    from fresco_b200 import NUwU

    x, radii, Sk, V, L = _inputs(2, 500, 12, 10, seed=3)
    pot = NUwU(radii, 12, Sk, V, L, eps=1e-10)
    e_h, g_h = pot.get_energy_gradient(x)
    xt = torch.tensor(x, device="cuda")
    e_d, g_d = pot.energy_gradient_device(xt)
    torch.cuda.synchronize()
    assert abs(e_d.item() - e_h) <= 1e-12 * abs(e_h)
    assert np.allclose(g_d.cpu().numpy(), g_h, rtol=1e-11, atol=1e-11 * np.abs(g_h).max())


def test_nuwu_bad_arguments():
    from fresco_b200 import NUwU

    x, radii, Sk, V, L = _inputs(2, 20, 3, 2, seed=1)
    with pytest.raises(AssertionError):
        NUwU(radii, 3, Sk[:-1], V, L)
    pot = NUwU(radii, 3, Sk, V, L)
    with pytest.raises(ValueError):
        pot.get_energy_gradient(x[:-1])
    with pytest.raises(ValueError):
        NUwU(radii, 3, Sk, V, L, precision="fp16")


@pytest.mark.parametrize("prec", ["fp32", "fp64"])
def test_nuwu_graph_replay_follows_buffer_contents(prec):
    """Repeated calls on the same buffers are replayed as a CUDA graph (captured at the second call); the
    replay must read the buffers' current contents, exactly as a direct evaluation does."""
    import torch

    from fresco_b200 import CombinedPotential, InversePower, NUwU

    N, K, kmax = 3000, 24, 10
    # spreading sums in a run-dependent order, so repeated evaluations agree to rounding only
    tol = 1e-5 if prec == "fp32" else 1e-11
    x0, radii, Sk, V, L = O.stealthy_nuwu_inputs(N, K, kmax, ndim=2, seed=11)
    rng = np.random.default_rng(3)
    pot = NUwU(radii, K, Sk, V, L, precision=prec)
    xt = torch.tensor(x0, device="cuda")
    g = torch.empty_like(xt)
    e = torch.zeros((), dtype=torch.float64, device="cuda")
    for it in range(5):
        xi = x0 + 0.01 * it * rng.standard_normal(x0.size)
        xt.copy_(torch.from_numpy(xi))
        pot.energy_gradient_device(xt, g, e)
        torch.cuda.synchronize()
        fresh = NUwU(radii, K, Sk, V, L, precision=prec)  # first call: direct launches
        e0, g0 = fresh.get_energy_gradient(xi)
        assert float(e.item()) == pytest.approx(e0, rel=tol), it
        np.testing.assert_allclose(g.cpu().numpy(), g0, rtol=0, atol=tol * np.abs(g0).max())

    # a combined potential replays all its parts
    box = np.array([2 * np.pi, 2 * np.pi])
    rep = InversePower(2.0, 1.0, 0.02 * np.ones(N), box)
    comb = CombinedPotential()
    comb.add_potential(pot)
    comb.add_potential(rep)
    for it in range(4):
        xi = x0 + 0.02 * it
        xt.copy_(torch.from_numpy(xi))
        comb.energy_gradient_device(xt, g, e)
        torch.cuda.synchronize()
        e_parts = NUwU(radii, K, Sk, V, L, precision=prec).get_energy_gradient(xi)[0]
        e_parts += InversePower(2.0, 1.0, 0.02 * np.ones(N), box).get_energy_gradient(xi)[0]
        assert float(e.item()) == pytest.approx(e_parts, rel=tol), it


@pytest.mark.parametrize("prec,eps,tol", PRECISIONS)
def test_interp_tile_copy_second_wait(prec, eps, tol):
    """With a first wait of zero polls every interior tile copy of the 2D interpolation outlasts it: the
    blocks raise status bit 8 (retry), wait again bounded by time, see the copy land and finish.  The
    results equal the default setting's and the oracle's; no timeout (bit 4) is raised."""
    from fresco_b200 import NUwU
    from fresco_b200._lib import check, lib

    K, kmax = 128, 80  # 512^2 fine grid: 64 tiles, 36 of them interior (copied by TMA)
    x, radii, Sk, V, L = _inputs(2, 20000, K, kmax, seed=21, radii_spread=False)
    ref = O.NUwU(radii, K, Sk, V, L)
    e_ref, g_ref = ref.get_energy_gradient(x)
    e0, g0 = NUwU(radii, K, Sk, V, L, eps=eps, precision=prec).get_energy_gradient(x)
    check(lib.fresco_debug_set_tile_wait_polls(0))
    try:
        pot = NUwU(radii, K, Sk, V, L, eps=eps, precision=prec)  # captures its graphs with the new setting
        results = [pot.get_energy_gradient(x) for _ in range(3)]  # direct launches, capture, replay
        st = pot.status()
    finally:
        check(lib.fresco_debug_set_tile_wait_polls(-1))
    assert st & 8 and not st & 4, st
    for e1, g1 in results:
        assert abs(e1 - e0) <= tol * abs(e0) and abs(e1 - e_ref) <= tol * abs(e_ref)
        assert np.linalg.norm(g1 - g0) <= tol * np.linalg.norm(g0)
        assert np.linalg.norm(g1 - g_ref) <= tol * np.linalg.norm(g_ref)
    after = NUwU(radii, K, Sk, V, L, eps=eps, precision=prec)
    after.get_energy_gradient(x)
    assert after.status() == 0


def test_interp3d_tile_copies_and_second_wait():
    """3D FP32: interior tiles of both fields arrive by tensor copies (the complex x/y field by a 4D
    copy while the block classifies its points, the real z field by a 3D copy after the first
    field's sums).  With the default first wait and
    with a first wait of zero polls (status bit 8: every copy waited for a second time), the results
    equal the oracle's; no timeout (bit 4) is raised."""
    from fresco_b200 import NUwU
    from fresco_b200._lib import check, lib

    K, kmax = 16, 8  # 64^3 fine grid of 16 x 16 x 8 tiles: interior tiles take the copies
    x, radii, Sk, V, L = _inputs(3, 4000, K, kmax, seed=22, radii_spread=False)
    e_ref, g_ref = O.NUwU(radii, K, Sk, V, L).get_energy_gradient(x)
    for polls in (-1, 0):
        check(lib.fresco_debug_set_tile_wait_polls(polls))
        try:
            pot = NUwU(radii, K, Sk, V, L, eps=1e-6, precision="fp32")
            results = [pot.get_energy_gradient(x) for _ in range(3)]  # direct launches, capture, replay
            st = pot.status()
        finally:
            check(lib.fresco_debug_set_tile_wait_polls(-1))
        assert not st & 4, st
        assert bool(st & 8) == (polls == 0), st
        for e1, g1 in results:
            assert abs(e1 - e_ref) <= 1e-5 * abs(e_ref)
            assert np.linalg.norm(g1 - g_ref) <= 1e-5 * np.linalg.norm(g_ref)


def test_objects_of_different_sizes_interleave():
    """A kernel's shared-memory limit is shared by every object that launches it: a smaller object
    made later must not lower it under a larger one (one-pass sorts of 800K and 500K points, and the
    LBFGS two-loop kernels of their 1.6M and 1M coordinates, interleaved)."""
    from fresco_b200 import NUwU
    from fresco_b200.optimize import LBFGS_CPP

    pots, xs = [], []
    for n in (800_000, 500_000):
        x, radii, Sk, V, L = O.stealthy_nuwu_inputs(n, 16, 8, ndim=2, seed=n % 97)
        pots.append(NUwU(radii, 16, Sk, V, L, eps=1e-6, precision="fp32"))
        xs.append(x)
    e_big = pots[0].get_energy_gradient(xs[0])[0]
    e_small = pots[1].get_energy_gradient(xs[1])[0]
    assert np.isfinite(e_small)
    assert abs(pots[0].get_energy_gradient(xs[0])[0] - e_big) <= 1e-6 * abs(e_big)
    opts = [LBFGS_CPP(x, p, M=4) for x, p in zip(xs, pots)]
    for _ in range(2):
        for o in opts:
            o.one_iteration()
    assert all(np.isfinite(o.get_result().energy) for o in opts)


@pytest.mark.parametrize("prec,eps,tol", PRECISIONS)
@pytest.mark.parametrize("ndim", [2, 3])
def test_nuwu_rare_heavy_points(prec, eps, tol, ndim):
    """A few points of radius ten times the others (weights about 10^4 (2D) or 10^6 (3D) times
    larger) scattered among many light ones, so that most subproblems hold one heavy point: the
    light points' contributions must not be quantised at the heavy point's scale."""
    from fresco_b200 import NUwU

    N, K, kmax = (20000, 64, 40) if ndim == 2 else (12000, 12, 8)
    _, _, Sk, V, L = _inputs(ndim, N, K, kmax, seed=40 + ndim, random_weights=True)
    rng = np.random.default_rng(40 + ndim)
    x = (rng.random((N, ndim)) * np.asarray(L)[None, :]).ravel()
    radii = np.full(N, 0.1)
    radii[rng.choice(N, N // 500, replace=False)] = 1.0
    ref = O.NUwU(radii, K, Sk, V, L)
    pot = NUwU(radii, K, Sk, V, L, eps=eps, precision=prec)
    _check(pot, ref, x, tol)
