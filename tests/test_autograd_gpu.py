"""torch.autograd path: device adjoint vs central finite differences and vs the reference gradient."""
import os

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _fd(f, x, idx, h):
    out = []
    for i in idx:
        xp, xm = x.copy(), x.copy()
        xp[i] += h
        xm[i] -= h
        out.append((f(xp) - f(xm)) / (2 * h))
    return np.array(out)


def _autograd(pot, x):
    import torch

    from fresco_b200.autograd import structure_factor_loss

    xt = torch.tensor(x, device="cuda", requires_grad=True)
    e = structure_factor_loss(pot, xt)
    e.backward()
    return float(e.item()), xt.grad.cpu().numpy()


def _away_from_map_jumps(x, L, rng, n):
    """Coordinates whose FD stencil does not cross the reference map's jumps at p = L/2 (mod L)."""
    ndim = len(L)
    ok = [i for i in range(x.size) if abs(((x[i] / L[i % ndim]) % 1.0) - 0.5) > 1e-3]
    return rng.choice(ok, n, replace=False)


def test_nuwu_3d_radial_fd_and_reference():
    """3D NUwU with S0 = 1 - exp(-(|k|/2)^2), V = 1/(1+|k|) (config-3 shape at a CPU-checkable size):
    autograd vs central differences (h = 1e-4, 64 random coordinates) and vs the reference gradient."""
    from fresco_b200 import NUwU

    d = dict(np.load(os.path.join(GOLDEN, "nuwu_3d_radial.npz")))
    pot = NUwU(d["radii"], float(d["K"]), d["Sk"], d["V"], d["L"], eps=1e-12)
    e, g = _autograd(pot, d["x"])
    assert abs(e - float(d["energy"])) <= 1e-10 * abs(float(d["energy"]))
    # L = 2 pi: the exact derivative coincides with the reference C++ gradient
    assert np.linalg.norm(g - d["grad"]) <= 1e-10 * np.linalg.norm(d["grad"])
    rng = np.random.default_rng(0)
    idx = _away_from_map_jumps(d["x"], d["L"], rng, 64)
    fd = _fd(pot.get_energy, d["x"], idx, 1e-4)
    assert np.max(np.abs(fd - g[idx])) <= 1e-5 * np.max(np.abs(g))


@pytest.mark.parametrize("L", [1.0, 2.7])
def test_nuwu_exact_mode_scales_reference(L):
    from fresco_b200 import NUwU

    x, radii, Sk, V, Lv = O.stealthy_nuwu_inputs(400, 7, 5, ndim=2, seed=4, L=np.full(2, L))
    pot = NUwU(radii, 7, Sk, V, Lv, eps=1e-12)
    e_ref, g_ref = pot.get_energy_gradient(x)
    e, g = _autograd(pot, x)
    assert pot.gradient_mode() == "reference"
    assert abs(e - e_ref) <= 1e-13 * abs(e_ref)
    np.testing.assert_allclose(g, g_ref * 2 * np.pi / L, rtol=1e-12, atol=1e-12 * np.abs(g).max())
    rng = np.random.default_rng(1)
    idx = _away_from_map_jumps(x, Lv, rng, 32)
    fd = _fd(pot.get_energy, x, idx, 1e-6 * L)
    assert np.max(np.abs(fd - g[idx])) <= 2e-5 * np.max(np.abs(g))


def test_uwu_exact_gradient_fd():
    from fresco_b200 import UwU

    rng = np.random.default_rng(3)
    shape = (14, 11)
    x = rng.random(shape).ravel()
    Sk = rng.random(shape)
    V = rng.random(shape)
    pot = UwU(np.array(shape), 3, Sk, V, np.ones(2))
    e, g = _autograd(pot, x)
    fd = _fd(pot.get_energy, x, range(x.size), 1e-6)
    assert np.max(np.abs(fd - g)) <= 1e-6 * np.max(np.abs(g))
    _, g_ref = pot.get_energy_gradient(x)
    assert np.linalg.norm(g - g_ref) > 1e-3 * np.linalg.norm(g)  # the reference formula differs (uwu.hpp:178)


def test_uwnu_exact_gradient_fd():
    from fresco_b200 import UwNU

    d = dict(np.load(os.path.join(GOLDEN, "uwnu_2d.npz")))
    pot = UwNU(d["N"], d["K"], d["Sk"], d["V"], d["L"], eps=1e-12)
    e, g = _autograd(pot, d["x"])
    np.testing.assert_allclose(g, d["grad"] * 2 * np.pi, rtol=1e-9, atol=1e-9 * np.abs(g).max())
    idx = np.random.default_rng(5).choice(d["x"].size, 32, replace=False)
    fd = _fd(pot.get_energy, d["x"], idx, 1e-6)
    assert np.max(np.abs(fd - g[idx])) <= 1e-6 * np.max(np.abs(g))


def test_nuwnu_exact_gradient_fd():
    from fresco_b200 import NUwNU

    d = dict(np.load(os.path.join(GOLDEN, "nuwnu_2d.npz")))
    pot = NUwNU(d["radii"], d["K"], d["Sk"], d["V"], d["L"])
    e, g = _autograd(pot, d["x"])
    rng = np.random.default_rng(6)
    idx = _away_from_map_jumps(d["x"], d["L"], rng, 32)
    fd = _fd(pot.get_energy, d["x"], idx, 1e-7)
    assert np.max(np.abs(fd - g[idx])) <= 1e-5 * np.max(np.abs(g))
    # the reference gradient omits c_j and the 2 pi / L factor (nuwnu.hpp:269)
    c = O.point_weights(d["radii"], 2)
    np.testing.assert_allclose(g, d["grad"] * np.repeat(c, 2) * 2 * np.pi, rtol=1e-9, atol=1e-12)


def test_autograd_composes_with_torch_terms():
    import torch

    from fresco_b200 import NUwU
    from fresco_b200.autograd import structure_factor_loss

    x, radii, Sk, V, L = O.stealthy_nuwu_inputs(300, 6, 4, ndim=2, seed=7)
    pot = NUwU(radii, 6, Sk, V, L, eps=1e-12)
    xt = torch.tensor(x, device="cuda", requires_grad=True)
    loss = 3.0 * structure_factor_loss(pot, xt) + (xt ** 2).sum()
    loss.backward()
    _, g = pot.get_energy_gradient(x)
    np.testing.assert_allclose(xt.grad.cpu().numpy(), 3.0 * g + 2 * x, rtol=1e-11, atol=1e-9)
