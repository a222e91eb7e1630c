"""UwU on the device against the golden vectors (reference C++) and the oracle; FIRE on UwU."""
import os

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(np.asarray(b)), 1e-300))


@pytest.mark.parametrize("prec,tol", [("fp64", 1e-12), ("fp32", 1e-5)])
def test_uwu_golden(prec, tol):
    from fresco_b200 import UwU

    d = dict(np.load(os.path.join(GOLDEN, "uwu_2d.npz")))
    p = UwU(d["N"], 6, d["Sk"], d["V"], d["L"], precision=prec)
    e, g = p.get_energy_gradient(d["x"])
    assert rel(e, d["energy"]) < tol
    assert rel(g, d["grad"]) < tol
    assert rel(p.get_energy(d["x"]), d["energy_only"]) < tol


@pytest.mark.parametrize("shape", [(21, 14), (25, 49), (16, 13), (64,), (7, 9, 10), (8, 8, 8)])
def test_uwu_shapes_random_targets(shape):
    from fresco_b200 import UwU

    rng = np.random.default_rng(sum(shape))
    x = rng.random(shape).ravel()
    Sk = rng.random(shape) * (rng.random(shape) < 0.6)
    V = rng.random(shape) * (rng.random(shape) < 0.7)
    ref = O.UwU(np.array(shape), 3, Sk, V, np.ones(len(shape)))
    e0, g0 = ref.get_energy_gradient(x)
    for prec, tol in [("fp64", 1e-11), ("fp32", 2e-5)]:
        p = UwU(np.array(shape), 3, Sk, V, np.ones(len(shape)), precision=prec)
        e, g = p.get_energy_gradient(x)
        assert rel(e, e0) < tol, prec
        assert rel(g, g0) < tol, prec


def test_fire_uwu_golden_trajectory():
    from fresco_b200 import UwU
    from fresco_b200.optimize import ModifiedFireCPP

    d = dict(np.load(os.path.join(GOLDEN, "fire_uwu_2d.npz")))
    p = UwU(d["N"], 3, d["Sk"], d["V"], d["L"])
    opt = ModifiedFireCPP(d["x"], p)
    for i in range(len(d["traj_energy"])):
        opt.run(1)
        r = opt.get_result()
        assert rel(r.energy, d["traj_energy"][i]) < 1e-10, i
        assert rel(r.rms, d["traj_rms"][i]) < 1e-10, i
    r = opt.get_result()
    assert rel(r.coords, d["x_final"]) < 1e-10
    assert r.nfev == int(d["nfev"])


@pytest.mark.parametrize("N,kb", [(512, 40), (1024, 100)])
def test_uwu_band_transforms(N, kb):
    """N x N grids (N a power of two >= 512) with the active entries in a narrow band of the
    half spectrum take the band kernels (register FFTs reading and writing the FP64 arrays):
    asymmetric targets against the oracle's FFTs, accumulation, the exact gradient mode, and a
    non-finite intensity."""
    import torch

    from fresco_b200 import CombinedPotential, UwU
    from fresco_b200.autograd import structure_factor_loss

    rng = np.random.default_rng(N + kb)
    x = rng.random(N * N)
    k = np.fft.fftshift(np.fft.fftfreq(N, 1.0 / N))  # centred layout, as the reference's Python layer takes it
    inside = (np.abs(k)[:, None] <= kb) & (np.abs(k)[None, :] <= kb)
    Sk = np.where(inside & (rng.random((N, N)) < 0.5), 1e-3 + 1e-3 * rng.random((N, N)), 0.0)
    V = np.where(inside & (rng.random((N, N)) < 0.7), rng.random((N, N)), 0.0)
    V[N // 2, N // 2] = 0.0
    ref = O.UwU(np.array([N, N]), kb, Sk, V, np.ones(2))
    e0, g0 = ref.get_energy_gradient(x)
    for prec, tol in [("fp64", 1e-10), ("fp32", 1e-5)]:
        p = UwU(np.array([N, N]), kb, Sk, V, np.ones(2), precision=prec)
        assert "fft=band" in p.describe(), p.describe()
        e, g = p.get_energy_gradient(x)
        assert rel(e, e0) < tol, prec
        assert rel(g, g0) < tol, prec
        assert rel(p.get_energy(x), e0) < tol, prec
        assert p.status() == 0
    # accumulation (CombinedPotential of the same potential twice)
    p = UwU(np.array([N, N]), kb, Sk, V, np.ones(2))
    c = CombinedPotential()
    c.add_potential(p)
    c.add_potential(p)
    ec, gc = c.get_energy_gradient(x)
    assert rel(ec, 2 * e0) < 1e-10 and rel(gc, 2 * g0) < 1e-10
    # exact mode: autograd against central differences
    xt = torch.tensor(x, device="cuda", requires_grad=True)
    structure_factor_loss(p, xt).backward()
    ga = xt.grad.cpu().numpy()
    idx = rng.choice(x.size, 8, replace=False)
    for i in idx:
        xp, xm = x.copy(), x.copy()
        xp[i] += 1e-4
        xm[i] -= 1e-4
        fd = (p.get_energy(xp) - p.get_energy(xm)) / 2e-4
        assert abs(fd - ga[i]) <= 1e-5 * np.max(np.abs(ga)), (i, fd, ga[i])
    xb = x.copy()
    xb[7] = np.nan
    eb, gb = p.get_energy_gradient(xb)
    assert np.isnan(eb) and np.isnan(gb).any() and p.status() != 0
