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
