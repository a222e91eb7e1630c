"""Device-resident LBFGS / FIRE against the reference optimisers (golden trajectories) and the oracle."""
import os

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(np.asarray(b)), 1e-300))


def test_lbfgs_golden_trajectory():
    from fresco_b200 import CombinedPotential, InversePower, NUwU
    from fresco_b200.optimize import LBFGS_CPP

    d = dict(np.load(os.path.join(GOLDEN, "lbfgs_combined_2d.npz")))
    nu = NUwU(d["radii"], float(d["K"]), d["Sk"], d["V"], d["L"], eps=1e-13)
    rep = InversePower(2.0, 1.0, d["rep_radii"], d["L"], use_cell_lists=True)
    comb = CombinedPotential()
    comb.add_potential(nu)
    comb.add_potential(rep)
    opt = LBFGS_CPP(d["x"], comb, tol=1e-12, M=10)
    for i in range(len(d["traj_energy"])):
        res = opt.one_iteration()
        assert rel(res.energy, d["traj_energy"][i]) < 1e-8, i
        assert res.nfev == d["traj_nfev"][i], i
    res = opt.get_result()
    assert rel(res.coords, d["x_final"]) < 1e-8
    assert rel(res.H0, d["H0"]) < 1e-6
    assert res.nsteps == len(d["traj_energy"])


def test_lbfgs_matches_oracle_with_backtracking():
    """Small maxstep / maxErise so the line search backtracks; rel_energy variant too."""
    from fresco_b200 import NUwU
    from fresco_b200.optimize import LBFGS_CPP

    x, radii, Sk, V, L = O.stealthy_nuwu_inputs(300, 6, 4, ndim=2, seed=8)
    for kw in [dict(maxstep=0.5, maxErise=1e-12), dict(maxstep=0.05, rel_energy=True, maxErise=1e-9)]:
        pot = NUwU(radii, 6, Sk, V, L, eps=1e-13)
        ref = O.NUwU(radii, 6, Sk, V, L)
        opt = LBFGS_CPP(x, pot, M=5, **kw)
        oref = O.LBFGS(x, ref, M=5, maxstep=kw["maxstep"], maxErise=kw["maxErise"],
                       rel_energy=kw.get("rel_energy", False))
        for _ in range(12):
            opt.one_iteration()
            oref.one_iteration()
        res = opt.get_result()
        assert rel(res.energy, oref.f) < 1e-8
        assert res.nfev == oref.nfev
        assert rel(res.coords, oref.x) < 1e-8


def test_lbfgs_run_stop_and_reset():
    from fresco_b200 import NUwU
    from fresco_b200.optimize import LBFGS_CPP

    # L = 1 (continuous map; see test_lbfgs_config1_converges_below_1e12)
    x, radii, Sk, V, L = O.stealthy_nuwu_inputs(200, 5, 3, ndim=2, seed=9, L=np.ones(2))
    pot = NUwU(radii, 5, Sk, V, L, eps=1e-13)
    opt = LBFGS_CPP(x, pot, tol=1e-4, M=8, nsteps=500)
    res = opt.run()
    assert res.success and res.rms <= 1e-4
    assert opt.stop_criterion_satisfied()
    n1 = opt.get_niter()
    res2 = opt.run(10)  # already converged: no iteration
    assert opt.get_niter() == n1 and res2.energy == res.energy
    opt.reset(x)
    assert opt.get_niter() == 0 and opt.get_result().nfev == 1
    assert opt.get_maxiter() == 500


def test_lbfgs_config1_converges_below_1e12():
    """2D NUwU, N=4096 seeded uniform points, 65x65 modes, S0=0 on 0<|k|<=16, M=10, FP64, run in
    chunks until E < 1e-12.  The box is expressed in the reference's own L=1 convention
    (examples/NUwU.ipynb): with L=2pi the reference map (p - round(p/L)) 2pi/L (nuwu.hpp:219) jumps by
    one radian at p = pi, the energy is discontinuous there and LBFGS stalls in the reference too."""
    from fresco_b200 import NUwU
    from fresco_b200.optimize import LBFGS_CPP

    d = dict(np.load(os.path.join(GOLDEN, "nuwu_2d_n4096.npz")))
    x = d["x"] / (2 * np.pi)
    pot = NUwU(d["radii"], 32, d["Sk"], d["V"], np.ones(2), eps=1e-13)
    ref = O.NUwU(d["radii"], 32, d["Sk"], d["V"], np.ones(2))
    e0, _ = pot.get_energy_gradient(x)
    assert abs(e0 - ref.get_energy(x)) <= 1e-10 * abs(e0)
    opt = LBFGS_CPP(x, pot, tol=0.0, M=10, nsteps=100000)
    energy = e0
    for _ in range(40):
        res = opt.run(250)
        energy = res.energy
        if energy < 1e-12:
            break
    assert energy < 1e-12, energy
    assert ref.get_energy(res.coords) < 1e-11


def test_fire_matches_oracle():
    from fresco_b200 import NUwU
    from fresco_b200.optimize import ModifiedFireCPP

    x, radii, Sk, V, L = O.stealthy_nuwu_inputs(300, 6, 4, ndim=2, seed=10)
    pot = NUwU(radii, 6, Sk, V, L, eps=1e-13)
    ref = O.NUwU(radii, 6, Sk, V, L)
    opt = ModifiedFireCPP(x, pot, dtstart=0.01, dtmax=0.1, maxstep=0.05, tol=1e-12)
    oref = O.ModifiedFire(x, ref, dtstart=0.01, dtmax=0.1, maxstep=0.05, tol=1e-12)
    for _ in range(30):
        opt.run(1)
        oref.run(1)
        assert rel(opt.get_result().energy, oref.f) < 1e-8
    res = opt.get_result()
    assert rel(res.coords, oref.x) < 1e-8
    assert res.nfev == oref.nfev


def test_fire_one_iteration_before_run_matches_reference_sequence():
    """MODIFIED_FIRE::one_iteration does not initialise f, g (modified_fire.hpp:160-178): the first call
    steps from f = 0, g = 0.  Through the Python API, get_result() then calls success(), which
    initialises them (opt.pyx:81-93, optimizer.hpp:169, 174-180), exactly as in the reference."""
    from fresco_b200 import NUwU
    from fresco_b200.optimize import ModifiedFireCPP

    x, radii, Sk, V, L = O.stealthy_nuwu_inputs(100, 4, 3, ndim=2, seed=11)
    pot = NUwU(radii, 4, Sk, V, L, eps=1e-13)
    opt = ModifiedFireCPP(x, pot)
    r1 = opt.one_iteration()
    assert r1.energy == 0.0 and r1.nfev == 1
    assert np.array_equal(r1.coords, x)
    oref = O.ModifiedFire(x, O.NUwU(radii, 4, Sk, V, L))
    oref.one_iteration()
    oref.stop_criterion_satisfied()  # what get_result() triggers
    for _ in range(4):
        r = opt.one_iteration()
        oref.one_iteration()
        oref.stop_criterion_satisfied()
        assert rel(r.energy, oref.f) < 1e-9
    assert r.nfev == oref.nfev
    assert rel(r.coords, oref.x) < 1e-9


def test_result_container_and_events():
    from fresco_b200 import NUwU
    from fresco_b200.optimize import LBFGS_CPP

    x, radii, Sk, V, L = O.stealthy_nuwu_inputs(100, 4, 3, ndim=2, seed=12)
    pot = NUwU(radii, 4, Sk, V, L)
    seen = []
    opt = LBFGS_CPP(x, pot, events=[lambda coords, energy, rms: seen.append(energy)])
    res = opt.run(5)
    assert len(seen) == 5 and seen[-1] == res.energy
    coords, energy, rms, nfev, same = res
    assert energy == res[1] and rms == res.rms and nfev == res.nfev and same is res


def test_graph_lbfgs_golden_trajectory():
    """The device-state LBFGS (one graph launch per evaluation) on the reference's golden trajectory:
    NUwU + cell-list repulsion, same final energy, coordinates, iterations and evaluations."""
    from fresco_b200 import CombinedPotential, InversePower, NUwU
    from fresco_b200.optimize import LBFGS_Graph

    d = dict(np.load(os.path.join(GOLDEN, "lbfgs_combined_2d.npz")))
    nu = NUwU(d["radii"], float(d["K"]), d["Sk"], d["V"], d["L"], eps=1e-13)
    rep = InversePower(2.0, 1.0, d["rep_radii"], d["L"], use_cell_lists=True)
    comb = CombinedPotential()
    comb.add_potential(nu)
    comb.add_potential(rep)
    opt = LBFGS_Graph(d["x"], comb, tol=1e-12, M=10)
    n = len(d["traj_energy"])
    opt.run(n)
    res = opt.get_result()
    assert res.nsteps == n
    assert res.nfev == d["traj_nfev"][-1]
    assert rel(res.energy, d["traj_energy"][-1]) < 1e-8
    assert rel(res.coords, d["x_final"]) < 1e-8


def test_graph_lbfgs_matches_lbfgs_cpp_fp32():
    from fresco_b200 import NUwU
    from fresco_b200.optimize import LBFGS_CPP, LBFGS_Graph

    x, radii, Sk, V, L = O.stealthy_nuwu_inputs(5000, 32, 12, ndim=2, seed=4, L=np.ones(2))
    pot = NUwU(radii, 32, Sk, V, L, precision="fp32")
    e0 = pot.get_energy(x)
    a = LBFGS_CPP(x, pot, M=4)
    b = LBFGS_Graph(x, NUwU(radii, 32, Sk, V, L, precision="fp32"), M=4)
    a.run(20)
    b.run(20)
    ra, rb = a.get_result(), b.get_result()
    assert ra.nsteps == rb.nsteps
    # FP32 spreading accumulates with float atomics in no fixed order, so two runs of either optimiser
    # drift apart by about 1e-5 over 20 iterations, and an energy rise that sits at the backtracking
    # threshold (lbfgs.cpp:206-236) can be accepted in one run and halved in the other; exact parity
    # is the FP64 golden test above.  The loss falls by orders of magnitude, so its noise is measured
    # against its start.
    assert abs(ra.nfev - rb.nfev) <= 2
    if ra.nfev == rb.nfev:
        assert abs(rb.energy - ra.energy) < 1e-6 * e0
        assert rel(rb.coords, ra.coords) < 2e-4
    else:
        assert ra.energy < 1e-2 * e0 and rb.energy < 1e-2 * e0


def test_graph_fire_matches_fire_cpp():
    """ModifiedFire_Graph (one CUDA graph launch per iteration, loop state on the device) against
    ModifiedFireCPP in FP64: same trajectory, iterations and evaluations, through one_iteration,
    run(niter) in chunks, the stop at tol, reset and both step-back settings."""
    from fresco_b200 import NUwU
    from fresco_b200.optimize import ModifiedFire_Graph, ModifiedFireCPP

    x, radii, Sk, V, L = O.stealthy_nuwu_inputs(300, 6, 4, ndim=2, seed=10)
    for stepback in (True, False):
        kw = dict(dtstart=0.01, dtmax=0.1, maxstep=0.05, tol=1e-12, stepback=stepback)
        a = ModifiedFireCPP(x, NUwU(radii, 6, Sk, V, L, eps=1e-13), **kw)
        b = ModifiedFire_Graph(x, NUwU(radii, 6, Sk, V, L, eps=1e-13), **kw)
        ra, rb = a.one_iteration(), b.one_iteration()  # before run: steps from f = 0, g = 0
        assert rb.nfev == ra.nfev == 1
        if stepback:  # P = 0, a step back: f stays 0
            assert rb.energy == ra.energy == 0.0
        else:  # f = E(x) from two potential objects, equal up to the order of FP64 sums
            assert rel(rb.energy, ra.energy) < 1e-12
        for niter in (1, 3, 7, 40):
            ra, rb = a.run(niter), b.run(niter)
            assert rb.nsteps == ra.nsteps and rb.nfev == ra.nfev, (niter, ra.nsteps, rb.nsteps)
            assert rel(rb.energy, ra.energy) < 1e-8
            assert rel(rb.coords, ra.coords) < 1e-8
            assert rel(rb.grad, ra.grad) < 1e-8
        a.reset(x)
        b.reset(x)
        assert b.get_niter() == 0 and b.get_result().nfev == a.get_result().nfev == 1
        ra, rb = a.run(12), b.run(12)
        assert rb.nsteps == ra.nsteps == 12 and rb.nfev == ra.nfev
        assert rel(rb.coords, ra.coords) < 1e-8

    # the stop at tol: both stop on the same iteration
    x, radii, Sk, V, L = O.stealthy_nuwu_inputs(200, 5, 3, ndim=2, seed=9, L=np.ones(2))
    a = ModifiedFireCPP(x, NUwU(radii, 5, Sk, V, L, eps=1e-13), tol=1e-3, nsteps=3000)
    b = ModifiedFire_Graph(x, NUwU(radii, 5, Sk, V, L, eps=1e-13), tol=1e-3, nsteps=3000)
    ra, rb = a.run(), b.run()
    assert ra.success and rb.success and rb.rms <= 1e-3
    assert rb.nsteps == ra.nsteps and rb.nfev == ra.nfev
    assert rel(rb.coords, ra.coords) < 1e-8
    assert b.run(10).nsteps == rb.nsteps  # converged: no iteration


@pytest.mark.parametrize("graph_first", [False, True])
def test_graph_fire_combined_potential(graph_first):
    """The graph FIRE on NUwU + cell-list repulsion (the golden combined inputs): the repulsion's cell
    sort and pair kernels are captured into the loop's branches; same trajectory as ModifiedFireCPP."""
    from fresco_b200 import CombinedPotential, InversePower, NUwU
    from fresco_b200.optimize import ModifiedFire_Graph, ModifiedFireCPP

    d = dict(np.load(os.path.join(GOLDEN, "lbfgs_combined_2d.npz")))

    def comb():
        c = CombinedPotential()
        c.add_potential(NUwU(d["radii"], float(d["K"]), d["Sk"], d["V"], d["L"], eps=1e-13))
        c.add_potential(InversePower(2.0, 1.0, d["rep_radii"], d["L"], use_cell_lists=True))
        return c

    kw = dict(dtstart=0.01, dtmax=0.1, maxstep=0.05, tol=1e-10)
    a, b = ModifiedFireCPP(d["x"], comb(), **kw), ModifiedFire_Graph(d["x"], comb(), **kw)
    if graph_first:
        rb, ra = b.run(40), a.run(40)
    else:
        ra, rb = a.run(40), b.run(40)
    assert rb.nsteps == ra.nsteps == 40 and rb.nfev == ra.nfev
    assert rel(rb.energy, ra.energy) < 1e-8
    assert rel(rb.coords, ra.coords) < 1e-8


def test_checkpoint_resumes_exactly(tmp_path):
    """save_state / load_state: stopping, saving, loading into a fresh optimiser and continuing gives the
    uninterrupted trajectory (LBFGS memory, FIRE velocities and step sizes, counters); a FIRE image loads
    into the graph form too; mismatched images are refused."""
    from fresco_b200 import NUwU
    from fresco_b200.optimize import LBFGS_CPP, ModifiedFire_Graph, ModifiedFireCPP

    x, radii, Sk, V, L = O.stealthy_nuwu_inputs(400, 8, 5, ndim=2, seed=13, L=np.ones(2))

    def pot():
        return NUwU(radii, 8, Sk, V, L, eps=1e-13)

    # tol far below the reachable rms: two potential objects agree to the last few bits, and a stop
    # decision at the tolerance would turn on those bits; a wrong load diverges at the percent level
    a = LBFGS_CPP(x, pot(), M=5, tol=1e-12)
    a.run(10)
    img = a.save_state()
    ra = a.run(12)
    b = LBFGS_CPP(np.zeros_like(x), pot(), M=5, tol=1e-12)
    b.load_state(img)
    rb = b.run(12)
    assert rb.nsteps == ra.nsteps == 22 and rb.nfev == ra.nfev
    assert rel(rb.energy, ra.energy) < 1e-8 and rel(rb.coords, ra.coords) < 1e-8
    assert rel(rb.H0, ra.H0) < 1e-6
    with pytest.raises(ValueError, match="memory length"):
        LBFGS_CPP(x, pot(), M=4).load_state(img)
    with pytest.raises(ValueError, match="another optimiser family"):
        ModifiedFireCPP(x, pot()).load_state(img)
    with pytest.raises(ValueError, match="another number of coordinates"):
        LBFGS_CPP(x[:-2], NUwU(radii[:-1], 8, Sk, V, L), M=5).load_state(img)

    kw = dict(dtstart=0.01, dtmax=0.1, maxstep=0.05, tol=1e-12)
    f = ModifiedFireCPP(x, pot(), **kw)
    f.run(15)
    f.save_checkpoint(str(tmp_path / "fire.npy"))
    rf = f.run(15)
    for cls in (ModifiedFireCPP, ModifiedFire_Graph):
        g = cls(np.zeros_like(x), pot(), **kw)
        g.load_checkpoint(str(tmp_path / "fire.npy"))
        rg = g.run(15)
        assert rg.nsteps == rf.nsteps == 30 and rg.nfev == rf.nfev, cls.__name__
        assert rel(rg.energy, rf.energy) < 1e-8 and rel(rg.coords, rf.coords) < 1e-8, cls.__name__
