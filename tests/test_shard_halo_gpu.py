"""Repulsion over a pattern split into spatial slabs with a halo exchange (ShardedInversePower(halo=True),
fresco_inversepower_halo_create): every rank evaluates only its own points' pairs against its own points
and the other ranks' points next to its columns.  The reference evaluates the cell-list repulsion in one
process (source/fresco/cell_list_potential.hpp:442-465, inversepower_potential.hpp:104-124); the
single-GPU InversePower, parity-tested against the reference, is the oracle here.  Several ranks are
emulated on one GPU by host threads whose gathers and sums meet at host barriers (no kernel waits on
another one)."""
import threading

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(np.asarray(b)), 1e-300))


class HostSum:
    """The sum over `n` emulated ranks (rank order, the same bits on every rank)."""

    def __init__(self, n):
        self.n = n
        self.bar = threading.Barrier(n, timeout=60)
        self.bufs = [None] * n

    def fn(self, rank):
        def reduce(t):
            self.bufs[rank] = t.cpu()
            self.bar.wait()
            total = self.bufs[0].clone()
            for r in range(1, self.n):
                total += self.bufs[r]
            self.bar.wait()
            t.copy_(total)

        return reduce


class HostGatherV:
    """The all-gather of arrays of varying length over `n` emulated ranks."""

    def __init__(self, n):
        self.bar = threading.Barrier(n, timeout=60)
        self.bufs = [None] * n

    def fn(self, rank):
        import torch

        def gatherv(local):
            self.bufs[rank] = local.cpu()
            self.bar.wait()
            cat = torch.cat(self.bufs)
            counts = [int(b.numel()) for b in self.bufs]
            self.bar.wait()
            return cat.to(local.device), counts

        return gatherv


def _pattern(ndim, n, seed, L=1.0, phi=0.5):
    """n points uniform in [0, L)^ndim (some outside the box by whole periods), radii 1 +- 20% scaled to
    a packing fraction of about phi."""
    rng = np.random.default_rng(seed)
    x = rng.random((n, ndim)) * L
    x[rng.random(n) < 0.05] += L * rng.integers(-2, 3, (1, ndim))
    r = 1.0 + 0.2 * (rng.random(n) - 0.5)
    vol = {1: 2.0, 2: np.pi, 3: 4.0 / 3.0 * np.pi}[ndim]
    scale = (phi * L ** ndim / (vol * np.sum(r ** ndim))) ** (1.0 / ndim)
    return x.ravel(), r * scale, np.full(ndim, L)


def _run_ranks(ndim, x, radii, boxv, cuts, evaluate="energy_gradient"):
    """Evaluates the halo shards of the slabs [cuts[r], cuts[r+1]) on emulated ranks: per rank
    (energy, gradient or None, (exported, halo))."""
    from fresco_b200.shard import HaloExchange, ShardedInversePower

    R = len(cuts) - 1
    hs, hg = HostSum(R), HostGatherV(R)
    shards = [ShardedInversePower(2.0, 1.0, radii, boxv, cuts[r], cuts[r + 1], halo=True, rank=r, nranks=R,
                                  exchange=HaloExchange(fn=hs.fn(r), gatherv_fn=hg.fn(r))) for r in range(R)]
    out, errs = [None] * R, []

    def drive(r):
        try:
            xs = x[ndim * cuts[r]:ndim * cuts[r + 1]]
            if evaluate == "energy":
                out[r] = (shards[r].get_energy(xs), None, shards[r].halo_stats())
            else:
                e, g = shards[r].get_energy_gradient(xs)
                out[r] = (e, g, shards[r].halo_stats())
        except Exception as exc:  # noqa: BLE001
            errs.append(exc)
            hs.bar.abort()
            hg.bar.abort()

    threads = [threading.Thread(target=drive, args=(r,)) for r in range(R)]
    for t in threads:
        t.start()
    for t in threads:
        t.join(timeout=300)
    assert not errs, errs
    return out


@pytest.mark.parametrize("ndim,n", [(1, 3000), (2, 20000), (3, 20000)])
def test_halo_one_process_equals_inversepower(ndim, n):
    from fresco_b200 import InversePower
    from fresco_b200.shard import ShardedInversePower

    x, radii, boxv = _pattern(ndim, n, seed=ndim)
    ref = InversePower(2.0, 1.0, radii, boxv, use_cell_lists=True)
    e0, g0 = ref.get_energy_gradient(x)
    sh = ShardedInversePower(2.0, 1.0, radii, boxv, 0, n, halo=True)
    assert "InversePowerHalo" in sh.describe()
    e1, g1 = sh.get_energy_gradient(x)
    assert e0 > 0 and abs(e1 - e0) <= 1e-12 * e0 and rel(g1, g0) < 1e-12
    assert sh.halo_stats() == (0, 0)  # nothing to exchange with no other process
    assert abs(sh.get_energy(x) - e0) <= 1e-12 * e0


@pytest.mark.parametrize("ndim,n,R", [(2, 30000, 3), (3, 30000, 2), (1, 4000, 4)])
def test_halo_ranks_equal_single_process(ndim, n, R):
    """Spatial slabs (points ordered by spatial_order, equal index slabs): every rank's energy is the
    pattern's, the concatenated gradient is the single-process one, and only a small share of the points
    travels.  The same split of the unordered points is still exact, with every point exported."""
    from fresco_b200 import InversePower
    from fresco_b200.shard import spatial_order

    x, radii, boxv = _pattern(ndim, n, seed=10 + ndim)
    cuts = [n * r // R for r in range(R + 1)]
    ref = InversePower(2.0, 1.0, radii, boxv, use_cell_lists=True)
    for order in ("spatial", "given"):
        if order == "spatial":
            p = spatial_order(x, boxv)
            xo, ro = x.reshape(n, ndim)[p].ravel(), radii[p]
        else:
            xo, ro = x, radii
        e0, g0 = InversePower(2.0, 1.0, ro, boxv, use_cell_lists=True).get_energy_gradient(xo)
        assert abs(e0 - ref.get_energy(x)) <= 1e-12 * e0
        out = _run_ranks(ndim, xo, ro, boxv, cuts)
        for e, _, _ in out:
            assert e == out[0][0] and abs(e - e0) <= 1e-12 * e0
        assert rel(np.concatenate([g for _, g, _ in out]), g0) < 1e-12
        exported = [s[0] for _, _, s in out]
        if order == "spatial":
            # the columns at the two ends of each slab (a few percent of the points) travel
            assert sum(exported) < 0.3 * n, exported
            assert all(s[1] > 0 for _, _, s in out)
        else:
            assert sum(exported) > 0.8 * n, exported  # most columns hold points of every rank
        energy_only = _run_ranks(ndim, xo, ro, boxv, cuts, evaluate="energy")
        for e, _, _ in energy_only:
            assert abs(e - e0) <= 1e-12 * e0


def test_halo_nonfinite_coordinate_makes_every_rank_nan():
    from fresco_b200.shard import spatial_order

    n, R = 9000, 3
    x, radii, boxv = _pattern(2, n, seed=5)
    p = spatial_order(x, boxv)
    xo, ro = x.reshape(n, 2)[p].ravel(), radii[p]
    cuts = [n * r // R for r in range(R + 1)]
    bad = xo.copy()
    bad[2 * (cuts[1] + 7)] = np.nan  # a point of rank 1
    out = _run_ranks(2, bad, ro, boxv, cuts)
    for e, g, _ in out:
        assert np.isnan(e) and np.isnan(g).all()
    out = _run_ranks(2, xo, ro, boxv, cuts)
    assert all(np.isfinite(e) for e, _, _ in out)


def test_halo_refusals():
    from fresco_b200.shard import ShardedInversePower

    x, radii, boxv = _pattern(2, 2000, seed=6)
    with pytest.raises(ValueError, match="cell lists"):  # fewer than 3 cells per dimension
        ShardedInversePower(2.0, 1.0, radii * 40, boxv, 0, 2000, halo=True)
    with pytest.raises(ValueError, match="periodic"):
        ShardedInversePower(2.0, 1.0, radii, boxv, 0, 2000, halo=True, method="cartesian")
    with pytest.raises(ValueError, match="process group or an exchange"):
        ShardedInversePower(2.0, 1.0, radii, boxv, 0, 1000, halo=True)


def _golden():
    import os

    return dict(np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "lbfgs_combined_2d.npz")))


def test_two_ranks_nuwu_plus_halo_repulsion_match_single_process():
    """The golden combined pattern (NUwU + cell-list repulsion), points in spatial order, over two
    emulated ranks: ShardedNUwU and the halo repulsion shard in one CombinedPotential per rank,
    ShardedLBFGS; the concatenated trajectory is the single-process LBFGS_CPP one and the reference's
    golden energies."""
    from fresco_b200 import CombinedPotential, InversePower, NUwU
    from fresco_b200.optimize import LBFGS_CPP
    from fresco_b200.shard import (HaloExchange, Reducer, ShardedInversePower, ShardedLBFGS, ShardedNUwU,
                                   spatial_order, weight_factor_sum)

    d = _golden()
    N = len(d["radii"])
    p = spatial_order(d["x"], d["L"])
    x = d["x"].reshape(N, 2)[p].ravel()
    radii, rep_radii = d["radii"][p], d["rep_radii"][p]
    cut = 128
    totals = (N, weight_factor_sum(radii, 2))
    hs, he, hg = HostSum(2), HostSum(2), HostGatherV(2)
    opts, keep = [], []
    for r, (a, b) in enumerate([(0, cut), (cut, N)]):
        comb = CombinedPotential()
        nu = ShardedNUwU(radii[a:b], float(d["K"]), d["Sk"], d["V"], d["L"], eps=1e-13, totals=totals)
        rp = ShardedInversePower(2.0, 1.0, rep_radii, d["L"], a, b, halo=True, rank=r, nranks=2,
                                 exchange=HaloExchange(fn=he.fn(r), gatherv_fn=hg.fn(r)))
        comb.add_potential(nu)
        comb.add_potential(rp)
        keep.append((nu, rp))
        opts.append(ShardedLBFGS(x[2 * a:2 * b], comb, M=10, tol=1e-12, reducer=Reducer(fn=hs.fn(r))))
    res, errs = [None, None], []

    def drive(r):
        try:
            res[r] = opts[r].run(15)
        except Exception as e:  # noqa: BLE001
            errs.append(e)
            for bar in (hs.bar, he.bar, hg.bar):
                bar.abort()

    threads = [threading.Thread(target=drive, args=(r,)) for r in range(2)]
    for t in threads:
        t.start()
    for t in threads:
        t.join(timeout=300)
    assert not errs, errs
    ref_comb = CombinedPotential()
    ref_comb.add_potential(NUwU(radii, float(d["K"]), d["Sk"], d["V"], d["L"], eps=1e-13))
    ref_comb.add_potential(InversePower(2.0, 1.0, rep_radii, d["L"], use_cell_lists=True))
    ra = LBFGS_CPP(x, ref_comb, M=10, tol=1e-12).run(15)
    r0, r1 = res
    assert r0.energy == r1.energy and r0.rms == r1.rms
    assert r0.nfev == r1.nfev == ra.nfev and r0.nsteps == r1.nsteps == ra.nsteps == 15
    assert rel(r0.energy, ra.energy) < 1e-8
    assert rel(np.concatenate([r0.coords, r1.coords]), ra.coords) < 1e-8
    assert rel(r0.energy, d["traj_energy"][-1]) < 1e-8  # the reference's own golden trajectory
    assert keep[0][1].halo_stats()[0] < N // 2  # not every point travelled
