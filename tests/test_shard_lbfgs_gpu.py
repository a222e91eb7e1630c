"""LBFGS over one NUwU pattern split between processes (ShardedLBFGS): the device LBFGS with every
dot product's partial sums and the shard's rho reduced over the ranks.  One process: the reduction
is the identity and the trajectory is LBFGS_CPP's.  Two ranks are emulated on one GPU by two host
threads whose reducers meet at a host barrier (no kernel waits on another one): the concatenated
trajectory is the single-process one."""
import threading

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(np.asarray(b)), 1e-300))


class HostSum:
    """The sum over `n` emulated ranks: each copies its array to the host, meets the others at a barrier,
    and takes the rank-ordered sum back (every rank gets the same bits)."""

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


def _inputs():
    return O.stealthy_nuwu_inputs(3000, 16, 8, ndim=2, seed=21, L=np.ones(2))


def test_one_rank_matches_lbfgs_cpp():
    from fresco_b200 import NUwU
    from fresco_b200.optimize import LBFGS_CPP
    from fresco_b200.shard import ShardedLBFGS, ShardedNUwU, weight_factor_sum

    x, radii, Sk, V, L = _inputs()
    ref = LBFGS_CPP(x, NUwU(radii, 16, Sk, V, L, eps=1e-13), M=5)
    shard = ShardedNUwU(radii, 16, Sk, V, L, eps=1e-13, totals=(len(radii), weight_factor_sum(radii, 2)))
    opt = ShardedLBFGS(x, shard, M=5)
    for _ in range(4):
        ra, rb = ref.run(5), opt.run(5)
        assert rb.nfev == ra.nfev and rb.nsteps == ra.nsteps
        assert rel(rb.energy, ra.energy) < 1e-9
        assert rel(rb.coords, ra.coords) < 1e-9
        assert rel(rb.rms, ra.rms) < 1e-8
    assert opt.reducer.calls == 0  # one process: nothing to exchange, no hooks
    # the same run through the exchange hooks, with an identity reducer
    from fresco_b200.shard import Reducer

    shard2 = ShardedNUwU(radii, 16, Sk, V, L, eps=1e-13, totals=(len(radii), weight_factor_sum(radii, 2)))
    hooked = ShardedLBFGS(x, shard2, M=5, reducer=Reducer(fn=lambda t: None))
    rh = hooked.run(20)
    assert hooked.reducer.calls > 0 and rh.nfev == ra.nfev and rh.nsteps == ra.nsteps
    assert rel(rh.energy, ra.energy) < 1e-9 and rel(rh.coords, ra.coords) < 1e-9
    # a slab of a larger pattern without a group or a reducer is refused
    half = ShardedNUwU(radii[:100], 16, Sk, V, L, totals=(len(radii), weight_factor_sum(radii, 2)))
    with pytest.raises(ValueError, match="process group or a reducer"):
        ShardedLBFGS(x[:200], half)


def test_two_ranks_emulated_match_single_process():
    from fresco_b200 import NUwU
    from fresco_b200.optimize import LBFGS_CPP
    from fresco_b200.shard import Reducer, ShardedLBFGS, ShardedNUwU, weight_factor_sum

    x, radii, Sk, V, L = _inputs()
    N = len(radii)
    cut = 1234  # unequal slabs
    totals = (N, weight_factor_sum(radii, 2))
    hs = HostSum(2)
    parts = [(0, cut), (cut, N)]
    opts = []
    for r, (a, b) in enumerate(parts):
        shard = ShardedNUwU(radii[a:b], 16, Sk, V, L, eps=1e-13, totals=totals)
        opts.append(ShardedLBFGS(x[2 * a:2 * b], shard, M=5, reducer=Reducer(fn=hs.fn(r))))
    ref = LBFGS_CPP(x, NUwU(radii, 16, Sk, V, L, eps=1e-13), M=5)
    res = [None, None]
    errs = []

    def drive(r):
        try:
            res[r] = opts[r].run(15)
        except Exception as e:  # noqa: BLE001
            errs.append(e)
            hs.bar.abort()

    threads = [threading.Thread(target=drive, args=(r,)) for r in range(2)]
    for t in threads:
        t.start()
    for t in threads:
        t.join(timeout=300)
    assert not errs, errs
    ra = ref.run(15)
    r0, r1 = res
    assert r0.energy == r1.energy and r0.rms == r1.rms  # the same scalars on every rank
    assert r0.nfev == r1.nfev == ra.nfev and r0.nsteps == r1.nsteps == ra.nsteps == 15
    assert rel(r0.energy, ra.energy) < 1e-9
    assert rel(np.concatenate([r0.coords, r1.coords]), ra.coords) < 1e-9
    assert rel(np.concatenate([r0.grad, r1.grad]), ra.grad) < 1e-8


def test_reducer_is_refused_where_there_is_no_exchange():
    import ctypes as C

    from fresco_b200 import InversePower, NUwU
    from fresco_b200._lib import check, lib
    from fresco_b200.optimize import ModifiedFireCPP
    from fresco_b200.shard import Reducer, ShardedLBFGS, ShardedNUwU, weight_factor_sum

    x, radii, Sk, V, L = _inputs()
    red = Reducer()
    plain = NUwU(radii, 16, Sk, V, L)  # kept alive while its handle is in use
    with pytest.raises(ValueError, match="only a shard"):
        check(lib.fresco_potential_set_reducer(plain.handle, C.cast(red.c_fn, C.c_void_p), None))
    rep = InversePower(2.0, 1.0, np.full(len(radii), 0.005), L, use_cell_lists=True)
    with pytest.raises(ValueError, match="no exchange step"):
        check(lib.fresco_potential_set_reducer(rep.handle, C.cast(red.c_fn, C.c_void_p), None))
    shard = ShardedNUwU(radii, 16, Sk, V, L, totals=(len(radii), weight_factor_sum(radii, 2)))
    with pytest.raises(ValueError, match="expected"):
        ShardedLBFGS(x[:-2], shard)
    fire = ModifiedFireCPP(x, NUwU(radii, 16, Sk, V, L))
    with pytest.raises(ValueError, match="does not run over a sharded pattern"):
        check(lib.fresco_optimizer_set_reducer(fire._h, C.cast(red.c_fn, C.c_void_p), None, x.size))


class HostGather:
    """The all-gather over `n` emulated ranks: local arrays to the host, a barrier, the rank-ordered
    concatenation back into each rank's full array."""

    def __init__(self, n):
        self.bar = threading.Barrier(n, timeout=60)
        self.bufs = [None] * n

    def fn(self, rank):
        import torch

        def gather(local, full):
            self.bufs[rank] = local.cpu()
            self.bar.wait()
            cat = torch.cat(self.bufs)
            self.bar.wait()
            full.copy_(cat)

        return gather


def _golden():
    import os

    d = dict(np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "lbfgs_combined_2d.npz")))
    return d


def test_sharded_repulsion_one_process_equals_inversepower():
    from fresco_b200 import InversePower
    from fresco_b200.shard import ShardedInversePower

    d = _golden()
    n = len(d["rep_radii"])
    sh = ShardedInversePower(2.0, 1.0, d["rep_radii"], d["L"], 0, n)
    ref = InversePower(2.0, 1.0, d["rep_radii"], d["L"], use_cell_lists=True)
    e0, g0 = ref.get_energy_gradient(d["x"])
    e1, g1 = sh.get_energy_gradient(d["x"])
    assert e0 > 0 and abs(e1 - e0) <= 1e-12 * e0 and rel(g1, g0) < 1e-12
    assert abs(sh.get_energy(d["x"]) - e0) <= 1e-12 * e0
    with pytest.raises(ValueError, match="process group or an exchange"):
        ShardedInversePower(2.0, 1.0, d["rep_radii"], d["L"], 0, n // 2)


def test_two_ranks_nuwu_plus_repulsion_match_single_process():
    """The golden combined pattern (NUwU + cell-list repulsion) over two emulated ranks: ShardedNUwU and
    ShardedInversePower in one CombinedPotential per rank, ShardedLBFGS; the concatenated trajectory is
    the single-process LBFGS_CPP one."""
    from fresco_b200 import CombinedPotential, InversePower, NUwU
    from fresco_b200.optimize import LBFGS_CPP
    from fresco_b200.shard import Exchange, Reducer, ShardedInversePower, ShardedLBFGS, ShardedNUwU, weight_factor_sum

    d = _golden()
    N = len(d["radii"])
    cut = 100
    totals = (N, weight_factor_sum(d["radii"], 2))
    hs, he, hg = HostSum(2), HostSum(2), HostGather(2)
    opts, keep = [], []
    for r, (a, b) in enumerate([(0, cut), (cut, N)]):
        comb = CombinedPotential()
        nu = ShardedNUwU(d["radii"][a:b], float(d["K"]), d["Sk"], d["V"], d["L"], eps=1e-13, totals=totals)
        rp = ShardedInversePower(2.0, 1.0, d["rep_radii"], d["L"], a, b,
                                 exchange=Exchange(fn=he.fn(r), gather_fn=hg.fn(r)))
        comb.add_potential(nu)
        comb.add_potential(rp)
        keep.append((nu, rp))
        opts.append(ShardedLBFGS(d["x"][2 * a:2 * b], comb, M=10, tol=1e-12, reducer=Reducer(fn=hs.fn(r))))
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
    ref_comb.add_potential(NUwU(d["radii"], float(d["K"]), d["Sk"], d["V"], d["L"], eps=1e-13))
    ref_comb.add_potential(InversePower(2.0, 1.0, d["rep_radii"], d["L"], use_cell_lists=True))
    ra = LBFGS_CPP(d["x"], ref_comb, M=10, tol=1e-12).run(15)
    r0, r1 = res
    assert r0.energy == r1.energy and r0.rms == r1.rms
    assert r0.nfev == r1.nfev == ra.nfev and r0.nsteps == r1.nsteps == ra.nsteps == 15
    assert rel(r0.energy, ra.energy) < 1e-8
    assert rel(np.concatenate([r0.coords, r1.coords]), ra.coords) < 1e-8
    assert rel(r0.energy, d["traj_energy"][-1]) < 1e-8  # the reference's own golden trajectory


def test_graph_optimisers_refuse_exchange_steps():
    """A potential with a host exchange step is never captured: the graph-captured optimisers refuse it,
    and a CombinedPotential holding it evaluates without capture (its result stays right)."""
    from fresco_b200 import CombinedPotential, InversePower
    from fresco_b200.optimize import LBFGS_Graph, ModifiedFire_Graph
    from fresco_b200.shard import ShardedInversePower

    d = _golden()
    n = len(d["rep_radii"])
    sh = ShardedInversePower(2.0, 1.0, d["rep_radii"], d["L"], 0, n)
    with pytest.raises(ValueError, match="exchanges between processes"):
        ModifiedFire_Graph(d["x"], sh).run(3)
    with pytest.raises(ValueError, match="exchanges between processes"):
        LBFGS_Graph(d["x"], sh)
    comb = CombinedPotential()
    comb.add_potential(sh)
    ref = InversePower(2.0, 1.0, d["rep_radii"], d["L"], use_cell_lists=True)
    e0, g0 = ref.get_energy_gradient(d["x"])
    for _ in range(3):  # repeated calls: the second would capture a graph
        e1, g1 = comb.get_energy_gradient(d["x"])
        assert abs(e1 - e0) <= 1e-12 * e0 and rel(g1, g0) < 1e-12
