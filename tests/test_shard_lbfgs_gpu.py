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
