"""One NUwU pattern whose points are split over the processes of a torch.distributed group.

The reference evaluates a pattern's loss in one process (fresco/potentials/nuwu.pyx:10-44,
source/fresco/nuwu.hpp:210-317).  For a pattern too large for one GPU each rank holds a slab of
the points.  rho(k) = sum_j c_j exp(i k.x_j) is linear in the points, so per evaluation

1. every rank computes rho of its own points at the active modes (V(k) != 0 or V(-k) != 0)
   with its own sort, spread and type-1 transform (``fresco_nuwu_shard_rho``);
2. one all-reduce sums the ranks' rho arrays (2 doubles per active mode; NCCL over NVLink for
   CUDA tensors);
3. every rank finishes the mode pass with the pattern's rho (the same loss on every rank) and
   interpolates its own points (``fresco_nuwu_shard_finish``).

The weights are normalised over the whole pattern (nuwu.hpp:125-149): ``shard_totals`` sums
the point counts and weight factors of all ranks once, at construction.  A rank may hold no
points.  Non-finite coordinates on any rank make the loss NaN on every rank.
"""
from __future__ import annotations

import ctypes as C

from . import _lib
from ._lib import check, dptr, lib
from .potentials import BasePotential, CombinedPotential, Distance, _f64, _precision

__all__ = ["ShardedNUwU", "ShardedInversePower", "ShardedLBFGS", "Reducer", "Exchange", "HaloExchange",
           "gather_varying", "spatial_order", "shard_totals", "weight_factor_sum"]


def _dist(group):
    try:
        import torch.distributed as dist
    except ImportError:  # pragma: no cover
        return None
    if not dist.is_available() or not dist.is_initialized():
        return None
    if dist.get_world_size(group) <= 1:
        return None
    return dist


def weight_factor_sum(radii, ndim: int) -> float:
    """Sum over the points of NUwU's per-point weight factor (the area factor applied once per
    dimension, nuwu.hpp:131-141), as the library computes it."""
    r = _f64(radii)
    out = C.c_double(0.0)
    check(lib.fresco_nuwu_weight_sum(dptr(r), r.size, int(ndim), C.byref(out)))
    return out.value


def shard_totals(radii_local, ndim: int, group=None, device=None):
    """(n_total, weight_sum_total) over all ranks of `group` (this rank's values without a group)."""
    n = len(radii_local)
    ws = weight_factor_sum(radii_local, ndim)
    dist = _dist(group)
    if dist is None:
        return n, ws
    import torch

    if device is None:
        device = "cuda" if dist.get_backend(group) == "nccl" else "cpu"
    t = torch.tensor([float(n), ws], dtype=torch.float64, device=device)
    dist.all_reduce(t, group=group)
    return int(round(float(t[0]))), float(t[1])


class ShardedNUwU(BasePotential):
    """This rank's share of one NUwU pattern (fresco/potentials/nuwu.pyx:10-23 arguments, with
    `radii_local` the radii of this rank's points).

    ``totals = (n_total, weight_sum_total)`` skips the group reduction of ``shard_totals`` (a
    caller that knows them, or one that drives several shards itself).  ``get_energy_gradient``
    takes this rank's coordinates and returns the pattern's loss and this rank's gradient; the
    three steps are also available as ``rho``, ``reduce`` and ``finish``.
    """

    def __init__(self, radii_local, K, Sk, V, L, eps=1e-6, precision="fp64", group=None, totals=None):
        self.radii = _f64(radii_local)
        self.N = len(self.radii)
        self.K = float(K)
        self.Sk = _f64(Sk)
        self.V = _f64(V)
        assert len(self.Sk) == len(self.V)
        self.L = _f64(L)
        self.ndim = len(self.L)
        self.eps = float(eps)
        self.precision = str(precision)
        self.group = group
        self.n_total, self.weight_sum = totals if totals is not None else shard_totals(self.radii, self.ndim, group)
        h = _lib.handle_t()
        check(lib.fresco_nuwu_shard_create(dptr(self.radii), self.N, int(self.n_total), float(self.weight_sum),
                                           self.K, dptr(self.Sk), dptr(self.V), self.Sk.size, dptr(self.L), self.ndim,
                                           self.eps, _precision(precision), C.byref(h)))
        self._h = h
        n = C.c_int64(0)
        check(lib.fresco_nuwu_shard_nrho(self._h, C.byref(n)))
        self.n_rho = int(n.value)

    def __del__(self):
        h, self._h = getattr(self, "_h", None), None
        if h:
            try:
                lib.fresco_potential_destroy(h)
            except Exception:
                pass

    @staticmethod
    def _stream(x):
        import torch

        return torch.cuda.current_stream(x.device).cuda_stream

    def _device_x(self, x):
        import torch

        if isinstance(x, torch.Tensor):
            if not x.is_cuda or x.dtype != torch.float64:
                raise ValueError("device coordinates must be a float64 CUDA tensor")
            return x.contiguous()
        xa = _f64(x)
        if xa.size != self.N * self.ndim:
            raise ValueError(f"expected {self.N * self.ndim} coordinates, got {xa.size}")
        return torch.from_numpy(xa).to("cuda")

    def rho(self, x):
        """rho of this rank's points at the active modes: a float64 CUDA tensor of 2 * n_rho values."""
        import torch

        xd = self._device_x(x)
        r = torch.empty(2 * max(self.n_rho, 1), dtype=torch.float64, device=xd.device)
        check(lib.fresco_nuwu_shard_rho(self._h, xd.data_ptr(), xd.numel(), r.data_ptr(), self._stream(xd)))
        self._x = xd  # the last coordinates stay referenced until the next call
        return r

    def reduce(self, rho):
        """Sums rho over the ranks of the group in place (no-op without a multi-rank group)."""
        dist = _dist(self.group)
        if dist is not None:
            dist.all_reduce(rho, group=self.group)
        return rho

    def finish(self, rho, want_grad=True):
        """(energy tensor, gradient tensor or None) from the summed rho."""
        import torch

        e = torch.zeros((), dtype=torch.float64, device=rho.device)
        g = torch.empty(self.N * self.ndim, dtype=torch.float64, device=rho.device) if want_grad else None
        check(lib.fresco_nuwu_shard_finish(self._h, rho.data_ptr(), g.data_ptr() if want_grad else None,
                                           e.data_ptr(), self._stream(rho)))
        return e, g

    def get_energy_gradient(self, x):
        import torch

        r = self.reduce(self.rho(x))
        e, g = self.finish(r, want_grad=True)
        if isinstance(x, torch.Tensor):
            return float(e.item()), g
        return float(e.item()), g.cpu().numpy()

    def get_energy(self, x):
        r = self.reduce(self.rho(x))
        e, _ = self.finish(r, want_grad=False)
        return float(e.item())

    def status(self) -> int:
        st = C.c_int(0)
        check(lib.fresco_potential_status(self._h, None, C.byref(st)))
        return st.value


# fresco_reduce_fn: (device address, count, CUDA stream, context)
REDUCE_FN = C.CFUNCTYPE(None, C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p)


class _DeviceArray:
    """A float64 device array at a raw address, for a zero-copy torch view (CUDA array interface)."""

    def __init__(self, ptr, count):
        self.__cuda_array_interface__ = {"shape": (int(count),), "typestr": "<f8", "data": (int(ptr), False),
                                         "version": 3, "strides": None}


class Reducer:
    """The exchange step of a pattern split over processes, as the library calls it: a fresco_reduce_fn
    that views the device array as a float64 tensor and sums it over the processes in place, on the
    library's stream.  `fn(tensor)` does the sum (default: torch.distributed.all_reduce over `group`, a
    no-op without a multi-rank group).  Exceptions cannot cross the C boundary: they are kept and raised
    by `check()`."""

    def __init__(self, group=None, fn=None):
        self.group = group
        self.fn = fn
        self.error = None
        self.calls = 0
        self._streams = {}
        self.c_fn = REDUCE_FN(self._call)  # kept alive with this object

    def active(self) -> bool:
        """Whether there is anything to sum: a custom `fn`, or a process group of several ranks."""
        return self.fn is not None or _dist(self.group) is not None

    def _call(self, ptr, count, stream, ctx):
        try:
            self.calls += 1
            if self.error is not None or count <= 0:
                return
            import torch

            t = torch.as_tensor(_DeviceArray(ptr, count), device="cuda")
            with torch.cuda.stream(self._stream(stream, t.device)):
                if self.fn is not None:
                    self.fn(t)
                else:
                    dist = _dist(self.group)
                    if dist is not None:
                        dist.all_reduce(t, group=self.group)
        except BaseException as exc:  # noqa: BLE001 (reported by check())
            if self.error is None:
                self.error = exc

    def _stream(self, stream, device):
        import torch

        key = int(stream or 0)
        st = self._streams.get(key)
        if st is None:
            st = self._streams[key] = torch.cuda.ExternalStream(key, device=device)
        return st

    def check(self):
        if self.error is not None:
            err, self.error = self.error, None
            raise RuntimeError(f"the exchange step failed: {err!r}") from err


# fresco_gather_fn: (local address, local count, full address, full count, CUDA stream, context)
GATHER_FN = C.CFUNCTYPE(None, C.c_void_p, C.c_int64, C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p)


class Exchange(Reducer):
    """A Reducer that also gathers: the library's fresco_gather_fn concatenates the ranks' local arrays
    in rank order into a full device array.  `gather_fn(local, full)` does it (default: an NCCL
    all-gather over `group` of arrays padded to the longest, `counts` doubles per rank; a plain copy
    without a multi-rank group)."""

    def __init__(self, group=None, fn=None, gather_fn=None, counts=None):
        super().__init__(group, fn)
        self.gather_fn = gather_fn
        self.counts = counts
        self.c_gather = GATHER_FN(self._gather)

    def active(self) -> bool:
        return super().active() or self.gather_fn is not None

    def _gather(self, lptr, lcount, fptr, fcount, stream, ctx):
        try:
            self.calls += 1
            if self.error is not None:
                return
            import torch

            full = torch.as_tensor(_DeviceArray(fptr, fcount), device="cuda")
            local = torch.as_tensor(_DeviceArray(lptr, lcount), device="cuda") if lcount > 0 else full[:0]
            with torch.cuda.stream(self._stream(stream, full.device)):
                if self.gather_fn is not None:
                    self.gather_fn(local, full)
                    return
                dist = _dist(self.group)
                if dist is None:
                    full.copy_(local)
                    return
                m = max(self.counts)
                buf = torch.zeros(m, dtype=torch.float64, device=full.device)
                buf[:lcount].copy_(local)
                out = torch.empty(m * len(self.counts), dtype=torch.float64, device=full.device)
                dist.all_gather_into_tensor(out, buf, group=self.group)
                off = 0
                for r, c in enumerate(self.counts):
                    full[off:off + c].copy_(out[r * m:r * m + c])
                    off += c
        except BaseException as exc:  # noqa: BLE001 (reported by check())
            if self.error is None:
                self.error = exc


# fresco_gatherv_fn: (local address, local count, full address, full capacity, host counts, stream, context)
GATHERV_FN = C.CFUNCTYPE(None, C.c_void_p, C.c_int64, C.c_void_p, C.c_int64, C.POINTER(C.c_int64), C.c_void_p,
                         C.c_void_p)


def gather_varying(local, group=None):
    """All-gather of 1-D tensors whose lengths differ between the ranks of `group`: returns the
    concatenation in rank order and the list of lengths.  Two collectives (the lengths, then the
    arrays padded to the longest); CPU tensors over gloo and CUDA tensors over NCCL alike."""
    import torch

    dist = _dist(group)
    if dist is None:
        return local, [int(local.numel())]
    ws = dist.get_world_size(group)
    n = torch.tensor([local.numel()], dtype=torch.int64, device=local.device)
    ns = [torch.zeros_like(n) for _ in range(ws)]
    dist.all_gather(ns, n, group=group)
    counts = [int(c.item()) for c in ns]
    m = max(max(counts), 1)
    buf = torch.zeros(m, dtype=local.dtype, device=local.device)
    buf[:local.numel()].copy_(local)
    outs = [torch.empty_like(buf) for _ in range(ws)]
    dist.all_gather(outs, buf, group=group)
    return torch.cat([o[:c] for o, c in zip(outs, counts)]), counts


def spatial_order(x, boxv):
    """Permutation of the points (x flat, D coordinates per point) in the order of their coordinate along
    axis 0 wrapped into the box: split into equal index slabs after it, every slab is a spatial slab,
    which is what makes the halo exchange of ShardedInversePower(halo=True) small.  Apply it to the
    coordinates and the radii alike (the losses do not depend on the order of the points)."""
    import numpy as np

    boxv = np.asarray(boxv, dtype=np.float64)
    pts = np.asarray(x, dtype=np.float64).reshape(-1, boxv.size)
    return np.argsort(np.mod(pts[:, 0], boxv[0]), kind="stable")


class HaloExchange(Reducer):
    """A Reducer that also gathers arrays of varying length (the library's fresco_gatherv_fn): the
    column marks and the exported points of a ShardedInversePower(halo=True).  `gatherv_fn(local)`
    returns (concatenation in rank order, lengths) (default: gather_varying over `group`, the local
    array alone without a multi-rank group)."""

    def __init__(self, group=None, fn=None, gatherv_fn=None):
        super().__init__(group, fn)
        self.gatherv_fn = gatherv_fn
        self.c_gatherv = GATHERV_FN(self._gatherv)

    def active(self) -> bool:
        return super().active() or self.gatherv_fn is not None

    def _gatherv(self, lptr, lcount, fptr, fcap, counts_ptr, stream, ctx):
        try:
            self.calls += 1
            if self.error is not None:
                return
            import torch

            full = torch.as_tensor(_DeviceArray(fptr, fcap), device="cuda")
            local = torch.as_tensor(_DeviceArray(lptr, lcount), device="cuda") if lcount > 0 else full[:0]
            with torch.cuda.stream(self._stream(stream, full.device)):
                if self.gatherv_fn is not None:
                    cat, counts = self.gatherv_fn(local)
                else:
                    cat, counts = gather_varying(local, self.group)
                if sum(counts) > fcap:
                    raise RuntimeError(f"gathered {sum(counts)} values into room for {fcap}")
                full[:cat.numel()].copy_(cat)
            for r, c in enumerate(counts):
                counts_ptr[r] = int(c)
        except BaseException as exc:  # noqa: BLE001 (reported by check())
            if self.error is None:
                self.error = exc
            counts_ptr[0] = -1  # a size the library rejects: the evaluation stops with an error


class ShardedInversePower(BasePotential):
    """InversePower (fresco/potentials/inversepower_potential.pyx:16-79, cell lists) over one pattern
    split into index slabs: this rank owns points [lo, hi) of the pattern whose radii `radii_all` are
    given, and takes its slab's coordinates.  The slabs of the ranks, in rank order, must tile
    [0, n_total).  Combines with a ShardedNUwU in a CombinedPotential for ShardedLBFGS; every rank
    holds the pattern's energy and its slab's gradient.

    halo=False: each evaluation all-gathers the slabs and evaluates the whole pattern's repulsion
    (any box, any order of the points).
    halo=True (periodic box of at least 3 cells per dimension): each evaluation exchanges only the
    points next to another rank's points (a halo; see fresco_inversepower_halo_create) and evaluates
    this slab's pairs.  It is small when the slabs are spatial slabs: order the points with
    spatial_order before the split.  `rank` and `nranks` default to the group's."""

    def __init__(self, a, eps, radii_all, boxv, lo, hi, group=None, exchange=None, method=Distance.PERIODIC,
                 halo=False, rank=None, nranks=None):
        self.a, self.eps = float(a), float(eps)
        self.radii = _f64(radii_all)
        self.boxv = _f64(boxv)
        self.ndim = self.boxv.size
        self.lo, self.hi = int(lo), int(hi)
        self.N = self.hi - self.lo
        self.n_total = self.radii.size
        self.halo = bool(halo)
        dist = _dist(group)
        slabs = None
        if dist is not None and exchange is None:
            slabs = [None] * dist.get_world_size(group)
            dist.all_gather_object(slabs, (self.lo, self.hi), group=group)
            ends = [0] + [h for _, h in slabs]
            if any(l != e for (l, _), e in zip(slabs, ends)) or ends[-1] != self.n_total:
                raise ValueError("the ranks' slabs must tile [0, n_total) in rank order")
        elif exchange is None and (self.lo, self.hi) != (0, self.n_total):
            raise ValueError("a slab of a larger pattern needs a multi-rank process group or an exchange")
        periodic = method == Distance.PERIODIC if isinstance(method, Distance) else \
            str(getattr(method, "name", method)).upper().endswith("PERIODIC")
        h = _lib.handle_t()
        if self.halo:
            if not periodic:
                raise ValueError("the halo exchange needs a periodic box")
            if exchange is None:
                exchange = HaloExchange(group)
            if rank is None or nranks is None:
                if dist is not None:
                    rank, nranks = dist.get_rank(group), dist.get_world_size(group)
                elif exchange.gatherv_fn is None:
                    rank, nranks = 0, 1
                else:
                    raise ValueError("an exchange without a process group needs rank and nranks")
            self.rank, self.nranks = int(rank), int(nranks)
            self.exchange = exchange
            check(lib.fresco_inversepower_halo_create(self.a, self.eps, dptr(self.radii), self.n_total,
                                                      dptr(self.boxv), self.ndim, self.lo, self.hi, self.rank,
                                                      self.nranks, C.cast(exchange.c_gatherv, C.c_void_p),
                                                      C.cast(exchange.c_fn, C.c_void_p), None, C.byref(h)))
        else:
            if exchange is None:
                exchange = Exchange(group)
                if slabs is not None:
                    exchange.counts = [(hh - ll) * self.ndim for ll, hh in slabs]
            self.exchange = exchange
            check(lib.fresco_inversepower_shard_create(self.a, self.eps, dptr(self.radii), self.n_total,
                                                       dptr(self.boxv), self.ndim, int(periodic), self.lo, self.hi,
                                                       C.cast(exchange.c_gather, C.c_void_p),
                                                       C.cast(exchange.c_fn, C.c_void_p), None, C.byref(h)))
        self._set_handle(h)

    def halo_stats(self):
        """(points exported, halo points kept) in the last evaluation of a halo=True shard."""
        e, k = C.c_int64(), C.c_int64()
        check(lib.fresco_inversepower_halo_stats(self._h, C.byref(e), C.byref(k)))
        return int(e.value), int(k.value)

    def get_energy(self, x):
        try:
            return super().get_energy(x)
        finally:
            self.exchange.check()

    def get_energy_gradient(self, x, out=None):
        try:
            return super().get_energy_gradient(x, out=out)
        finally:
            self.exchange.check()


def _enable_reducer(shard, reducer):
    check(lib.fresco_potential_set_reducer(shard._h, C.cast(reducer.c_fn, C.c_void_p), None))
    shard._reducer = reducer


class ShardedLBFGS:
    """LBFGS_CPP (fresco/optimize/_lbfgs_cpp.pyx:38-84, source/lbfgs.cpp:9-258) over one pattern split
    between processes: this rank's coordinates `x_local` and its `ShardedNUwU`.  The device LBFGS runs
    on every rank with its slab of x; each of its dot products (two-loop recursion, step norm, accept
    test, rms over all n_total * ndim coordinates) has its block partial sums all-reduced before use,
    and each evaluation all-reduces the shard's rho.  Every rank therefore sees the same scalars and
    takes the same steps: the trajectory is the single-process one, up to the order of the sums.
    `reducer`: a `Reducer` (default: all-reduce over `group`).  The result methods are those of
    LBFGS_CPP, with this rank's coordinates and gradient."""

    def __init__(self, x_local, shard, tol=1e-5, M=4, maxstep=0.1, maxErise=1e-4, H0=0.1, iprint=-1,
                 nsteps=10000, verbosity=0, rel_energy=False, group=None, reducer=None, events=None):
        from .optimize import GradientOptimizer

        x = _f64(x_local)
        parts = list(shard._parts) if isinstance(shard, CombinedPotential) else [shard]
        nuwu = [p for p in parts if isinstance(p, ShardedNUwU)]
        rep = [p for p in parts if isinstance(p, ShardedInversePower)]
        if not nuwu and not rep:
            raise ValueError("ShardedLBFGS expects a ShardedNUwU or a CombinedPotential of sharded potentials")
        first = (nuwu or rep)[0]
        if x.size != first.N * first.ndim:
            raise ValueError(f"expected {first.N * first.ndim} coordinates, got {x.size}")
        total_ndof = int(first.n_total) * first.ndim
        self.shard = shard
        self.reducer = reducer if reducer is not None else Reducer(group)
        # one process holding the whole pattern has nothing to exchange: no hooks
        hooks = self.reducer.active()
        for p in nuwu:
            if hooks:
                _enable_reducer(p, self.reducer)
            elif p.n_total != p.N:
                raise ValueError("a shard of a larger pattern needs a multi-rank process group or a reducer")
        h = _lib.handle_t()
        check(lib.fresco_lbfgs_create(shard._h, dptr(x), x.size, float(tol), int(M), float(maxstep),
                                      float(maxErise), float(H0), int(bool(rel_energy)), int(nsteps), int(iprint),
                                      int(verbosity), C.byref(h)))
        self._opt = GradientOptimizer()
        self._opt._h = h
        self._opt._n = x.size
        self._opt.events = [] if events is None else events
        if hooks:
            check(lib.fresco_optimizer_set_reducer(h, C.cast(self.reducer.c_fn, C.c_void_p), None, total_ndof))

    def _checked(self, f, *a):
        try:
            return f(*a)
        finally:
            self.reducer.check()
            parts = list(self.shard._parts) if isinstance(self.shard, CombinedPotential) else [self.shard]
            for p in parts:
                if isinstance(p, ShardedInversePower):
                    p.exchange.check()

    def run(self, niter=None):
        return self._checked(self._opt.run, niter)

    def one_iteration(self):
        return self._checked(self._opt.one_iteration)

    def get_result(self):
        return self._checked(self._opt.get_result)

    def stop_criterion_satisfied(self):
        return self._checked(self._opt.stop_criterion_satisfied)

    def save_state(self):
        return self._opt.save_state()

    def load_state(self, image):
        self._opt.load_state(image)

    def get_niter(self):
        return self._opt.get_niter()

    def get_maxiter(self):
        return self._opt.get_maxiter()
