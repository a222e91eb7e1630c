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
from .potentials import _f64, _precision


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


class ShardedNUwU:
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
