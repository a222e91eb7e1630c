"""Batched ensembles of independent 2D NUwU patterns, and their sharding over ranks.

``NUwUEnsemble`` holds P patterns, each the argument set of one
``fresco.potentials.NUwU(radii, K, Sk, V, L, eps)`` (fresco/potentials/nuwu.pyx:10-23)
with its own point count and mode grid, in one common box ``L``, and evaluates
all of them with one set of launches per group of equal mode grids.
``EnsembleLBFGS`` runs ``LBFGS_CPP(x0_p, NUwU_p, ...).run(niter)``
(fresco/optimize/_lbfgs_cpp.pyx:38-84, opt.pyx:26-54) for every pattern at once,
with each pattern's LBFGS state on the device; a step (one evaluation of every
pattern) is one CUDA graph launch.  Per pattern, energies, gradients and
trajectories are those of the single-pattern classes.

The coordinates of all patterns form one vector, pattern p at
``x[offsets[p]:offsets[p+1]]``; every call also accepts a list of per-pattern
arrays.

Across ranks (one process per GPU) the patterns are independent:
``shard_patterns`` assigns them by a cost model (longest processing time
first, cost N w^2 + G log2 G per pattern) and ``gather_results`` collects the
per-pattern results on every rank.  Nothing on the data path is a collective.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import _lib
from ._lib import check, dptr, lib
from .optimize import DeviceLBFGS, Result
from .potentials import _f64, _precision

__all__ = ["NUwUEnsemble", "EnsembleLBFGS", "pattern_cost", "shard_patterns", "gather_results"]


def _i64(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.int64).ravel())


class NUwUEnsemble:
    """P NUwU losses evaluated together (batched form of fresco/potentials/nuwu.pyx:9-44).

    ``radii``, ``Sk`` and ``V`` are sequences with one entry per pattern (``Sk[p]``
    and ``V[p]`` flat, x fastest, of length (2K_p+1)^2 as for ``NUwU``); ``K``
    is a number or one per pattern and, as in the reference, unused (the mode
    grid follows from len(V_p)).  ``L`` is the common box.
    """

    def __init__(self, radii, K, Sk, V, L, eps=1e-6, precision="fp64"):
        self.radii = [_f64(r) for r in radii]
        P = len(self.radii)
        if P < 1:
            raise ValueError("an ensemble needs at least one pattern")
        self.K = [float(k) for k in (K if np.ndim(K) else [K] * P)]
        self.Sk = [_f64(s) for s in Sk]
        self.V = [_f64(v) for v in V]
        if len(self.Sk) != P or len(self.V) != P or len(self.K) != P:
            raise ValueError("radii, K, Sk and V need one entry per pattern")
        for s, v in zip(self.Sk, self.V):
            assert len(s) == len(v)
        self.L = _f64(L)
        self.ndim = len(self.L)
        self.eps = float(eps)
        self.precision = str(precision)
        npts = _i64([len(r) for r in self.radii])
        nmodes = _i64([len(v) for v in self.V])
        allr = np.ascontiguousarray(np.concatenate(self.radii))
        allsk = np.ascontiguousarray(np.concatenate(self.Sk))
        allv = np.ascontiguousarray(np.concatenate(self.V))
        h = _lib.handle_t()
        check(lib.fresco_nuwu_ensemble_create(P, npts.ctypes.data_as(C.POINTER(C.c_int64)), dptr(allr),
                                              nmodes.ctypes.data_as(C.POINTER(C.c_int64)), dptr(allsk), dptr(allv),
                                              dptr(self.L), self.ndim, self.eps, _precision(precision), C.byref(h)))
        self._h = h
        off = np.zeros(P + 1, dtype=np.int64)
        check(lib.fresco_ensemble_info(self._h, None, None, off.ctypes.data_as(C.POINTER(C.c_int64))))
        self.offsets = off

    def __del__(self):
        h, self._h = getattr(self, "_h", None), None
        if h:
            try:
                lib.fresco_ensemble_destroy(h)
            except Exception:
                pass

    def __reduce__(self):
        return (self.__class__, (self.radii, self.K, self.Sk, self.V, self.L, self.eps, self.precision), {})

    def __setstate__(self, d):
        pass

    @property
    def handle(self):
        return self._h

    @property
    def n_patterns(self):
        return len(self.offsets) - 1

    @property
    def ndof(self):
        return int(self.offsets[-1])

    def concat(self, x):
        """One float64 vector from a list of per-pattern coordinate arrays (or a flat vector)."""
        if isinstance(x, (list, tuple)):
            if len(x) != self.n_patterns:
                raise ValueError("one coordinate array per pattern expected")
            x = np.concatenate([_f64(a) for a in x])
        x = _f64(x)
        if x.size != self.ndof:
            raise ValueError(f"the coordinate array has size {x.size}, the ensemble expects {self.ndof}")
        return x

    def split(self, x):
        """Per-pattern views of a vector in the ensemble's layout."""
        return [x[self.offsets[p]:self.offsets[p + 1]] for p in range(self.n_patterns)]

    def get_energies(self, x):
        x = self.concat(x)
        e = np.empty(self.n_patterns)
        check(lib.fresco_ensemble_energy_gradient(self._h, dptr(x), x.size, None, dptr(e)))
        return e

    def get_energies_gradient(self, x, out=None):
        """(energies[P], gradient in the x layout); ``out`` may receive the gradient."""
        x = self.concat(x)
        g = np.empty(x.size) if out is None else out
        if g.dtype != np.float64 or not g.flags.c_contiguous or g.size != x.size:
            raise ValueError("out must be a C-contiguous float64 array of the coordinate size")
        e = np.empty(self.n_patterns)
        check(lib.fresco_ensemble_energy_gradient(self._h, dptr(x), x.size, dptr(g), dptr(e)))
        return e, g

    def get_energies_gradient_device(self, x, grad, energies, stream=0):
        """Device-pointer form (torch CUDA tensors or raw pointers), asynchronous on ``stream``."""
        def ptr(t):
            return t.data_ptr() if hasattr(t, "data_ptr") else int(t)
        check(lib.fresco_ensemble_energy_gradient_device(self._h, C.c_void_p(ptr(x)), self.ndof,
                                                         C.c_void_p(ptr(grad)), C.c_void_p(ptr(energies)),
                                                         C.c_void_p(int(stream))))

    def tune(self, x):
        """Times the tiled / direct spreading split per group on x and keeps the fastest."""
        x = self.concat(x)
        check(lib.fresco_ensemble_tune(self._h, dptr(x), x.size))

    def set_split(self, ratio):
        """Patterns whose tap work N w^2 is below ``ratio`` x the tile cells of
        their bins use the direct kernels (0: all tiled; ``tune`` picks it)."""
        check(lib.fresco_ensemble_set_split(self._h, float(ratio)))

    def set_subproblem_cap(self, cap):
        """Largest subproblem of the tile kernels (points per block, 160..640); ``tune`` picks it
        per group of equal grids together with the split."""
        check(lib.fresco_ensemble_set_subproblem_cap(self._h, int(cap)))

    def status(self):
        """Per-pattern status bits raised since the last call (1: non-finite coordinate)."""
        st = np.zeros(self.n_patterns, dtype=np.int32)
        check(lib.fresco_ensemble_status(self._h, st.ctypes.data_as(C.POINTER(C.c_int))))
        return st

    def describe(self):
        buf = C.create_string_buffer(4096)
        check(lib.fresco_ensemble_describe(self._h, buf, len(buf)))
        return buf.value.decode()


class EnsembleLBFGS(DeviceLBFGS):
    """``LBFGS_CPP.run(niter)`` for every pattern of a ``NUwUEnsemble`` at once.

    Parameters and defaults as fresco/optimize/_lbfgs_cpp.pyx:43 (tol, M,
    maxstep, maxErise, H0, rel_energy).  ``x0`` is a flat vector in the
    ensemble's layout or a list of per-pattern arrays.
    """

    def __init__(self, x0, ensemble, tol=1e-5, M=4, maxstep=0.1, maxErise=1e-4, H0=0.1, rel_energy=False):
        if not isinstance(ensemble, NUwUEnsemble):
            raise TypeError("ensemble must be a NUwUEnsemble")
        self.ensemble = ensemble
        x = ensemble.concat(x0)
        self._ndof = x.size
        self._npat = ensemble.n_patterns
        self.tol = float(tol)
        h = _lib.handle_t()
        check(lib.fresco_ensemble_lbfgs_create(ensemble.handle, dptr(x), x.size, self.tol, int(M), float(maxstep),
                                               float(maxErise), float(H0), int(bool(rel_energy)), C.byref(h)))
        self._h = h

    def get_results(self):
        """One ``Result`` per pattern, as ``LBFGS_CPP.get_result()`` (opt.pyx:81-93)."""
        x, g, f, rms, it, nfev, _ = self.state(True)
        out = []
        for p, (xs, gs) in enumerate(zip(self.ensemble.split(x), self.ensemble.split(g))):
            r = Result()
            r.energy = float(f[p])
            r.coords = xs.copy()
            r.grad = gs.copy()
            r.rms = float(rms[p])
            r.nsteps = int(it[p])
            r.nfev = int(nfev[p])
            r.success = bool(rms[p] <= self.tol)
            out.append(r)
        return out


def pattern_cost(n_points, n_modes_per_dim, w=7):
    """Relative cost of one evaluation: spreading + interpolation N w^2 and the
    two transforms of the fine grid G log2 G (nf about 2 n)."""
    nf = 2 * int(n_modes_per_dim)
    G = nf * nf
    return float(n_points) * w * w + G * math.log2(max(G, 2))


def shard_patterns(costs, world_size):
    """Longest-processing-time-first assignment of patterns to ranks.

    Returns one sorted list of pattern indices per rank; every pattern appears
    exactly once and the heaviest rank carries at most 4/3 of the optimum.
    """
    if world_size < 1:
        raise ValueError("world_size must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i))
    load = [0.0] * world_size
    parts = [[] for _ in range(world_size)]
    for i in order:
        r = min(range(world_size), key=lambda k: (load[k], k))
        parts[r].append(i)
        load[r] += float(costs[i])
    return [sorted(p) for p in parts]


def gather_results(local, indices, group=None):
    """Collects ``{pattern index: result}`` from every rank (torch.distributed
    all_gather_object); returns the results ordered by pattern index."""
    import torch.distributed as dist

    mine = dict(zip(indices, local))
    if dist.is_available() and dist.is_initialized() and dist.get_world_size(group) > 1:
        parts = [None] * dist.get_world_size(group)
        dist.all_gather_object(parts, mine, group=group)
    else:
        parts = [mine]
    merged = {}
    for d in parts:
        merged.update(d)
    return [merged[i] for i in sorted(merged)]
