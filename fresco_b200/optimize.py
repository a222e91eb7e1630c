"""Drop-in counterparts of ``fresco.optimize`` with device-resident state.

Mirrors fresco/optimize/_lbfgs_cpp.pyx:38-84 (``LBFGS_CPP``),
_modified_fire_cpp.pyx:13-44 (``ModifiedFireCPP``), opt.pyx:17-93
(``GradientOptimizer``) and result.py:10-87 (``Result``).  The optimiser's
x, g and memory live in HBM; the C++ driver (libfresco_b200) calls the
potential on the device without any host round trip of the vectors.

Checkpointing (``run(isave=..., file_name=...)``): the reference dumps the
coordinates with hickle to ``<file_name>_odd.hkl`` / ``_even.hkl``
alternately (opt.pyx:42-54).  hickle is not a dependency here; the same
alternation is written with ``numpy.save`` to ``<file_name>_odd.npy`` /
``_even.npy``.
"""
from __future__ import annotations

import copy
import ctypes as C

import numpy as np

from . import _lib
from ._lib import check, dptr, lib
from .potentials import BasePotential

__all__ = ["Result", "GradientOptimizer", "LBFGS_CPP", "ModifiedFireCPP", "ModifiedFire_Graph", "LBFGS_Graph"]


class Result(dict):
    """Container of optimiser results (fresco/optimize/result.py:10-87)."""

    def __getattr__(self, name):
        try:
            return self[name]
        except KeyError:
            raise AttributeError(name)

    __setattr__ = dict.__setitem__
    __delattr__ = dict.__delitem__

    def __repr__(self):
        if list(self.keys()):
            m = max(map(len, list(self.keys()))) + 1
            return "\n".join([k.rjust(m) + ": " + repr(v) for k, v in self.items()])
        return self.__class__.__name__ + "()"

    def __getitem__(self, i):
        if isinstance(i, slice):
            return tuple(self[j] for j in range(*i.indices(5)))
        if i in range(4):
            i = {0: "coords", 1: "energy", 2: "rms", 3: "nfev"}[i]
        elif i == 4:
            return self
        return dict.__getitem__(self, i)

    def __iter__(self):
        return iter((self.coords, self.energy, self.rms, self.nfev, self))


class GradientOptimizer:
    """Python interface of the device optimisers (fresco/optimize/opt.pyx:17-93)."""

    _h = None
    res = None

    def __del__(self):
        h, self._h = self._h, None
        if h:
            try:
                lib.fresco_optimizer_destroy(h)
            except Exception:
                pass

    def one_iteration(self):
        check(lib.fresco_optimizer_one_iteration(self._h))
        self.res = self.get_result()
        for event in self.events:
            event(coords=self.res.coords, energy=self.res.energy, rms=self.res.rms)
        return self.res

    def run(self, niter=None, isave=None, file_name="unknown"):
        if not self.events:
            if niter is None and isave is None:
                check(lib.fresco_optimizer_run(self._h, -1))
            elif isave is None:
                check(lib.fresco_optimizer_run(self._h, int(niter)))
            else:
                if niter is None:
                    niter = self.get_maxiter() - self.get_niter()
                i = 0
                odd = True
                while i < niter:
                    check(lib.fresco_optimizer_run(self._h, int(isave)))
                    self.res = self.get_result()
                    np.save(file_name + ("_odd.npy" if odd else "_even.npy"), np.asarray(self.res.coords))
                    i += isave
                    odd = not odd
            self.res = self.get_result()
        else:
            if niter is None:
                niter = self.get_maxiter() - self.get_niter()
            for _ in range(niter):
                if self.stop_criterion_satisfied():
                    break
                self.res = self.one_iteration()
        return copy.deepcopy(self.res)

    def reset(self, coords):
        x = np.ascontiguousarray(np.asarray(coords, dtype=np.float64).ravel())
        check(lib.fresco_optimizer_reset(self._h, dptr(x), x.size))

    def stop_criterion_satisfied(self):
        out = C.c_int(0)
        check(lib.fresco_optimizer_stop_criterion_satisfied(self._h, C.byref(out)))
        return bool(out.value)

    def _state(self, want_vectors=True):
        x = np.empty(self._n) if want_vectors else None
        g = np.empty(self._n) if want_vectors else None
        f = C.c_double()
        rms = C.c_double()
        nfev = C.c_int()
        niter = C.c_int()
        maxiter = C.c_int()
        h0 = C.c_double()
        check(lib.fresco_optimizer_get_state(self._h, dptr(x) if want_vectors else None,
                                             dptr(g) if want_vectors else None, C.byref(f), C.byref(rms),
                                             C.byref(nfev), C.byref(niter), C.byref(maxiter), C.byref(h0)))
        return x, g, f.value, rms.value, nfev.value, niter.value, maxiter.value, h0.value

    def get_maxiter(self):
        return self._state(False)[6]

    def get_niter(self):
        return self._state(False)[5]

    def get_result(self):
        x, g, f, rms, nfev, niter, _, _ = self._state(True)
        res = Result()
        res.energy = f
        res.coords = x
        res.grad = g
        res.rms = rms
        res.nsteps = niter
        res.nfev = nfev
        res.success = bool(self.stop_criterion_satisfied())
        return res

    def save_state(self):
        """Exact-resume image of the optimiser's device state and counters (uint8 array): x, g, the LBFGS
        memory pairs or the FIRE velocities and step sizes.  No reference counterpart (the reference
        checkpoints coordinates only, opt.pyx:42-54)."""
        nb = C.c_int64()
        check(lib.fresco_optimizer_state_bytes(self._h, C.byref(nb)))
        img = np.empty(nb.value, dtype=np.uint8)
        check(lib.fresco_optimizer_save_state(self._h, img.ctypes.data_as(C.c_void_p)))
        return img

    def load_state(self, image):
        """Continues the trajectory saved by save_state (same family, coordinate count and memory length;
        this optimiser keeps its own parameters)."""
        img = np.ascontiguousarray(np.asarray(image, dtype=np.uint8).ravel())
        check(lib.fresco_optimizer_load_state(self._h, img.ctypes.data_as(C.c_void_p), img.size))
        self.res = None

    def save_checkpoint(self, file_name):
        """save_state() written to `file_name` (numpy .npy)."""
        np.save(file_name, self.save_state())

    def load_checkpoint(self, file_name):
        self.load_state(np.load(file_name))

    def device_state(self):
        """(x, g) device pointers of the optimiser state."""
        dx = C.c_void_p()
        dg = C.c_void_p()
        check(lib.fresco_optimizer_device_state(self._h, C.byref(dx), C.byref(dg)))
        return dx.value, dg.value


def _as_potential(potential):
    if not isinstance(potential, BasePotential):
        raise TypeError("the potential must be a fresco_b200 potential (Python-callback potentials are not supported)")
    return potential


class LBFGS_CPP(GradientOptimizer):
    """LBFGS with backtracking line search (fresco/optimize/_lbfgs_cpp.pyx:38-84)."""

    def __init__(self, x0, potential, tol=1e-5, M=4, maxstep=0.1, maxErise=1e-4, H0=0.1, iprint=-1,
                 energy=None, gradient=None, nsteps=10000, verbosity=0, events=None, logger=None,
                 rel_energy=False):
        self.pot = _as_potential(potential)
        if logger is not None:
            print("warning c++ LBFGS is ignoring logger")
        x = np.ascontiguousarray(np.asarray(x0, dtype=np.float64).ravel())
        self._n = x.size
        h = _lib.handle_t()
        check(lib.fresco_lbfgs_create(self.pot.handle, dptr(x), x.size, float(tol), int(M), float(maxstep),
                                      float(maxErise), float(H0), int(bool(rel_energy)), int(nsteps), int(iprint),
                                      int(verbosity), C.byref(h)))
        self._h = h
        if energy is not None and gradient is not None:
            g = np.ascontiguousarray(np.asarray(gradient, dtype=np.float64).ravel())
            check(lib.fresco_optimizer_set_func_gradient(self._h, float(energy), dptr(g), g.size))
        self.events = [] if events is None else events

    def set_H0(self, H0):
        """LBFGS::set_H0 (fresco/optimize/_lbfgs_cpp.pyx:72-74): the inverse-Hessian scale of the next step."""
        check(lib.fresco_lbfgs_set_H0(self._h, float(H0)))

    def get_result(self):
        res = super().get_result()
        res["H0"] = float(self._state(False)[7])
        return res


class ModifiedFireCPP(GradientOptimizer):
    """Modified FIRE (fresco/optimize/_modified_fire_cpp.pyx:13-44)."""

    def __init__(self, x0, potential, dtstart=0.1, dtmax=1, maxstep=0.5, Nmin=5, finc=1.1, fdec=0.5, fa=0.99,
                 astart=0.1, tol=1e-3, stepback=True, iprint=-1, energy=None, gradient=None, nsteps=10000,
                 verbosity=0, events=None):
        self.pot = _as_potential(potential)
        x = np.ascontiguousarray(np.asarray(x0, dtype=np.float64).ravel())
        self._n = x.size
        h = _lib.handle_t()
        check(lib.fresco_fire_create(self.pot.handle, dptr(x), x.size, float(dtstart), float(dtmax),
                                     float(maxstep), int(Nmin), float(finc), float(fdec), float(fa), float(astart),
                                     float(tol), int(bool(stepback)), int(nsteps), int(iprint), int(verbosity),
                                     C.byref(h)))
        self._h = h
        if energy is not None and gradient is not None:
            g = np.ascontiguousarray(np.asarray(gradient, dtype=np.float64).ravel())
            check(lib.fresco_optimizer_set_func_gradient(self._h, float(energy), dptr(g), g.size))
        self.events = [] if events is None else events


class ModifiedFire_Graph(GradientOptimizer):
    """ModifiedFireCPP with each iteration one CUDA graph launch: same arguments (iprint and verbosity
    are accepted and ignored), same trajectory, iterations and evaluations."""

    def __init__(self, x0, potential, dtstart=0.1, dtmax=1, maxstep=0.5, Nmin=5, finc=1.1, fdec=0.5, fa=0.99,
                 astart=0.1, tol=1e-3, stepback=True, iprint=-1, energy=None, gradient=None, nsteps=10000,
                 verbosity=0, events=None):
        self.pot = _as_potential(potential)
        x = np.ascontiguousarray(np.asarray(x0, dtype=np.float64).ravel())
        self._n = x.size
        h = _lib.handle_t()
        check(lib.fresco_fire_graph_create(self.pot.handle, dptr(x), x.size, float(dtstart), float(dtmax),
                                           float(maxstep), int(Nmin), float(finc), float(fdec), float(fa),
                                           float(astart), float(tol), int(bool(stepback)), int(nsteps), C.byref(h)))
        self._h = h
        if energy is not None and gradient is not None:
            g = np.ascontiguousarray(np.asarray(gradient, dtype=np.float64).ravel())
            check(lib.fresco_optimizer_set_func_gradient(self._h, float(energy), dptr(g), g.size))
        self.events = [] if events is None else events


class DeviceLBFGS:
    """Driver of the device-state LBFGS (ensemble_lbfgs.cu): every pattern's
    iteration (lbfgs.cpp:9-258) is a state machine on the device, and one
    step (one evaluation of every pattern) is one CUDA graph launch."""

    _h = None
    _ndof = 0
    _npat = 1

    def __del__(self):
        h, self._h = self._h, None
        if h:
            try:
                lib.fresco_ensemble_lbfgs_destroy(h)
            except Exception:
                pass

    def run(self, niter):
        """Every pattern iterates until rms <= tol or ``niter`` more iterations
        (optimizer.hpp:97-112); returns the number of evaluation steps used."""
        steps = C.c_int(0)
        check(lib.fresco_ensemble_lbfgs_run(self._h, int(niter), C.byref(steps)))
        return steps.value

    def steps(self, n):
        """Exactly ``n`` steps (one evaluation of every pattern each)."""
        check(lib.fresco_ensemble_lbfgs_steps(self._h, int(n)))

    def state(self, with_vectors=True):
        """(x, g, f, rms, iterations, evaluations, active) with per-pattern arrays."""
        P, n = self._npat, self._ndof
        x = np.empty(n) if with_vectors else None
        g = np.empty(n) if with_vectors else None
        f = np.empty(P)
        rms = np.empty(P)
        it = np.zeros(P, dtype=np.int32)
        nfev = np.zeros(P, dtype=np.int32)
        active = np.zeros(P, dtype=np.int32)
        ip = C.POINTER(C.c_int)
        check(lib.fresco_ensemble_lbfgs_state(self._h, dptr(x) if with_vectors else None,
                                              dptr(g) if with_vectors else None, dptr(f), dptr(rms),
                                              it.ctypes.data_as(ip), nfev.ctypes.data_as(ip),
                                              active.ctypes.data_as(ip)))
        return x, g, f, rms, it, nfev, active


class LBFGS_Graph(DeviceLBFGS):
    """``LBFGS_CPP`` (fresco/optimize/_lbfgs_cpp.pyx:38-84) with the whole iteration on the device.

    Same parameters, iterations, evaluation counts and trajectory as
    ``LBFGS_CPP``; ``run(niter)`` replays one CUDA graph per evaluation
    (direction, trial point, potential, accept test, memory update) and reads
    the iteration state back only every few evaluations.  No per-iteration
    printing or event callbacks.
    """

    def __init__(self, x0, potential, tol=1e-5, M=4, maxstep=0.1, maxErise=1e-4, H0=0.1, rel_energy=False):
        self.pot = _as_potential(potential)
        x = np.ascontiguousarray(np.asarray(x0, dtype=np.float64).ravel())
        self._ndof = x.size
        self.tol = float(tol)
        h = _lib.handle_t()
        check(lib.fresco_lbfgs_graph_create(self.pot.handle, dptr(x), x.size, self.tol, int(M), float(maxstep),
                                            float(maxErise), float(H0), int(bool(rel_energy)), C.byref(h)))
        self._h = h

    def get_result(self):
        x, g, f, rms, it, nfev, _ = self.state(True)
        res = Result()
        res.energy = float(f[0])
        res.coords = x
        res.grad = g
        res.rms = float(rms[0])
        res.nsteps = int(it[0])
        res.nfev = int(nfev[0])
        res.success = bool(rms[0] <= self.tol)
        return res

