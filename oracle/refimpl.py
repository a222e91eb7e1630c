"""ctypes access to oracle/_ref/libfresco_ref.so (test infrastructure only).

The library is the reference's own C++ for the loss-and-gradient path,
compiled unchanged by ``oracle/Makefile`` against this folder's FINUFFT/FFTW
API shim.  It pins the numpy restatement (oracle.py) and is
the CPU baseline timed by ``bench.py``.  Transforms run either as exact FP64
direct sums (``set_mode(EXACT)``) or as the CPU ES-kernel NUFFT restatement at
the plan tolerance (``set_mode(ES)``); FINUFFT itself is not available here.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

LIB_PATH = Path(__file__).resolve().parent / "_ref" / "libfresco_ref.so"

AUTO, EXACT, ES = 0, 1, 2

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)
_lib = None


def available() -> bool:
    return LIB_PATH.exists()


def lib():
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise FileNotFoundError(f"{LIB_PATH} not built (make -C oracle)")
        L = C.CDLL(str(LIB_PATH))
        sig = {
            "fresco_shim_set_mode": (None, [C.c_int]),
            "fresco_shim_profile": (None, [_dp, C.c_int]),
            "fresco_shim_get_mode": (C.c_int, []),
            "ref_set_threads": (None, [C.c_int]),
            "ref_get_threads": (C.c_int, []),
            "ref_nuwu_create": (C.c_void_p, [_dp, C.c_int64, C.c_double, _dp, _dp, C.c_int64, _dp, C.c_int,
                                             C.c_double]),
            "ref_uwu_create": (C.c_void_p, [_ip, C.c_int, C.c_double, _dp, _dp, C.c_int64, _dp, C.c_double]),
            "ref_uwnu_create": (C.c_void_p, [_ip, C.c_int, _dp, C.c_int64, _dp, _dp, _dp, C.c_double]),
            "ref_nuwnu_create": (C.c_void_p, [_dp, C.c_int64, _dp, C.c_int64, _dp, _dp, _dp, C.c_int, C.c_double]),
            "ref_inversepower_create": (C.c_void_p, [C.c_double, C.c_double, _dp, C.c_int64, _dp, C.c_int, C.c_int,
                                                     C.c_int, C.c_double]),
            "ref_combined_create": (C.c_void_p, []),
            "ref_combined_add": (None, [C.c_void_p, C.c_void_p]),
            "ref_energy": (C.c_double, [C.c_void_p, _dp, C.c_int64]),
            "ref_energy_gradient": (C.c_double, [C.c_void_p, _dp, C.c_int64, _dp]),
            "ref_destroy": (None, [C.c_void_p]),
            "ref_lbfgs_create": (C.c_void_p, [C.c_void_p, _dp, C.c_int64, C.c_double, C.c_int, C.c_double,
                                              C.c_double, C.c_double, C.c_int, C.c_int]),
            "ref_fire_create": (C.c_void_p, [C.c_void_p, _dp, C.c_int64, C.c_double, C.c_double, C.c_double, C.c_int,
                                             C.c_double, C.c_double, C.c_double, C.c_double, C.c_double, C.c_int,
                                             C.c_int]),
            "ref_lbfgs_set_H0": (None, [C.c_void_p, C.c_double]),
            "ref_opt_run": (None, [C.c_void_p, C.c_int]),
            "ref_opt_one_iteration": (None, [C.c_void_p]),
            "ref_opt_state": (None, [C.c_void_p, _dp, _dp, _dp, _dp, _ip, _ip, _dp]),
            "ref_opt_destroy": (None, [C.c_void_p]),
            "ref_pps_create": (C.c_void_p, [_dp, C.c_int64, C.c_int, _dp, C.c_double, C.c_uint64]),
            "ref_pps_run": (None, [C.c_void_p, C.c_int64]),
            "ref_pps_set_seed": (None, [C.c_void_p, C.c_uint64]),
            "ref_pps_get": (None, [C.c_void_p, _dp, _dp, C.POINTER(C.c_uint64)]),
            "ref_pps_destroy": (None, [C.c_void_p]),
            "ref_last_error": (C.c_char_p, []),
            "ref_overlap": (C.c_int64, [_dp, C.c_int64, _dp, C.c_int, C.c_int, C.c_int, C.c_double, _dp,
                                        C.POINTER(C.c_int64), C.c_int64, C.POINTER(C.c_uint64)]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def set_mode(mode: int) -> None:
    lib().fresco_shim_set_mode(int(mode))


def shim_profile(reset: bool = True) -> dict:
    """Seconds spent per stage of the ES-kernel NUFFT since the last reset."""
    out = (C.c_double * 5)()
    lib().fresco_shim_profile(out, int(bool(reset)))
    return dict(zip(("setpts", "spread", "fft", "modes", "interp"), list(out)))


def set_threads(n: int) -> None:
    lib().ref_set_threads(int(n))


def get_threads() -> int:
    return int(lib().ref_get_threads())


def _d(a):
    a = np.ascontiguousarray(np.asarray(a, dtype=np.float64).ravel())
    return a, a.ctypes.data_as(_dp)


class RefPotential:
    _h = None
    _keep = ()

    def __del__(self):
        if self._h:
            lib().ref_destroy(self._h)
            self._h = None

    def get_energy(self, x):
        xa, xp = _d(x)
        return float(lib().ref_energy(self._h, xp, xa.size))

    def get_energy_gradient(self, x):
        xa, xp = _d(x)
        g = np.zeros(xa.size)
        e = lib().ref_energy_gradient(self._h, xp, xa.size, g.ctypes.data_as(_dp))
        return float(e), g


class NUwU(RefPotential):
    def __init__(self, radii, K, Sk, V, L, eps=1e-6):
        r, rp = _d(radii)
        s, sp = _d(Sk)
        v, vp = _d(V)
        l, lp = _d(L)
        self._h = lib().ref_nuwu_create(rp, r.size, float(K), sp, vp, s.size, lp, l.size, float(eps))


class UwU(RefPotential):
    """Takes centred Sk/V and applies ifftshift like fresco/potentials/uwu.pyx:14-15."""

    def __init__(self, N, K, Sk, V, L, eps=1e-6):
        g = np.ascontiguousarray(np.asarray(N, dtype=np.int32).ravel())
        s, sp = _d(np.fft.ifftshift(np.asarray(Sk, dtype=np.float64)))
        v, vp = _d(np.fft.ifftshift(np.asarray(V, dtype=np.float64)))
        l, lp = _d(L)
        self._keep = (g,)
        self._h = lib().ref_uwu_create(g.ctypes.data_as(_ip), g.size, float(K), sp, vp, s.size, lp, float(eps))


class UwNU(RefPotential):
    def __init__(self, N, K, Sk, V, L, eps=1e-6):
        g = np.ascontiguousarray(np.asarray(N, dtype=np.int32).ravel())
        k, kp = _d(K)
        s, sp = _d(Sk)
        v, vp = _d(V)
        l, lp = _d(L)
        self._keep = (g,)
        self._h = lib().ref_uwnu_create(g.ctypes.data_as(_ip), l.size, kp, s.size, sp, vp, lp, float(eps))


class NUwNU(RefPotential):
    def __init__(self, radii, K, Sk, V, L, eps=1e-6):
        r, rp = _d(radii)
        k, kp = _d(K)
        s, sp = _d(Sk)
        v, vp = _d(V)
        l, lp = _d(L)
        self._h = lib().ref_nuwnu_create(rp, r.size, kp, k.size // l.size, sp, vp, lp, l.size, float(eps))


class InversePower(RefPotential):
    def __init__(self, a, eps, radii, boxv, use_cell_lists=False, ncellx_scale=1.0, periodic=True):
        r, rp = _d(radii)
        b, bp = _d(boxv)
        self._h = lib().ref_inversepower_create(float(a), float(eps), rp, r.size, bp, b.size, int(periodic),
                                                int(use_cell_lists), float(ncellx_scale))
        if not self._h:
            raise ValueError("unsupported InversePower configuration")


class CombinedPotential(RefPotential):
    def __init__(self):
        self._h = lib().ref_combined_create()
        self._parts = []

    def add_potential(self, p):
        lib().ref_combined_add(self._h, p._h)
        self._parts.append(p)


class _RefOpt:
    _h = None

    def __del__(self):
        if self._h:
            lib().ref_opt_destroy(self._h)
            self._h = None

    def run(self, niter):
        lib().ref_opt_run(self._h, int(niter))

    def one_iteration(self):
        lib().ref_opt_one_iteration(self._h)

    def state(self):
        x = np.zeros(self.n)
        g = np.zeros(self.n)
        f = C.c_double()
        rms = C.c_double()
        nfev = C.c_int()
        nit = C.c_int()
        h0 = C.c_double()
        lib().ref_opt_state(self._h, x.ctypes.data_as(_dp), g.ctypes.data_as(_dp), C.byref(f), C.byref(rms),
                            C.byref(nfev), C.byref(nit), C.byref(h0))
        return dict(coords=x, grad=g, energy=f.value, rms=rms.value, nfev=nfev.value, nsteps=nit.value, H0=h0.value)


class LBFGS(_RefOpt):
    def __init__(self, x0, pot, tol=1e-5, M=4, maxstep=0.1, maxErise=1e-4, H0=0.1, rel_energy=False, nsteps=10000):
        x, xp = _d(x0)
        self.n = x.size
        self.pot = pot
        self._h = lib().ref_lbfgs_create(pot._h, xp, x.size, tol, M, maxstep, maxErise, H0, int(rel_energy), nsteps)

    def set_H0(self, H0):
        lib().ref_lbfgs_set_H0(self._h, float(H0))


class ModifiedFire(_RefOpt):
    def __init__(self, x0, pot, dtstart=0.1, dtmax=1.0, maxstep=0.5, Nmin=5, finc=1.1, fdec=0.5, fa=0.99,
                 astart=0.1, tol=1e-3, stepback=True, nsteps=10000):
        x, xp = _d(x0)
        self.n = x.size
        self.pot = pot
        self._h = lib().ref_fire_create(pot._h, xp, x.size, dtstart, dtmax, maxstep, Nmin, finc, fdec, fa, astart, tol,
                                        int(stepback), nsteps)


def host_cores() -> int:
    return len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)


class PointPatternStatistics:
    """The reference's PointPatternStatistics<ndim> (point_pattern_statistics.hpp:36-111), built serially."""

    def __init__(self, coords, boxv, radius, rseed):
        x, xp = _d(coords)
        b, bp = _d(boxv)
        self._keep = (x, b)
        self._h = lib().ref_pps_create(xp, x.size // b.size, b.size, bp, float(radius), C.c_uint64(int(rseed)))

    def __del__(self):
        h, self._h = getattr(self, "_h", None), None
        if h and _lib is not None:
            try:
                _lib.ref_pps_destroy(h)
            except Exception:
                pass

    def run(self, n):
        lib().ref_pps_run(self._h, int(n))

    def set_generator_seed(self, seed):
        lib().ref_pps_set_seed(self._h, C.c_uint64(int(seed)))

    def mean_var_count(self):
        m, v, c = C.c_double(), C.c_double(), C.c_uint64()
        lib().ref_pps_get(self._h, C.byref(m), C.byref(v), C.byref(c))
        return m.value, v.value, c.value


def overlapping_particles(radii, boxv, coords, periodic=True, cell_lists=False, ncellx_scale=1.0, changed=None):
    """The reference's CheckOverlap{Periodic,Cartesian}[CellLists] (check_overlap.hpp:24-130,
    check_overlap_cell_lists.hpp:87-180), sorted indices."""
    r, rp = _d(radii)
    b, bp = _d(boxv)
    x, xp = _d(coords)
    ch = np.ascontiguousarray(np.asarray([] if changed is None else changed, dtype=np.int64).ravel())
    out = np.zeros(max(r.size, 1), dtype=np.uint64)
    n = lib().ref_overlap(rp, r.size, bp, b.size, int(periodic), int(cell_lists), float(ncellx_scale), xp,
                          ch.ctypes.data_as(C.POINTER(C.c_int64)), ch.size,
                          out.ctypes.data_as(C.POINTER(C.c_uint64)))
    if n < 0:
        raise RuntimeError(lib().ref_last_error().decode())
    return out[:n].copy()
