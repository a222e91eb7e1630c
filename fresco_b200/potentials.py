"""Drop-in counterparts of ``fresco.potentials`` backed by the B200 library.

Class names, constructor signatures, defaults and return conventions follow
the reference's Cython bindings (fresco/potentials/nuwu.pyx:9-44,
uwu.pyx:9-43, uwnu.pyx:9-43, nuwnu.pyx:9-44, combine_potentials.pyx:10-30,
inversepower_potential.pyx:14-91).  Differences, all supersets:

* ``precision`` keyword ("fp64", the default, or "fp32") selects the FP64
  form or the FP32 spread/FFT/interpolation form with FP64 reductions;
* ``get_energy_gradient`` returns the gradient as a float64 ndarray (the
  reference returns its ``vector[double]`` member as a list); given a CUDA
  ``torch.Tensor`` it stays on the device and returns a tensor;
* a NaN/inf coordinate yields NaN energy and gradient (FINUFFT's error code
  is ignored by the reference, nuwu.hpp:191-192).
"""
from __future__ import annotations

import ctypes as C
from enum import Enum, unique

import numpy as np

from . import _lib
from ._lib import check, dptr, lib

__all__ = [
    "BasePotential",
    "NUwU",
    "UwU",
    "UwNU",
    "NUwNU",
    "InversePower",
    "CombinedPotential",
    "Distance",
]

_PREC = {"fp64": 0, "float64": 0, "double": 0, "fp32": 1, "float32": 1, "single": 1}


@unique
class Distance(Enum):
    """fresco/distances/distance_enum.py:3-6."""

    CARTESIAN = 1
    PERIODIC = 2


def _f64(a, name="array"):
    arr = np.ascontiguousarray(np.asarray(a, dtype=np.float64).ravel())
    return arr


def _precision(p):
    try:
        return _PREC[str(p).lower()]
    except KeyError:
        raise ValueError(f"precision must be 'fp64' or 'fp32', got {p!r}") from None


def _is_torch_cuda(x):
    t = type(x)
    return t.__module__.startswith("torch") and getattr(x, "is_cuda", False)


class BasePotential:
    """Common evaluation methods (fresco/potentials/_fresco.pyx:10-24)."""

    _h = None

    def _set_handle(self, h):
        self._h = h

    def __del__(self):
        h, self._h = self._h, None
        if h:
            try:
                lib.fresco_potential_destroy(h)
            except Exception:
                pass

    @property
    def handle(self):
        return self._h

    def ndof(self):
        return int(lib.fresco_potential_ndof(self._h))

    def describe(self) -> str:
        buf = C.create_string_buffer(1024)
        check(lib.fresco_potential_describe(self._h, buf, 1024))
        return buf.value.decode()

    # -- host path ---------------------------------------------------------
    def get_energy(self, x):
        if _is_torch_cuda(x):
            return float(self.energy_device(x).item())
        xa = _f64(x)
        e = C.c_double(0.0)
        check(lib.fresco_potential_energy(self._h, dptr(xa), xa.size, C.byref(e)))
        return e.value

    def get_energy_gradient(self, x, out=None):
        """(energy, gradient).  ``out``: optional C-contiguous float64 array that receives the
        gradient (e.g. page-locked memory for faster transfers); it is also returned."""
        if _is_torch_cuda(x):
            e, g = self.energy_gradient_device(x, grad=out)
            return float(e.item()), g
        xa = _f64(x)
        if out is None:
            grad = np.empty_like(xa)
        else:
            grad = out
            if (not isinstance(grad, np.ndarray) or grad.dtype != np.float64 or grad.size != xa.size
                    or not grad.flags["C_CONTIGUOUS"]):
                raise ValueError("out must be a C-contiguous float64 array of the coordinates' size")
        e = C.c_double(0.0)
        check(lib.fresco_potential_energy_gradient(self._h, dptr(xa), xa.size, dptr(grad), C.byref(e)))
        return e.value, grad

    # -- device path (torch CUDA tensors, asynchronous on the current stream)
    def energy_device(self, x, out=None, accumulate=False, stream=None):
        import torch

        x = x.contiguous()
        if x.dtype != torch.float64:
            raise ValueError("device coordinates must be float64")
        if out is None:
            out = torch.zeros((), dtype=torch.float64, device=x.device)
        s = stream if stream is not None else torch.cuda.current_stream(x.device).cuda_stream
        check(lib.fresco_potential_energy_device(self._h, x.data_ptr(), x.numel(), out.data_ptr(),
                                                 int(accumulate), s))
        return out

    def energy_gradient_device(self, x, grad=None, out=None, accumulate=False, stream=None):
        import torch

        x = x.contiguous()
        if x.dtype != torch.float64:
            raise ValueError("device coordinates must be float64")
        if grad is None:
            grad = torch.empty_like(x)
        if out is None:
            out = torch.zeros((), dtype=torch.float64, device=x.device)
        s = stream if stream is not None else torch.cuda.current_stream(x.device).cuda_stream
        check(lib.fresco_potential_energy_gradient_device(self._h, x.data_ptr(), x.numel(), grad.data_ptr(),
                                                          out.data_ptr(), int(accumulate), s))
        return out, grad

    def set_gradient_mode(self, mode):
        """'reference' (default): the reference's own gradient formula; 'exact': the derivative of the
        energy with respect to the input coordinates (used by fresco_b200.autograd)."""
        m = {"reference": 0, "exact": 1}.get(str(mode).lower(), mode)
        check(lib.fresco_potential_set_gradient_mode(self._h, int(m)))
        self._grad_mode = int(m)

    def gradient_mode(self) -> str:
        return "exact" if getattr(self, "_grad_mode", 0) == 1 else "reference"

    def status(self, stream=None) -> int:
        st = C.c_int(0)
        check(lib.fresco_potential_status(self._h, stream, C.byref(st)))
        return st.value

    def set_timing(self, enabled=True):
        check(lib.fresco_potential_set_timing(self._h, int(bool(enabled))))

    def get_timing(self):
        names = C.create_string_buffer(4096)
        tot = (C.c_double * 64)()
        cnt = (C.c_int * 64)()
        n = C.c_int(0)
        check(lib.fresco_potential_get_timing(self._h, 64, names, 4096, tot, cnt, C.byref(n)))
        raw = names.raw.split(b"\0")
        return {raw[i].decode(): (tot[i], cnt[i]) for i in range(n.value)}


class NUwU(BasePotential):
    """Point pattern vs. uniform k-grid (fresco/potentials/nuwu.pyx:9-44)."""

    def __init__(self, radii, K, Sk, V, L, eps=1e-6, precision="fp64"):
        self.radii = _f64(radii)
        self.N = len(self.radii)
        self.K = float(K)
        self.Sk = _f64(Sk)
        self.V = _f64(V)
        assert len(self.Sk) == len(self.V)
        self.L = _f64(L)
        self.ndim = len(self.L)
        self.eps = float(eps)
        self.precision = str(precision)
        h = _lib.handle_t()
        check(lib.fresco_nuwu_create(dptr(self.radii), self.N, self.K, dptr(self.Sk), dptr(self.V), self.Sk.size,
                                     dptr(self.L), self.ndim, self.eps, _precision(precision), C.byref(h)))
        self._set_handle(h)

    def __reduce__(self):
        return (self.__class__, (self.radii, self.K, self.Sk, self.V, self.L, self.eps, self.precision), {})

    def __setstate__(self, d):
        pass


class UwU(BasePotential):
    """Uniform grid vs. uniform k-grid (fresco/potentials/uwu.pyx:9-43); Sk and V are centred."""

    def __init__(self, N, K, Sk, V, L, eps=1e-6, precision="fp64"):
        self.N = np.asarray(N, dtype=np.int32).ravel()
        self.K = float(K)
        self.Sk_in = np.asarray(Sk, dtype=np.float64)
        self.V_in = np.asarray(V, dtype=np.float64)
        self.Sk = _f64(np.fft.ifftshift(self.Sk_in))
        self.V = _f64(np.fft.ifftshift(self.V_in))
        assert len(self.Sk) == len(self.V)
        self.L = _f64(L)
        self.ndim = len(self.L)
        self.eps = float(eps)
        self.precision = str(precision)
        grid = np.ascontiguousarray(self.N, dtype=np.int32)
        h = _lib.handle_t()
        check(lib.fresco_uwu_create(grid.ctypes.data_as(_lib.c_int_p), len(grid), self.K, dptr(self.Sk),
                                    dptr(self.V), self.Sk.size, dptr(self.L), self.eps, _precision(precision),
                                    C.byref(h)))
        self._set_handle(h)

    def __reduce__(self):
        return (self.__class__, (self.N, self.K, self.Sk_in, self.V_in, self.L, self.eps, self.precision), {})

    def __setstate__(self, d):
        pass


class UwNU(BasePotential):
    """Uniform grid vs. non-uniform k-points (fresco/potentials/uwnu.pyx:9-43)."""

    def __init__(self, N, K, Sk, V, L, eps=1e-6, precision="fp64"):
        self.N = np.asarray(N, dtype=np.int32).ravel()
        self.K = _f64(K)
        self.Sk = _f64(Sk)
        self.V = _f64(V)
        assert len(self.Sk) == len(self.V)
        self.L = _f64(L)
        self.ndim = len(self.L)
        self.eps = float(eps)
        self.precision = str(precision)
        grid = np.ascontiguousarray(self.N, dtype=np.int32)
        h = _lib.handle_t()
        check(lib.fresco_uwnu_create(grid.ctypes.data_as(_lib.c_int_p), self.ndim, dptr(self.K), self.Sk.size,
                                     dptr(self.Sk), dptr(self.V), dptr(self.L), self.eps, _precision(precision),
                                     C.byref(h)))
        self._set_handle(h)

    def __reduce__(self):
        return (self.__class__, (self.N, self.K, self.Sk, self.V, self.L, self.eps, self.precision), {})

    def __setstate__(self, d):
        pass


class NUwNU(BasePotential):
    """Point pattern vs. non-uniform k-points (fresco/potentials/nuwnu.pyx:9-44)."""

    def __init__(self, radii, K, Sk, V, L, eps=1e-6, precision="fp64"):
        self.radii = _f64(radii)
        self.N = len(self.radii)
        self.K = _f64(K)
        self.Sk = _f64(Sk)
        self.V = _f64(V)
        assert len(self.Sk) == len(self.V)
        self.L = _f64(L)
        self.ndim = len(self.L)
        self.eps = float(eps)
        self.precision = str(precision)
        nk = self.K.size // self.ndim
        h = _lib.handle_t()
        check(lib.fresco_nuwnu_create(dptr(self.radii), self.N, dptr(self.K), nk, dptr(self.Sk), dptr(self.V),
                                      dptr(self.L), self.ndim, self.eps, _precision(precision), C.byref(h)))
        self._set_handle(h)

    def __reduce__(self):
        return (self.__class__, (self.radii, self.K, self.Sk, self.V, self.L, self.eps, self.precision), {})

    def __setstate__(self, d):
        pass


def get_ncellsx_scale(radii, boxv, omp_threads=1):
    """Cell-size heuristic of fresco/distances/distance_utils.py:6-18 (informational here)."""
    ndim = len(boxv)
    radii = np.asarray(radii, dtype=np.float64)
    ncellsx_max = max(omp_threads, int(np.power(radii.size, 1.0 / ndim)))
    rcut = np.amax(radii) * 2
    ncellsx = 1 * boxv[0] / rcut
    if ncellsx <= ncellsx_max:
        return 1 if ncellsx >= omp_threads else np.ceil(omp_threads / ncellsx)
    return ncellsx_max / ncellsx


class InversePower(BasePotential):
    """Soft-sphere repulsion (fresco/potentials/inversepower_potential.pyx:14-91).

    E = sum over pairs with r < r_i + r_j of eps/a (1 - r/(r_i + r_j))^a
    (source/fresco/inversepower_potential.hpp:44-58); a = 2 is the harmonic
    repulsion.  The device always uses a cell list; ``use_cell_lists`` and
    ``ncellx_scale`` are kept for signature compatibility (results do not
    depend on the cell size).
    """

    def __init__(self, a, eps, radii, boxv, use_cell_lists=False, ncellx_scale=None, balance_omp=True,
                 method=Distance.PERIODIC):
        self.boxv = _f64(boxv)
        self.radii = _f64(radii)
        self.use_cell_lists = use_cell_lists
        self.ncellx_scale = 1.0 if ncellx_scale is None else float(ncellx_scale)
        self.balance_omp = balance_omp
        self.method = method
        self.ndim = self.boxv.size
        self.natoms = self.radii.size
        self.a = float(a)
        self.eps = float(eps)
        if isinstance(method, Distance):
            periodic = method == Distance.PERIODIC
        else:
            periodic = str(getattr(method, "name", method)).upper().endswith("PERIODIC")
        if self.ndim not in (1, 2, 3):
            raise NotImplementedError
        h = _lib.handle_t()
        check(lib.fresco_inversepower_create(self.a, self.eps, dptr(self.radii), self.natoms, dptr(self.boxv),
                                             self.ndim, int(periodic), int(bool(use_cell_lists)),
                                             self.ncellx_scale, C.byref(h)))
        self._set_handle(h)

    def __reduce__(self):
        return (self.__class__, (self.a, self.eps, self.radii, self.boxv, self.use_cell_lists, self.ncellx_scale,
                                 self.balance_omp, self.method), {})

    def __setstate__(self, d):
        pass


class CombinedPotential(BasePotential):
    """Sum of potentials (fresco/potentials/combine_potentials.pyx:10-30)."""

    def __init__(self):
        self._parts = []
        h = _lib.handle_t()
        check(lib.fresco_combined_create(C.byref(h)))
        self._set_handle(h)

    def add_potential(self, potential):
        if not isinstance(potential, BasePotential):
            raise TypeError("add_potential expects a fresco_b200 potential")
        check(lib.fresco_combined_add(self._h, potential.handle))
        self._parts.append(potential)
