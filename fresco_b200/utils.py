"""Structure measurement after a minimisation, computed on the device: the counterparts of
fresco.utils.export_structure (fresco/utils/utils.py:16-52), radial_profile (utils.py:138-152), and the
number-variance statistics PointPatternStatistics / BatchPPS (fresco/utils/c_utils.pyx:8-150)."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import check, dptr, lib


def export_structure(r, L, Nk=1001, radii=None, tol=1e-9):
    """S(k) and g(r) of a point pattern, as fresco.utils.export_structure.

    Returns ``(q, S, Sk, r / Nk, g, gr)``: integer radii q = 0..Nk//2 with the radial averages S of
    S(k) = |rho(k)|^2 / N, the Nk^d array Sk in centred order, the pair-correlation radii and their
    averages g, and the Nk^d array gr.  rho is the type-1 NUFFT of the points (weights 1, or the point
    volumes scaled to sum to N when radii are given) on Nk modes per dimension at tolerance tol.
    """
    L = np.ascontiguousarray(np.asarray(L, dtype=np.float64).ravel())
    ndim = L.size
    if ndim not in (2, 3):
        raise ValueError("Invalid dimension")
    x = np.ascontiguousarray(np.asarray(r, dtype=np.float64).reshape(-1, ndim))
    n = x.shape[0]
    rad = None if radii is None else np.ascontiguousarray(np.asarray(radii, dtype=np.float64).ravel())
    if rad is not None and rad.size != n:
        raise ValueError("radii must have one value per point")
    Nk = int(Nk)
    shape = (Nk,) * ndim
    sk = np.empty(shape)
    gr = np.empty(shape)
    R = Nk // 2
    s_rad = np.empty(R + 1)
    g_rad = np.empty(R + 1)
    check(lib.fresco_export_structure(dptr(x), n, ndim, dptr(L), Nk,
                                      dptr(rad) if rad is not None else C.cast(None, C.POINTER(C.c_double)),
                                      float(tol), dptr(sk), dptr(gr), dptr(s_rad), dptr(g_rad)))
    q = np.arange(R + 1)
    # the reference drops the last bin as the one beyond R; when no cell lies beyond R
    # (Nk < 6) that bin is a real one and is dropped all the same
    corner = int(np.sqrt(ndim * float(max(Nk // 2, Nk - 1 - Nk // 2)) ** 2))
    if corner <= R:
        q, s_rad, g_rad = q[:-1], s_rad[:-1], g_rad[:-1]
    return q, s_rad, sk, q / Nk, g_rad, gr


def radial_profile(data, center=None):
    """Average of an array over integer radii from its centre (utils.py:138-152); host numpy."""
    data = np.asarray(data)
    ndim = data.ndim
    R = int(data.shape[0] / 2)
    if center is None:
        center = np.array(data.shape) / 2
    center = np.asarray(center)
    for _ in range(ndim):
        center = np.expand_dims(center, axis=-1)
    idx = np.indices(data.shape)
    rr = np.sqrt(np.sum((idx - center) ** 2, axis=0)).astype(int)
    rr = np.where(rr <= R, rr, R + 1)
    tbin = np.bincount(rr.ravel(), data.ravel())
    nr = np.bincount(rr.ravel())
    return np.unique(rr).ravel()[:-1], (tbin / nr)[:-1]


class _WindowStats:
    """Number-variance window counts on the device (point_pattern_statistics.hpp:36-111,
    batch_pointstats.hpp:29-150, fresco/utils/c_utils.pyx:8-150): windows centred at the
    std::mt19937_64(rseed) stream's points, the same stream as the reference's; for each radius the
    running mean and variance (E[n^2] - E[n]^2, moments.hpp:28-52) of the number of points within it."""

    _h = None

    def _create(self, coords, boxv, radii, rseed):
        self.coords = np.ascontiguousarray(np.asarray(coords, dtype=np.float64).ravel())
        self.boxv = np.ascontiguousarray(np.asarray(boxv, dtype=np.float64).ravel())
        self.ndim = self.boxv.size
        self.natoms = len(self.coords) // max(self.ndim, 1)
        self.rseed = int(rseed)
        r = np.ascontiguousarray(np.asarray(radii, dtype=np.float64).ravel())
        self._nr = r.size
        if self.ndim not in (1, 2, 3):
            raise NotImplementedError
        h = _lib.handle_t()
        check(lib.fresco_window_stats_create(dptr(self.coords), self.natoms, self.ndim, dptr(self.boxv), dptr(r),
                                             r.size, C.c_uint64(self.rseed), C.byref(h)))
        self._h = h

    def __del__(self):
        h, self._h = self._h, None
        if h:
            try:
                lib.fresco_window_stats_destroy(h)
            except Exception:
                pass

    def _get(self):
        seed = C.c_uint64()
        mean = np.empty(self._nr)
        var = np.empty(self._nr)
        count = np.empty(self._nr, dtype=np.uint64)
        check(lib.fresco_window_stats_get(self._h, C.byref(seed), dptr(mean), dptr(var),
                                          count.ctypes.data_as(C.POINTER(C.c_uint64))))
        return seed.value, mean, var, count

    def get_seed(self):
        return self._get()[0]

    def set_generator_seed(self, seed):
        check(lib.fresco_window_stats_set_seed(self._h, C.c_uint64(int(seed))))

    def run(self, n):
        check(lib.fresco_window_stats_run(self._h, int(n)))

    @property
    def mean(self):
        return self.get_mean()

    @property
    def var(self):
        return self.get_variance()

    @property
    def mean_var(self):
        return self.get_mean(), self.get_variance()

    @property
    def count(self):
        return self.get_count()

    def __setstate__(self, d):
        pass


class PointPatternStatistics(_WindowStats):
    """PointPatternStatistics(coords, boxv, radius, rseed) (fresco/utils/c_utils.pyx:46-79): one window
    radius; get_mean / get_variance return floats, get_count an int."""

    def __init__(self, coords, boxv, radius, rseed):
        self.radius = float(radius)
        self._create(coords, boxv, [self.radius], rseed)

    def get_mean(self):
        return float(self._get()[1][0])

    def get_variance(self):
        return float(self._get()[2][0])

    def get_count(self):
        return int(self._get()[3][0])

    def __reduce__(self):
        return (self.__class__, (self.coords, self.boxv, self.radius, self.rseed), {})


class BatchPPS(_WindowStats):
    """BatchPPS(coords, boxv, radii, rseed) (fresco/utils/c_utils.pyx:118-150): several window radii,
    ascending, over the same windows; get_mean / get_variance / get_count return one value per radius."""

    def __init__(self, coords, boxv, radii, rseed):
        self.radii = np.ascontiguousarray(np.asarray(radii, dtype=np.float64).ravel())
        self._create(coords, boxv, self.radii, rseed)

    def get_mean(self):
        return self._get()[1]

    def get_variance(self):
        return self._get()[2]

    def get_count(self):
        return self._get()[3]

    def __reduce__(self):
        return (self.__class__, (self.coords, self.boxv, self.radii, self.rseed), {})
