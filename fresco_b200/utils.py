"""Structure measurement after a minimisation: the counterpart of fresco.utils.export_structure
(fresco/utils/utils.py:16-52) and radial_profile (utils.py:138-152), computed on the device."""
from __future__ import annotations

import ctypes as C

import numpy as np

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
