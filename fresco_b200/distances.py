"""Hard-core overlap check on the device: the counterpart of fresco.distances.CheckOverlap
(fresco/distances/_check_overlap.pyx:11-110; source/fresco/check_overlap.hpp:24-130,
check_overlap_cell_lists.hpp:87-180)."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import check, dptr, lib
from .potentials import Distance

__all__ = ["CheckOverlap", "Distance"]


class CheckOverlap:
    """CheckOverlap(radii, boxv, use_cell_lists=False, ncellx_scale=None, method=Distance.PERIODIC).

    ``get_overlapping_particles(coords)`` returns the indices (uint64) of the particles whose cores overlap
    another one, |r_ij|^2 < (r_i + r_j)^2, in ascending order (the reference returns them in the order of an
    unordered_set).  ``get_overlapping_particles_ca(coords, changed_atoms_idx)`` only counts pairs that hold a
    changed atom, except with ``use_cell_lists``, where the reference checks every pair.  Cell lists are always used on the device; ``use_cell_lists`` and ``ncellx_scale`` are kept
    for the constructor's signature and pickling (the result does not depend on them), and no cell-scale line
    is printed."""

    def __init__(self, radii, boxv, use_cell_lists=False, ncellx_scale=None, method=Distance.PERIODIC):
        self.boxv = np.ascontiguousarray(np.asarray(boxv, dtype=np.float64).ravel())
        self.radii = np.ascontiguousarray(np.asarray(radii, dtype=np.float64).ravel())
        self.use_cell_lists = use_cell_lists
        self.ncellx_scale = ncellx_scale
        self.method = method
        self.ndim = self.boxv.size
        self.natoms = self.radii.size
        if isinstance(method, Distance):
            periodic = method == Distance.PERIODIC
        else:
            periodic = str(getattr(method, "name", method)).upper().endswith("PERIODIC")
        if self.ndim not in (1, 2, 3):
            raise NotImplementedError
        if use_cell_lists and self.ndim == 1:  # the reference's cell lists refuse one dimension
            raise RuntimeError("CellLists::CellLists: Cell lists only work with more than 1 dimension "
                               "(due to the split of subdomains in y-dimension)")  # cell_lists.hpp:837-839
        h = _lib.handle_t()
        check(lib.fresco_overlap_create(dptr(self.radii), self.radii.size, dptr(self.boxv), self.ndim,
                                        int(periodic), C.byref(h)))
        self._h = h

    def __del__(self):
        h, self._h = getattr(self, "_h", None), None
        if h:
            try:
                lib.fresco_overlap_destroy(h)
            except Exception:
                pass

    def _find(self, coords, changed):
        x = np.ascontiguousarray(np.asarray(coords, dtype=np.float64).ravel())
        out = np.empty(max(self.natoms, 1), dtype=np.uint64)
        count = C.c_int64()
        if changed is None:
            cp, nc = None, 0
        else:
            ch = np.ascontiguousarray(np.asarray(changed, dtype=np.int64).ravel())
            cp, nc = ch.ctypes.data_as(C.POINTER(C.c_int64)), ch.size
            self._changed = ch  # keeps the buffer alive through the call
        check(lib.fresco_overlap_find(self._h, dptr(x), x.size, cp, nc,
                                      out.ctypes.data_as(C.POINTER(C.c_uint64)), C.byref(count)))
        return out[:count.value].copy()

    def get_overlapping_particles(self, coords):
        return self._find(coords, None)

    def get_overlapping_particles_ca(self, coords, changed_atoms_idx):
        if self.use_cell_lists:
            # The reference's cell-list check passes no old coordinates here (check_overlap_cell_lists.hpp:
            # 145-149), so its changed-atoms branch (:128) is never taken: the whole configuration is checked.
            return self._find(coords, None)
        return self._find(coords, changed_atoms_idx)

    def __reduce__(self):
        return (self.__class__, (self.radii, self.boxv, self.use_cell_lists, self.ncellx_scale, self.method), {})

    def __setstate__(self, d):
        pass
