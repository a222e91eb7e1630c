"""ctypes binding of the fresco_b200 C ABI (include/fresco_b200.h).

The shared library is built in-tree (``fresco_b200/libfresco_b200.so``, see
``fresco_b200.build``).  There is no CPU fallback: if the library is missing
or cannot be loaded, importing the package raises ``ImportError``.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

_LIB_PATH = Path(__file__).resolve().parent / "libfresco_b200.so"

FRESCO_OK = 0
FRESCO_ERR_INVALID = 1
FRESCO_ERR_RUNTIME = 2
FRESCO_ERR_NONFINITE = 3

c_double_p = C.POINTER(C.c_double)
c_int_p = C.POINTER(C.c_int)
c_int64 = C.c_int64
c_void_p = C.c_void_p
handle_t = C.c_void_p

# name -> (restype, [argtypes])
_SIGNATURES = {
    "fresco_last_error": (C.c_char_p, []),
    "fresco_abi_version": (C.c_int, []),
    "fresco_nuwu_create": (C.c_int, [c_double_p, c_int64, C.c_double, c_double_p, c_double_p, c_int64, c_double_p,
                                     C.c_int, C.c_double, C.c_int, C.POINTER(handle_t)]),
    "fresco_nuwu_shard_create": (C.c_int, [c_double_p, c_int64, c_int64, C.c_double, C.c_double, c_double_p,
                                           c_double_p, c_int64, c_double_p, C.c_int, C.c_double, C.c_int,
                                           C.POINTER(handle_t)]),
    "fresco_nuwu_weight_sum": (C.c_int, [c_double_p, c_int64, C.c_int, c_double_p]),
    "fresco_nuwu_shard_nrho": (C.c_int, [handle_t, C.POINTER(c_int64)]),
    "fresco_nuwu_shard_rho": (C.c_int, [handle_t, c_void_p, c_int64, c_void_p, c_void_p]),
    "fresco_nuwu_shard_finish": (C.c_int, [handle_t, c_void_p, c_void_p, c_void_p, c_void_p]),
    "fresco_uwu_create": (C.c_int, [c_int_p, C.c_int, C.c_double, c_double_p, c_double_p, c_int64, c_double_p,
                                    C.c_double, C.c_int, C.POINTER(handle_t)]),
    "fresco_uwnu_create": (C.c_int, [c_int_p, C.c_int, c_double_p, c_int64, c_double_p, c_double_p, c_double_p,
                                     C.c_double, C.c_int, C.POINTER(handle_t)]),
    "fresco_nuwnu_create": (C.c_int, [c_double_p, c_int64, c_double_p, c_int64, c_double_p, c_double_p, c_double_p,
                                      C.c_int, C.c_double, C.c_int, C.POINTER(handle_t)]),
    "fresco_inversepower_create": (C.c_int, [C.c_double, C.c_double, c_double_p, c_int64, c_double_p, C.c_int,
                                             C.c_int, C.c_int, C.c_double, C.POINTER(handle_t)]),
    "fresco_combined_create": (C.c_int, [C.POINTER(handle_t)]),
    "fresco_combined_add": (C.c_int, [handle_t, handle_t]),
    "fresco_potential_destroy": (None, [handle_t]),
    "fresco_potential_ndof": (c_int64, [handle_t]),
    "fresco_potential_energy": (C.c_int, [handle_t, c_double_p, c_int64, c_double_p]),
    "fresco_potential_energy_gradient": (C.c_int, [handle_t, c_double_p, c_int64, c_double_p, c_double_p]),
    "fresco_potential_energy_device": (C.c_int, [handle_t, c_void_p, c_int64, c_void_p, C.c_int, c_void_p]),
    "fresco_potential_energy_gradient_device": (C.c_int, [handle_t, c_void_p, c_int64, c_void_p, c_void_p, C.c_int,
                                                          c_void_p]),
    "fresco_nuwnu_energy_gradient_noalloc": (C.c_int, [c_void_p, c_int64, C.c_int, c_void_p, c_void_p, c_void_p,
                                                       c_void_p, c_int64, c_double_p, C.c_int, c_void_p, c_void_p,
                                                       C.c_int, c_void_p]),
    "fresco_export_structure": (C.c_int, [c_double_p, c_int64, C.c_int, c_double_p, C.c_int, c_double_p, C.c_double,
                                          c_double_p, c_double_p, c_double_p, c_double_p]),
    "fresco_potential_status": (C.c_int, [handle_t, c_void_p, c_int_p]),
    "fresco_debug_set_tile_wait_polls": (C.c_int, [C.c_int]),
    "fresco_potential_set_reducer": (C.c_int, [handle_t, c_void_p, c_void_p]),
    "fresco_optimizer_state_bytes": (C.c_int, [handle_t, C.POINTER(C.c_int64)]),
    "fresco_optimizer_save_state": (C.c_int, [handle_t, c_void_p]),
    "fresco_optimizer_load_state": (C.c_int, [handle_t, c_void_p, c_int64]),
    "fresco_inversepower_shard_create": (C.c_int, [C.c_double, C.c_double, c_double_p, c_int64, c_double_p, C.c_int,
                                                   C.c_int, c_int64, c_int64, c_void_p, c_void_p, c_void_p,
                                                   C.POINTER(handle_t)]),
    "fresco_inversepower_halo_create": (C.c_int, [C.c_double, C.c_double, c_double_p, c_int64, c_double_p, C.c_int,
                                                  c_int64, c_int64, C.c_int, C.c_int, c_void_p, c_void_p, c_void_p,
                                                  C.POINTER(handle_t)]),
    "fresco_inversepower_halo_stats": (C.c_int, [handle_t, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]),
    "fresco_optimizer_set_reducer": (C.c_int, [handle_t, c_void_p, c_void_p, c_int64]),
    "fresco_potential_set_gradient_mode": (C.c_int, [handle_t, C.c_int]),
    "fresco_potential_gradient_mode": (C.c_int, [handle_t, c_int_p]),
    "fresco_potential_set_timing": (C.c_int, [handle_t, C.c_int]),
    "fresco_potential_get_timing": (C.c_int, [handle_t, C.c_int, C.c_char_p, C.c_int, c_double_p, c_int_p, c_int_p]),
    "fresco_potential_describe": (C.c_int, [handle_t, C.c_char_p, C.c_int]),
    "fresco_lbfgs_create": (C.c_int, [handle_t, c_double_p, c_int64, C.c_double, C.c_int, C.c_double, C.c_double,
                                      C.c_double, C.c_int, C.c_int, C.c_int, C.c_int, C.POINTER(handle_t)]),
    "fresco_fire_create": (C.c_int, [handle_t, c_double_p, c_int64, C.c_double, C.c_double, C.c_double, C.c_int,
                                     C.c_double, C.c_double, C.c_double, C.c_double, C.c_double, C.c_int, C.c_int,
                                     C.c_int, C.c_int, C.POINTER(handle_t)]),
    "fresco_overlap_create": (C.c_int, [c_double_p, c_int64, c_double_p, C.c_int, C.c_int, C.POINTER(handle_t)]),
    "fresco_overlap_find": (C.c_int, [handle_t, c_double_p, c_int64, C.POINTER(C.c_int64), c_int64,
                                      C.POINTER(C.c_uint64), C.POINTER(C.c_int64)]),
    "fresco_overlap_destroy": (None, [handle_t]),
    "fresco_window_stats_create": (C.c_int, [c_double_p, c_int64, C.c_int, c_double_p, c_double_p, C.c_int,
                                             C.c_uint64, C.POINTER(handle_t)]),
    "fresco_window_stats_run": (C.c_int, [handle_t, c_int64]),
    "fresco_window_stats_set_seed": (C.c_int, [handle_t, C.c_uint64]),
    "fresco_window_stats_get": (C.c_int, [handle_t, C.POINTER(C.c_uint64), c_double_p, c_double_p,
                                          C.POINTER(C.c_uint64)]),
    "fresco_window_stats_destroy": (None, [handle_t]),
    "fresco_fire_graph_create": (C.c_int, [handle_t, c_double_p, c_int64, C.c_double, C.c_double, C.c_double,
                                           C.c_int, C.c_double, C.c_double, C.c_double, C.c_double, C.c_double,
                                           C.c_int, C.c_int, C.POINTER(handle_t)]),
    "fresco_optimizer_set_func_gradient": (C.c_int, [handle_t, C.c_double, c_double_p, c_int64]),
    "fresco_lbfgs_set_H0": (C.c_int, [handle_t, C.c_double]),
    "fresco_optimizer_run": (C.c_int, [handle_t, C.c_int]),
    "fresco_optimizer_one_iteration": (C.c_int, [handle_t]),
    "fresco_optimizer_reset": (C.c_int, [handle_t, c_double_p, c_int64]),
    "fresco_optimizer_stop_criterion_satisfied": (C.c_int, [handle_t, c_int_p]),
    "fresco_optimizer_get_state": (C.c_int, [handle_t, c_double_p, c_double_p, c_double_p, c_double_p, c_int_p,
                                             c_int_p, c_int_p, c_double_p]),
    "fresco_optimizer_device_state": (C.c_int, [handle_t, C.POINTER(c_void_p), C.POINTER(c_void_p)]),
    "fresco_optimizer_destroy": (None, [handle_t]),
    "fresco_nuwu_ensemble_create": (C.c_int, [C.c_int, C.POINTER(c_int64), c_double_p, C.POINTER(c_int64), c_double_p,
                                              c_double_p, c_double_p, C.c_int, C.c_double, C.c_int,
                                              C.POINTER(handle_t)]),
    "fresco_ensemble_info": (C.c_int, [handle_t, c_int_p, C.POINTER(c_int64), C.POINTER(c_int64)]),
    "fresco_ensemble_energy_gradient": (C.c_int, [handle_t, c_double_p, c_int64, c_double_p, c_double_p]),
    "fresco_ensemble_energy_gradient_device": (C.c_int, [handle_t, c_void_p, c_int64, c_void_p, c_void_p, c_void_p]),
    "fresco_ensemble_tune": (C.c_int, [handle_t, c_double_p, c_int64]),
    "fresco_ensemble_set_subproblem_cap": (C.c_int, [handle_t, C.c_int]),
    "fresco_ensemble_set_split": (C.c_int, [handle_t, C.c_double]),
    "fresco_ensemble_status": (C.c_int, [handle_t, c_int_p]),
    "fresco_ensemble_describe": (C.c_int, [handle_t, C.c_char_p, C.c_int]),
    "fresco_ensemble_destroy": (None, [handle_t]),
    "fresco_ensemble_lbfgs_create": (C.c_int, [handle_t, c_double_p, c_int64, C.c_double, C.c_int, C.c_double,
                                               C.c_double, C.c_double, C.c_int, C.POINTER(handle_t)]),
    "fresco_lbfgs_graph_create": (C.c_int, [handle_t, c_double_p, c_int64, C.c_double, C.c_int, C.c_double,
                                            C.c_double, C.c_double, C.c_int, C.POINTER(handle_t)]),
    "fresco_ensemble_lbfgs_run": (C.c_int, [handle_t, C.c_int, c_int_p]),
    "fresco_ensemble_lbfgs_steps": (C.c_int, [handle_t, C.c_int]),
    "fresco_ensemble_lbfgs_state": (C.c_int, [handle_t, c_double_p, c_double_p, c_double_p, c_double_p, c_int_p,
                                              c_int_p, c_int_p]),
    "fresco_ensemble_lbfgs_destroy": (None, [handle_t]),
}


def exported_symbols():
    """Names of every entry point the binding expects (all of include/fresco_b200.h)."""
    return sorted(_SIGNATURES)


def _load():
    if not _LIB_PATH.exists():
        raise ImportError(
            f"fresco_b200 CUDA library not built: {_LIB_PATH} is missing "
            "(run `python fresco_b200/build.py`); there is no CPU fallback"
        )
    lib = C.CDLL(str(_LIB_PATH), mode=os.RTLD_NOW | getattr(os, "RTLD_GLOBAL", 0))
    for name, (res, args) in _SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


lib = _load()
LIB_PATH = str(_LIB_PATH)


def check(rc: int) -> None:
    """Raises the Python exception matching a C status code."""
    if rc == FRESCO_OK:
        return
    msg = (lib.fresco_last_error() or b"").decode(errors="replace")
    if rc == FRESCO_ERR_INVALID:
        raise ValueError(msg)
    raise RuntimeError(msg or f"fresco_b200 error {rc}")


def dptr(a):
    """ctypes double* of a C-contiguous float64 numpy array."""
    return a.ctypes.data_as(c_double_p)
