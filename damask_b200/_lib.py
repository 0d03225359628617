"""ctypes binding of ``libdamask_b200.so`` (the C-ABI declared in ``include/damask_b200.h``).

The product path has no fallback: if the library cannot be loaded, every entry
point raises.  The library is built in-tree by :mod:`damask_b200.build`.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

from .config import (BATCH_INCREMENT_CB, INCREMENT_CB, BCStruct, GridSolverStruct, LoadStepStruct, NumericsStruct, PhaseStruct,
                     RestartStruct, SolutionStruct)

LIB_PATH = Path(__file__).resolve().parent / 'libdamask_b200.so'

EXPORTS = ['dmk_mech_init', 'dmk_mech_forward', 'dmk_mech_solution', 'dmk_materialpoint_forward',
           'dmk_mech_update_coords', 'dmk_get_field', 'dmk_set_field', 'dmk_field_size', 'dmk_get_aims',
           'dmk_constitutive_response', 'dmk_update_gamma', 'dmk_gamma_convolution', 'dmk_divergence_rms',
           'dmk_dPdF', 'dmk_get_iteration_counts', 'dmk_get_counters', 'dmk_get_timings', 'dmk_destroy',
           'dmk_last_error', 'dmk_get_launches', 'dmk_timer_start', 'dmk_timer_stop', 'dmk_phase_schmid',
           'dmk_phase_interaction', 'dmk_field_mean_noalloc', 'dmk_restart_write', 'dmk_restart_read',
           'dmk_get_coords', 'dmk_curl_rms', 'dmk_phase_slip_systems', 'dmk_vti_open', 'dmk_vti_geometry',
           'dmk_vti_label', 'dmk_vti_read_int', 'dmk_vti_read_real', 'dmk_vti_close', 'dmk_grid_run',
           'dmk_grid_run_ctx', 'dmk_fp64_peak', 'dmk_checkpoint_save', 'dmk_checkpoint_restore', 'dmk_adj_begin',
           'dmk_adj_record', 'dmk_adj_step', 'dmk_adj_finish', 'dmk_adj_local_jacobian', 'dmk_batch_create',
           'dmk_batch_solution', 'dmk_batch_stats', 'dmk_batch_destroy', 'dmk_batch_run', 'dmk_autotune',
           'dmk_get_tuning', 'dmk_set_tuning']

_lib = None

dp = C.POINTER(C.c_double)
ip = C.POINTER(C.c_int)


class DamaskError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f'{msg} (code {code})')
        self.code = code


def load(path: str | os.PathLike | None = None) -> C.CDLL:
    """Load the CUDA library (once)."""
    global _lib
    if _lib is not None:
        return _lib
    p = Path(path) if path else LIB_PATH
    if not p.exists():
        raise RuntimeError(f'{p} is missing: build it with "python -m damask_b200.build" (no CPU fallback exists)')
    lib = C.CDLL(str(p))
    vp = C.c_void_p
    sig = {
        'dmk_mech_init': (C.c_int, [C.POINTER(vp), ip, dp, ip, C.c_int, dp, C.POINTER(PhaseStruct),
                                    C.POINTER(NumericsStruct), C.c_int, C.c_int]),
        'dmk_mech_forward': (C.c_int, [vp, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double,
                                       C.POINTER(BCStruct), C.POINTER(BCStruct), dp]),
        'dmk_mech_solution': (C.c_int, [vp, C.POINTER(SolutionStruct)]),
        'dmk_materialpoint_forward': (C.c_int, [vp]),
        'dmk_mech_update_coords': (C.c_int, [vp]),
        'dmk_get_coords': (C.c_int, [vp, dp, dp]),
        'dmk_curl_rms': (C.c_int, [vp, dp, dp]),
        'dmk_phase_slip_systems': (C.c_int, [C.POINTER(PhaseStruct), C.POINTER(C.c_int)]),
        'dmk_vti_open': (C.c_int, [C.c_char_p, C.POINTER(vp)]),
        'dmk_vti_geometry': (C.c_int, [vp, ip, dp, dp]),
        'dmk_vti_label': (C.c_int, [vp, C.c_int, C.c_char_p, C.c_int, ip]),
        'dmk_vti_read_int': (C.c_int, [vp, C.c_char_p, C.POINTER(C.c_int64), C.c_int64]),
        'dmk_vti_read_real': (C.c_int, [vp, C.c_char_p, dp, C.c_int64]),
        'dmk_vti_close': (None, [vp]),
        'dmk_grid_run': (C.c_int, [C.POINTER(GridSolverStruct), C.POINTER(LoadStepStruct), C.c_int, C.c_int, C.c_int,
                                   C.c_int, INCREMENT_CB, C.c_void_p]),
        'dmk_grid_run_ctx': (C.c_int, [vp, C.POINTER(LoadStepStruct), C.c_int, C.c_int, C.c_int, C.c_int,
                                       INCREMENT_CB, C.c_void_p]),
        'dmk_fp64_peak': (C.c_int, [C.c_int, dp]),
        'dmk_get_field': (C.c_int, [vp, C.c_int, dp]),
        'dmk_set_field': (C.c_int, [vp, C.c_int, dp]),
        'dmk_field_size': (C.c_int, [vp, C.c_int]),
        'dmk_get_aims': (C.c_int, [vp, dp, dp, dp, dp, dp, dp, dp]),
        'dmk_restart_write': (C.c_int, [vp, C.POINTER(RestartStruct)]),
        'dmk_restart_read': (C.c_int, [vp, C.POINTER(RestartStruct)]),
        'dmk_constitutive_response': (C.c_int, [vp, dp, C.c_double, dp, dp, dp, dp, ip]),
        'dmk_update_gamma': (C.c_int, [vp, dp]),
        'dmk_gamma_convolution': (C.c_int, [vp, dp, dp]),
        'dmk_divergence_rms': (C.c_int, [vp, dp, dp]),
        'dmk_dPdF': (C.c_int, [vp, C.c_double, dp]),
        'dmk_get_iteration_counts': (C.c_int, [vp, ip]),
        'dmk_get_counters': (C.c_int, [vp, C.POINTER(C.c_int64)]),
        'dmk_get_timings': (C.c_int, [vp, dp]),
        'dmk_get_launches': (C.c_int, [vp, C.POINTER(C.c_int64)]),
        'dmk_timer_start': (C.c_int, [vp]),
        'dmk_timer_stop': (C.c_int, [vp, dp]),
        'dmk_phase_schmid': (C.c_int, [C.POINTER(PhaseStruct), C.c_int, dp]),
        'dmk_phase_interaction': (C.c_int, [C.POINTER(PhaseStruct), dp]),
        'dmk_field_mean_noalloc': (C.c_int, [C.c_void_p, C.c_int64, dp, C.c_void_p]),
        'dmk_checkpoint_save': (C.c_int, [vp, C.c_int]),
        'dmk_checkpoint_restore': (C.c_int, [vp, C.c_int]),
        'dmk_adj_begin': (C.c_int, [vp, C.c_int]),
        'dmk_adj_record': (C.c_int, [vp, C.c_int]),
        'dmk_adj_step': (C.c_int, [vp, C.c_int, dp, dp, ip]),
        'dmk_adj_finish': (C.c_int, [vp, dp]),
        'dmk_adj_local_jacobian': (C.c_int, [C.POINTER(PhaseStruct), C.c_double, dp, dp]),
        'dmk_batch_create': (C.c_int, [C.POINTER(vp), C.POINTER(vp), C.c_int]),
        'dmk_batch_solution': (C.c_int, [vp, ip, C.c_int, C.POINTER(SolutionStruct)]),
        'dmk_batch_stats': (C.c_int, [vp, dp]),
        'dmk_batch_destroy': (None, [vp]),
        'dmk_batch_run': (C.c_int, [vp, C.POINTER(C.POINTER(LoadStepStruct)), ip, C.c_int, C.c_int, BATCH_INCREMENT_CB,
                                    C.c_void_p, ip]),
        'dmk_autotune': (C.c_int, [vp, C.c_int, dp, ip]),
        'dmk_get_tuning': (C.c_int, [vp, ip, ip]),
        'dmk_set_tuning': (C.c_int, [vp, C.c_int, C.c_int]),
        'dmk_destroy': (None, [vp]),
        'dmk_last_error': (C.c_char_p, []),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib


def check(rc: int) -> None:
    if rc != 0:
        msg = _lib.dmk_last_error().decode() if _lib is not None else 'library not loaded'
        raise DamaskError(rc, msg or 'constitutive failure')
