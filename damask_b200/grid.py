"""Host side of the grid mechanical solver: the plugin object and the increment loop.

``SpectralBasic`` mirrors the five procedures DAMASK's grid driver selects for the
``spectral_basic`` solver (``src/grid/DAMASK_grid.f90:110-119,171-206``):
``init`` (constructor), ``forward``, ``solution``, ``update_coords`` and the
materialpoint forward that follows a converged increment.  All compute runs in
``libdamask_b200.so`` on the GPU; this module only marshals host arrays.

``run_load_cases`` restates the driver's increment loop with its global cutback
(``DAMASK_grid.f90:288-460``) for any object with that interface, so the same
host logic drives the CUDA path and, in tests, the CPU oracle.
"""
from __future__ import annotations

import ctypes as C
import time
from dataclasses import dataclass, field

import numpy as np

from . import _lib
from .config import LoadCase, Numerics, Phase, SolutionStruct, geometric_fraction

FIELDS = {'F': 0, 'P': 1, 'F_e': 2, 'F_p': 3, 'L_p': 4, 'S': 5, 'xi_sl': 6, 'gamma_sl': 7,
          'F_lastinc': 8, 'F_i': 9, 'L_i': 10, 'F_solver': 11}

PRECISIONS = {'fp64': 0, 'mixed': 1}


def _dp(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


class SpectralBasic:
    """grid_mechanical_spectral_basic on one GPU (B200, sm_100a)."""

    def __init__(self, cells, size, material: np.ndarray, quaternions: np.ndarray, phase: Phase,
                 numerics: Numerics | None = None, precision: str = 'fp64', device: int = 0):
        self.lib = _lib.load()
        self.cells = tuple(int(c) for c in cells)
        self.size = tuple(float(s) for s in size)
        self.N = int(np.prod(self.cells))
        self.phase = phase
        self.numerics = numerics or Numerics()
        self.precision = precision
        self._ps = phase.to_struct()
        self._ns = self.numerics.to_struct()
        mat = np.ascontiguousarray(material, dtype=np.int32).reshape(-1)
        if mat.size != self.N:
            raise ValueError('material map does not match the grid')
        q = np.ascontiguousarray(quaternions, dtype=np.float64).reshape(-1, 4)
        ctx = C.c_void_p()
        cells_a = (C.c_int * 3)(*self.cells)
        size_a = (C.c_double * 3)(*self.size)
        t0 = time.perf_counter()
        _lib.check(self.lib.dmk_mech_init(C.byref(ctx), cells_a, size_a, mat.ctypes.data_as(C.POINTER(C.c_int)),
                                          q.shape[0], _dp(q), C.byref(self._ps), C.byref(self._ns),
                                          PRECISIONS[precision], device))
        self.init_seconds = time.perf_counter() - t0
        self.ctx = ctx
        self.n_slip = phase.n_slip

    # -- the plugin procedures ------------------------------------------------------------------
    def forward(self, cutBack: bool, guess: bool, Delta_t: float, Delta_t_old: float, t_remaining: float,
                lc: LoadCase) -> None:
        q = (C.c_double * 4)(*lc.q_rot)
        d, s = lc.deformation_bc(), lc.stress_bc()
        _lib.check(self.lib.dmk_mech_forward(self.ctx, int(cutBack), int(guess), Delta_t, Delta_t_old, t_remaining,
                                             C.byref(d), C.byref(s), q))

    def solution(self) -> SolutionStruct:
        out = SolutionStruct()
        _lib.check(self.lib.dmk_mech_solution(self.ctx, C.byref(out)))
        return out

    def materialpoint_forward(self) -> None:
        _lib.check(self.lib.dmk_materialpoint_forward(self.ctx))

    def update_coords(self) -> None:
        _lib.check(self.lib.dmk_mech_update_coords(self.ctx))

    # -- fields and diagnostics -----------------------------------------------------------------
    def get_field(self, name: str, out: np.ndarray | None = None) -> np.ndarray:
        fid = FIELDS[name]
        k = self.lib.dmk_field_size(self.ctx, fid)
        if out is None:
            out = np.empty((self.N, k), dtype=np.float64)
        _lib.check(self.lib.dmk_get_field(self.ctx, fid, _dp(out)))
        return out

    def set_field(self, name: str, values: np.ndarray) -> None:
        v = np.ascontiguousarray(values, dtype=np.float64)
        _lib.check(self.lib.dmk_set_field(self.ctx, FIELDS[name], _dp(v)))

    def aims(self) -> dict:
        bufs = {k: np.zeros(n) for k, n in (('F_aim', 9), ('F_aim_lastinc', 9), ('F_aimDot', 9), ('P_aim', 9),
                                            ('C_volAvg', 81), ('C_volAvgLastInc', 81), ('C_minMaxAvg', 81))}
        _lib.check(self.lib.dmk_get_aims(self.ctx, *(_dp(b) for b in bufs.values())))
        return bufs

    def counters(self) -> np.ndarray:
        out = (C.c_int64 * 4)()
        _lib.check(self.lib.dmk_get_counters(self.ctx, out))
        return np.array(out[:])

    def timings(self) -> np.ndarray:
        out = np.zeros(3)
        _lib.check(self.lib.dmk_get_timings(self.ctx, _dp(out)))
        return out

    # -- operator-level entry points --------------------------------------------------------------
    def constitutive_response(self, F: np.ndarray, dt: float):
        F = np.ascontiguousarray(F, dtype=np.float64).reshape(self.N, 9)
        P = np.empty((self.N, 9))
        P_av, Cv, Cm = np.zeros(9), np.zeros(81), np.zeros(81)
        st = C.c_int()
        _lib.check(self.lib.dmk_constitutive_response(self.ctx, _dp(F), dt, _dp(P), _dp(P_av), _dp(Cv), _dp(Cm),
                                                      C.byref(st)))
        return P, P_av, Cv, Cm, st.value

    def iteration_counts(self) -> np.ndarray:
        out = np.zeros((self.N, 4), dtype=np.int32)
        _lib.check(self.lib.dmk_get_iteration_counts(self.ctx, out.ctypes.data_as(C.POINTER(C.c_int))))
        return out

    def update_gamma(self, Cmat: np.ndarray) -> None:
        c = np.ascontiguousarray(Cmat, dtype=np.float64).reshape(81)
        _lib.check(self.lib.dmk_update_gamma(self.ctx, _dp(c)))

    def gamma_convolution(self, field: np.ndarray, aim: np.ndarray) -> np.ndarray:
        f = np.array(field, dtype=np.float64).reshape(self.N, 9)
        a = np.ascontiguousarray(aim, dtype=np.float64).reshape(9)
        _lib.check(self.lib.dmk_gamma_convolution(self.ctx, _dp(f), _dp(a)))
        return f

    def divergence_rms(self, P: np.ndarray) -> float:
        p = np.ascontiguousarray(P, dtype=np.float64).reshape(self.N, 9)
        out = C.c_double()
        _lib.check(self.lib.dmk_divergence_rms(self.ctx, _dp(p), C.byref(out)))
        return out.value

    def dPdF(self, dt: float) -> np.ndarray:
        out = np.empty((self.N, 81))
        _lib.check(self.lib.dmk_dPdF(self.ctx, dt, _dp(out)))
        return out

    def close(self) -> None:
        if getattr(self, 'ctx', None):
            self.lib.dmk_destroy(self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class NotConverged(RuntimeError):
    """IO_error 950: no convergence after the maximum number of cutbacks."""


@dataclass
class IncrementStats:
    inc: int
    t: float
    cutback_level: int
    converged: bool
    iterations: int
    residual_evals: int
    seconds: float
    P_av: np.ndarray = field(default_factory=lambda: np.zeros((3, 3)))


def run_load_cases(solver, loadcases: list[LoadCase], N_cutback_max: int = 3, max_increments: int | None = None,
                   on_increment=None, sync=None) -> list[IncrementStats]:
    """The increment loop of DAMASK_grid (DAMASK_grid.f90:288-460) for one mechanical field.

    ``solver`` provides forward/solution/materialpoint_forward/update_coords.  Returns one
    record per converged (sub)increment.  Raises NotConverged like IO_error(950).
    """
    sub_step_factor = 2
    t = 0.0
    Delta_t = 1.0
    cut_back_level = 0
    cut_back = False
    total = 0
    stats: list[IncrementStats] = []
    for lc in loadcases:
        t_0 = t
        guess = lc.estimate_rate
        for inc in range(1, lc.N + 1):
            if max_increments is not None and total >= max_increments:
                return stats
            total += 1
            Delta_t_prev = Delta_t
            Delta_t = lc.t * geometric_fraction(lc.r, inc, lc.N) * float(sub_step_factor) ** (-float(cut_back_level))
            step_fraction = 0
            while step_fraction < sub_step_factor ** cut_back_level:
                t_remaining = lc.t + t_0 - t
                t = t + Delta_t
                step_fraction += 1
                t0 = time.perf_counter()
                solver.forward(cut_back, guess, Delta_t, Delta_t_prev, t_remaining, lc)
                if not cut_back:
                    solver.materialpoint_forward()
                sol = solver.solution()
                if sync is not None:
                    sync()
                dt_wall = time.perf_counter() - t0
                if sol.converged and sol.stagConverged:
                    solver.update_coords()
                    Delta_t_prev = Delta_t
                    cut_back = False
                    guess = True
                    rec = IncrementStats(total, t, cut_back_level, True, sol.iterationsNeeded, sol.residualEvals,
                                         dt_wall, np.array(sol.P_av[:]).reshape(3, 3, order='F'))
                    stats.append(rec)
                    if on_increment is not None:
                        on_increment(rec)
                elif cut_back_level < N_cutback_max:
                    cut_back = True
                    step_fraction = (step_fraction - 1) * sub_step_factor
                    cut_back_level += 1
                    t = t - Delta_t
                    Delta_t = Delta_t / float(sub_step_factor)
                else:
                    raise NotConverged(f'increment {total} did not converge after {N_cutback_max} cutbacks')
            cut_back_level = max(0, cut_back_level - 1)
    return stats
