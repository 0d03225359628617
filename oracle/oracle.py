"""ORACLE — test infrastructure only.

ctypes wrapper of the CPU FP64 restatement in ``oracle.cpp`` with the same method
names as :class:`damask_b200.grid.SpectralBasic`, so the reference driver loop
(``damask_b200.grid.run_load_cases``) can run either.  Only tests, the package
smoke check and the benchmark's CPU-baseline leg use it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

from damask_b200.config import BCStruct, LoadCase, Numerics, NumericsStruct, Phase, PhaseStruct, SolutionStruct

HERE = Path(__file__).resolve().parent
LIB = HERE / 'build' / 'liboracle.so'
FIELDS = {'F': 0, 'P': 1, 'F_e': 2, 'F_p': 3, 'L_p': 4, 'S': 5, 'xi_sl': 6, 'gamma_sl': 7,
          'F_lastinc': 8, 'F_i': 9, 'L_i': 10, 'F_solver': 11, 'O': 12, 'F_tau': 13, 'F_tau_lastinc': 14}
_lib = None
dp = C.POINTER(C.c_double)


def build() -> Path:
    subprocess.run(['make', '-s', '-C', str(HERE)], check=True)
    return LIB


def load() -> C.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    if not LIB.exists():
        build()
    lib = C.CDLL(str(LIB))
    vp = C.c_void_p
    sig = {
        'orc_create': (vp, [C.POINTER(C.c_int), dp, C.POINTER(C.c_int), C.c_int, dp, C.POINTER(PhaseStruct),
                            C.POINTER(NumericsStruct), C.c_int]),
        'orc_destroy': (None, [vp]),
        'orc_mech_init': (C.c_int, [vp]),
        'orc_mech_forward': (C.c_int, [vp, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double,
                                       C.POINTER(BCStruct), C.POINTER(BCStruct), dp]),
        'orc_mech_solution': (C.c_int, [vp, C.POINTER(SolutionStruct)]),
        'orc_materialpoint_forward': (C.c_int, [vp]),
        'orc_update_coords': (C.c_int, [vp]),
        'orc_get_coords': (None, [vp, dp, dp]),
        'orc_constitutive_response': (C.c_int, [vp, dp, C.c_double, dp, dp, dp, dp, C.POINTER(C.c_int)]),
        'orc_update_gamma': (None, [vp, dp]),
        'orc_gamma_convolution': (None, [vp, dp, dp]),
        'orc_divergence_rms': (C.c_double, [vp, dp]),
        'orc_curl_rms': (C.c_double, [vp, dp]),
        'orc_dPdF': (None, [vp, C.c_double, dp]),
        'orc_get_field': (C.c_int, [vp, C.c_int, dp]),
        'orc_set_field': (C.c_int, [vp, C.c_int, dp]),
        'orc_get_aims': (None, [vp, dp, dp, dp, dp]),
        'orc_counters': (None, [vp, C.POINTER(C.c_int64)]),
        'orc_schmid': (C.c_int, [C.POINTER(PhaseStruct), C.c_int, dp]),
        'orc_interaction': (C.c_int, [C.POINTER(PhaseStruct), dp]),
        'orc_fft3': (None, [dp, C.POINTER(C.c_int), C.c_int]),
        'orc_err_curl': (C.c_double, [vp]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib


def _p(a):
    return a.ctypes.data_as(dp)


class OracleSpectralBasic:
    """CPU restatement of grid_mechanical_spectral_basic (same interface as the GPU solver)."""

    def __init__(self, cells, size, material, quaternions, phase: Phase, numerics: Numerics | None = None,
                 threads: int | None = None, init: bool = True):
        self.lib = load()
        self.cells = tuple(int(c) for c in cells)
        self.size = tuple(float(s) for s in size)
        self.N = int(np.prod(self.cells))
        self.phase = phase
        self.numerics = numerics or Numerics()
        self._ps = phase.to_struct()
        self._ns = self.numerics.to_struct()
        mat = np.ascontiguousarray(material, dtype=np.int32).reshape(-1)
        q = np.ascontiguousarray(quaternions, dtype=np.float64).reshape(-1, 4)
        threads = threads or int(os.environ.get('OMP_NUM_THREADS', os.cpu_count() or 1))
        self.ctx = self.lib.orc_create((C.c_int * 3)(*self.cells), (C.c_double * 3)(*self.size),
                                       mat.ctypes.data_as(C.POINTER(C.c_int)), q.shape[0], _p(q),
                                       C.byref(self._ps), C.byref(self._ns), threads)
        if not self.ctx:
            raise ValueError('oracle: invalid phase or material map')
        self.n_slip = phase.n_slip
        if init:
            self.lib.orc_mech_init(self.ctx)

    def forward(self, cutBack, guess, Delta_t, Delta_t_old, t_remaining, lc: LoadCase) -> None:
        q = (C.c_double * 4)(*lc.q_rot)
        d, s = lc.deformation_bc(), lc.stress_bc()
        self.lib.orc_mech_forward(self.ctx, int(cutBack), int(guess), Delta_t, Delta_t_old, t_remaining,
                                  C.byref(d), C.byref(s), q)

    def solution(self) -> SolutionStruct:
        out = SolutionStruct()
        self.lib.orc_mech_solution(self.ctx, C.byref(out))
        return out

    def materialpoint_forward(self) -> None:
        self.lib.orc_materialpoint_forward(self.ctx)

    def update_coords(self) -> None:
        self.lib.orc_update_coords(self.ctx)

    def native_solver(self):
        """The oracle's procedures as a dmk_grid_solver table (its orc_bc and orc_solution have the
        layouts of dmk_bc and dmk_solution_state)."""
        from damask_b200.config import CTX_FN, FORWARD_FN, SOLUTION_FN, GridSolverStruct
        t = GridSolverStruct()
        t.ctx = self.ctx
        t.forward = C.cast(self.lib.orc_mech_forward, FORWARD_FN)
        t.solution = C.cast(self.lib.orc_mech_solution, SOLUTION_FN)
        t.update_coords = C.cast(self.lib.orc_update_coords, CTX_FN)
        t.materialpoint_forward = C.cast(self.lib.orc_materialpoint_forward, CTX_FN)
        return t

    def get_coords(self) -> tuple[np.ndarray, np.ndarray]:
        ip = np.empty((self.N, 3))
        nodes = np.empty((int(np.prod([c + 1 for c in self.cells])), 3))
        self.lib.orc_get_coords(self.ctx, _p(ip), _p(nodes))
        return ip, nodes

    def get_field(self, name: str) -> np.ndarray:
        k = self.n_slip if name in ('xi_sl', 'gamma_sl') else 4 if name == 'O' else 9
        out = np.empty((self.N, k))
        if self.lib.orc_get_field(self.ctx, FIELDS[name], _p(out)) != 0:
            raise KeyError(name)
        return out

    def set_field(self, name: str, values) -> None:
        v = np.ascontiguousarray(values, dtype=np.float64)
        if self.lib.orc_set_field(self.ctx, FIELDS[name], _p(v)) != 0:
            raise KeyError(name)

    def aims(self) -> dict:
        F, P, Cv, Cm = np.zeros(9), np.zeros(9), np.zeros(81), np.zeros(81)
        self.lib.orc_get_aims(self.ctx, _p(F), _p(P), _p(Cv), _p(Cm))
        return {'F_aim': F, 'P_aim': P, 'C_volAvg': Cv, 'C_minMaxAvg': Cm}

    def counters(self) -> np.ndarray:
        out = (C.c_int64 * 4)()
        self.lib.orc_counters(self.ctx, out)
        return np.array(out[:])

    def constitutive_response(self, F, dt):
        F = np.ascontiguousarray(F, dtype=np.float64).reshape(self.N, 9)
        P = np.empty((self.N, 9))
        P_av, Cv, Cm = np.zeros(9), np.zeros(81), np.zeros(81)
        st = C.c_int()
        self.lib.orc_constitutive_response(self.ctx, _p(F), dt, _p(P), _p(P_av), _p(Cv), _p(Cm), C.byref(st))
        return P, P_av, Cv, Cm, st.value

    def update_gamma(self, Cmat) -> None:
        c = np.ascontiguousarray(Cmat, dtype=np.float64).reshape(81)
        self.lib.orc_update_gamma(self.ctx, _p(c))

    def gamma_convolution(self, field, aim) -> np.ndarray:
        f = np.array(field, dtype=np.float64).reshape(self.N, 9)
        a = np.ascontiguousarray(aim, dtype=np.float64).reshape(9)
        self.lib.orc_gamma_convolution(self.ctx, _p(f), _p(a))
        return f

    def curl_rms(self, F) -> float:
        return self.lib.orc_curl_rms(self.ctx, _p(np.ascontiguousarray(F, dtype=np.float64)))

    def divergence_rms(self, P) -> float:
        p = np.ascontiguousarray(P, dtype=np.float64).reshape(self.N, 9)
        return self.lib.orc_divergence_rms(self.ctx, _p(p))

    def dPdF(self, dt) -> np.ndarray:
        out = np.empty((self.N, 81))
        self.lib.orc_dPdF(self.ctx, dt, _p(out))
        return out

    def close(self) -> None:
        if getattr(self, 'ctx', None):
            self.lib.orc_destroy(self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def schmid(phase: Phase, sense: int = 1) -> np.ndarray:
    lib = load()
    ps = phase.to_struct()
    out = np.zeros((phase.n_slip, 9))
    n = lib.orc_schmid(C.byref(ps), sense, _p(out))
    return out[:n].reshape(n, 3, 3).transpose(0, 2, 1)


def interaction(phase: Phase) -> np.ndarray:
    lib = load()
    ps = phase.to_struct()
    out = np.zeros((phase.n_slip, phase.n_slip))
    n = lib.orc_interaction(C.byref(ps), _p(out))
    if n < 0:
        raise ValueError('too few interaction values')
    return out


def fft3(x: np.ndarray, sign: int = -1) -> np.ndarray:
    """3D complex FFT of an array indexed [z, y, x] (x fastest), unnormalised."""
    lib = load()
    a = np.ascontiguousarray(x, dtype=np.complex128).copy()
    n = (C.c_int * 3)(a.shape[2], a.shape[1], a.shape[0])
    lib.orc_fft3(a.ctypes.data_as(dp), n, sign)
    return a
