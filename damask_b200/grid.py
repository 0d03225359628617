"""Host side of the grid mechanical solver: the plugin objects and the increment loop.

``SpectralBasic`` mirrors the five procedures DAMASK's grid driver selects for the
``spectral_basic`` solver (``src/grid/DAMASK_grid.f90:110-119,171-206``):
``init`` (constructor), ``forward``, ``solution``, ``update_coords`` and the
materialpoint forward that follows a converged increment; ``SpectralPolarization`` the
same for ``spectral_polarization``.  All compute runs in ``libdamask_b200.so`` on the
GPU; this module only marshals host arrays.

``run_load_cases`` restates the driver's increment loop with its global cutback
(``DAMASK_grid.f90:288-460``) for any object with that interface, so the same
host logic drives the CUDA path and, in tests, the CPU oracle;
``run_load_cases_native`` runs the library's C++ version of that loop.
"""
from __future__ import annotations

import copy
import ctypes as C
import time
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

from . import _lib
from .config import LoadCase, Numerics, Phase, RestartStruct, SolutionStruct, geometric_fraction

FIELDS = {'F': 0, 'P': 1, 'F_e': 2, 'F_p': 3, 'L_p': 4, 'S': 5, 'xi_sl': 6, 'gamma_sl': 7,
          'F_lastinc': 8, 'F_i': 9, 'L_i': 10, 'F_solver': 11, 'O': 12, 'F_tau': 13, 'F_tau_lastinc': 14}

PRECISIONS = {'fp64': 0, 'mixed': 1}


def _dp(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def node_count(cells) -> int:
    return int(np.prod([c + 1 for c in cells]))


def coordinates0(cells, size) -> tuple[np.ndarray, np.ndarray]:
    """Undeformed cell centres and nodes, x fastest (IPcoordinates0 and nodes0,
    src/grid/discretization_grid.f90:270-313)."""
    step = np.asarray(size, float) / np.asarray(cells)
    ijk = np.stack(np.meshgrid(*[np.arange(c) for c in cells], indexing='ij'), -1).reshape(-1, 3, order='F')
    nodes = np.stack(np.meshgrid(*[np.arange(c + 1) for c in cells], indexing='ij'), -1).reshape(-1, 3, order='F')
    return step * (ijk + 0.5), step * nodes


def displacements(cells, size, ip: np.ndarray, nodes: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    """u_p and u_n of the result file: current minus undeformed coordinates
    (discretization_result, src/discretization.f90:81-96)."""
    ip0, nodes0 = coordinates0(cells, size)
    return ip - ip0, nodes - nodes0


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
        # running totals over all solution calls: updates, state iterations, Newton
        # iterations, residual evaluations; and device ms by stage
        self.total_counters = np.zeros(4, dtype=np.int64)
        self.total_ms = np.zeros(3)

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
        self.total_counters += self.counters()
        self.total_ms += self.timings()
        return out

    def materialpoint_forward(self) -> None:
        _lib.check(self.lib.dmk_materialpoint_forward(self.ctx))

    def autotune(self, reps: int = 2) -> dict:
        """dmk_autotune: time the constitutive evaluation at the current state for every stress-kernel
        variant and voxel-chunk count and keep the fastest (results unchanged)."""
        rep = np.zeros(36)
        n = C.c_int()
        _lib.check(self.lib.dmk_autotune(self.ctx, int(reps), _dp(rep), C.byref(n)))
        return {'candidates': [(int(rep[3 * k]), int(rep[3 * k + 1]), float(rep[3 * k + 2])) for k in range(n.value)],
                'chosen': self.tuning()}

    def tuning(self) -> tuple[int, int]:
        """(stress-kernel blocks per SM, voxel chunks) in use."""
        b, k = C.c_int(), C.c_int()
        _lib.check(self.lib.dmk_get_tuning(self.ctx, C.byref(b), C.byref(k)))
        return b.value, k.value

    def set_tuning(self, stress_blocks: int, chunks: int) -> None:
        _lib.check(self.lib.dmk_set_tuning(self.ctx, int(stress_blocks), int(chunks)))

    def update_coords(self) -> None:
        _lib.check(self.lib.dmk_mech_update_coords(self.ctx))

    def get_coords(self) -> tuple[np.ndarray, np.ndarray]:
        """Cell-centre (N, 3) and node ((c1+1)(c2+1)(c3+1), 3) coordinates, x fastest."""
        ip = np.empty((self.N, 3))
        nodes = np.empty((node_count(self.cells), 3))
        _lib.check(self.lib.dmk_get_coords(self.ctx, _dp(ip), _dp(nodes)))
        return ip, nodes

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

    # -- restart (grid_mech_spectral_basic.f90:198-235,378-416; phase_mechanical.f90:1248-1280) --
    RESTART_FIELDS = ('F', 'F_lastinc', 'F_phase', 'F_p', 'L_p')
    RESTART_AIMS = ('P_aim', 'F_aim', 'F_aim_lastinc', 'F_aimDot', 'C_volAvg', 'C_volAvgLastInc', 'C_minMaxAvg')

    @property
    def restart_fields(self) -> tuple:
        pol = ('F_tau', 'F_tau_lastinc') if self.numerics.solver == 'spectral_polarization' else ()
        return self.RESTART_FIELDS + pol

    def restart_write(self) -> dict:
        """The data the reference writes to its restart file, as numpy arrays (per voxel,
        voxel-major)."""
        d = {k: np.empty((self.N, 9)) for k in self.restart_fields}
        d['omega_plastic'] = np.empty((self.N, 2 * self.phase.n_slip))
        r = RestartStruct()
        for k in self.restart_fields + ('omega_plastic',):
            setattr(r, k, _dp(d[k]))
        _lib.check(self.lib.dmk_restart_write(self.ctx, C.byref(r)))
        for k in self.RESTART_AIMS:
            d[k] = np.array(getattr(r, k)[:])
        return d

    def restart_read(self, d: dict) -> None:
        """Resume from restart data on this (freshly initialised) context."""
        keep = {k: np.ascontiguousarray(d[k], dtype=np.float64) for k in self.restart_fields + ('omega_plastic',)}
        if keep['omega_plastic'].shape != (self.N, 2 * self.phase.n_slip) or \
                any(keep[k].shape != (self.N, 9) for k in self.restart_fields):
            raise ValueError('restart data do not match the grid and phase of this context')
        r = RestartStruct()
        for k, v in keep.items():
            setattr(r, k, _dp(v))
        for k in self.RESTART_AIMS:
            getattr(r, k)[:] = [float(x) for x in np.ravel(d[k])]
        _lib.check(self.lib.dmk_restart_read(self.ctx, C.byref(r)))


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

    def launches(self) -> int:
        out = C.c_int64()
        _lib.check(self.lib.dmk_get_launches(self.ctx, C.byref(out)))
        return out.value

    def timer_start(self) -> None:
        _lib.check(self.lib.dmk_timer_start(self.ctx))

    def timer_stop(self) -> float:
        ms = C.c_double()
        _lib.check(self.lib.dmk_timer_stop(self.ctx, C.byref(ms)))
        return ms.value

    # -- device checkpoints and the adjoint of increments ----------------------------------------
    def checkpoint_save(self, slot: int) -> None:
        """The complete solver and phase state into device checkpoint `slot` (dmk_checkpoint_save)."""
        _lib.check(self.lib.dmk_checkpoint_save(self.ctx, int(slot)))

    def checkpoint_restore(self, slot: int) -> None:
        _lib.check(self.lib.dmk_checkpoint_restore(self.ctx, int(slot)))

    def adj_begin(self, n_slots: int) -> None:
        _lib.check(self.lib.dmk_adj_begin(self.ctx, int(n_slots)))

    def adj_record(self, slot: int) -> None:
        _lib.check(self.lib.dmk_adj_record(self.ctx, int(slot)))

    def adj_step(self, slot: int, P_av_bar: np.ndarray, theta_bar: np.ndarray) -> int:
        """One increment of the adjoint (dmk_adj_step): P_av_bar (3, 3) = dL/d<P> of the increment;
        theta_bar (20,) accumulates.  Returns the Krylov iterations of the transposed solve."""
        pb = np.ascontiguousarray(np.asarray(P_av_bar, float).reshape(3, 3).reshape(-1, order='F'))
        its = C.c_int()
        _lib.check(self.lib.dmk_adj_step(self.ctx, int(slot), _dp(pb), _dp(theta_bar), C.byref(its)))
        return its.value

    def adj_finish(self, theta_bar: np.ndarray) -> None:
        _lib.check(self.lib.dmk_adj_finish(self.ctx, _dp(theta_bar)))

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

    def curl_rms(self, F: np.ndarray) -> float:
        f = np.ascontiguousarray(F, dtype=np.float64).reshape(self.N, 9)
        out = C.c_double()
        _lib.check(self.lib.dmk_curl_rms(self.ctx, _dp(f), C.byref(out)))
        return out.value

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


class SpectralPolarization(SpectralBasic):
    """grid_mech_spectral_polarization on one GPU: the augmented-Lagrangian / polarization
    scheme with F and F_tau as solution fields (alpha, beta, eps_*_curl(F) from numerics)."""

    def __init__(self, cells, size, material: np.ndarray, quaternions: np.ndarray, phase: Phase,
                 numerics: Numerics | None = None, precision: str = 'fp64', device: int = 0):
        num = copy.copy(numerics or Numerics())
        num.solver = 'spectral_polarization'
        super().__init__(cells, size, material, quaternions, phase, num, precision, device)


def mechanical_solver(name: str):
    """The plugin class for load.yaml ``solver: mechanical: <name>`` (DAMASK_grid.f90:171-206)."""
    return {'spectral_basic': SpectralBasic, 'spectral_polarization': SpectralPolarization}[name]


def save_restart(path, data: dict, increment: int, phase_name: str = 'phase', homogenization_name: str = 'SX') -> None:
    """The restart file <job>_restart.hdf5 in the reference's layout: the solver group of
    grid_mech_spectral_basic.f90:378-416 (F, F_lastinc per voxel; P_aim, F_aim, F_aim_lastinc,
    F_aimDot; C_volAvg, C_volAvgLastInc, C_minMaxAvg; the polarization scheme adds F_tau and
    F_tau_lastinc, grid_mech_spectral_polarization.f90:412-415), the phase group of
    mechanical_restartWrite (phase_mechanical.f90:1248-1261: omega_plastic, F, F_p, F_i, L_p, L_i)
    and the homogenization group (homogenization.f90:492-517, no state for one constituent).
    Fortran arrays (3,3,N) are HDF5 datasets of shape (N,3,3), as libhdf5 stores them.  The
    increment is kept as the root attribute 'restart_increment' (the reference's driver takes it
    from its command line)."""
    from .dadf5 import H5Writer
    N = np.asarray(data['F']).shape[0]

    def t33n(a):
        return np.ascontiguousarray(np.asarray(a, dtype=np.float64).reshape(N, 3, 3))

    with H5Writer(path) as w:
        w.dataset('solver/F', t33n(data['F']))
        w.dataset('solver/F_lastinc', t33n(data['F_lastinc']))
        for k in ('P_aim', 'F_aim', 'F_aim_lastinc', 'F_aimDot'):
            w.dataset(f'solver/{k}', np.asarray(data[k], dtype=np.float64).reshape(3, 3))
        for k in ('C_volAvg', 'C_volAvgLastInc', 'C_minMaxAvg'):
            w.dataset(f'solver/{k}', np.asarray(data[k], dtype=np.float64).reshape(3, 3, 3, 3))
        for k in ('F_tau', 'F_tau_lastinc'):
            if k in data:
                w.dataset(f'solver/{k}', t33n(data[k]))
        g = f'phase/{phase_name}'
        w.dataset(f'{g}/omega_plastic', np.ascontiguousarray(data['omega_plastic'], dtype=np.float64))
        w.dataset(f'{g}/F', t33n(data['F_phase']))
        w.dataset(f'{g}/F_p', t33n(data['F_p']))
        w.dataset(f'{g}/F_i', np.tile(np.eye(3), (N, 1, 1)))
        w.dataset(f'{g}/L_p', t33n(data['L_p']))
        w.dataset(f'{g}/L_i', np.zeros((N, 3, 3)))
        w.group(f'homogenization/{homogenization_name}')
        w.attrs('/', {'restart_increment': np.int64(increment)})


def load_restart(path, phase_name: str = 'phase') -> tuple[dict, int]:
    """The restart data of save_restart (or of the reference's restart file, whose increment is
    then 0: the caller knows it) as the arrays of SpectralBasic.restart_read."""
    from .h5read import DADF5
    f = DADF5(path)
    d = {'F': f.read('solver/F'), 'F_lastinc': f.read('solver/F_lastinc')}
    N = d['F'].shape[0]
    d = {k: v.reshape(N, 9) for k, v in d.items()}
    for k in ('P_aim', 'F_aim', 'F_aim_lastinc', 'F_aimDot', 'C_volAvg', 'C_volAvgLastInc', 'C_minMaxAvg'):
        d[k] = f.read(f'solver/{k}').reshape(-1)
    for k in ('F_tau', 'F_tau_lastinc'):
        if k in f.keys('solver'):
            d[k] = f.read(f'solver/{k}').reshape(N, 9)
    g = f'phase/{phase_name}'
    d['omega_plastic'] = f.read(f'{g}/omega_plastic')
    d['F_phase'] = f.read(f'{g}/F').reshape(N, 9)
    d['F_p'] = f.read(f'{g}/F_p').reshape(N, 9)
    d['L_p'] = f.read(f'{g}/L_p').reshape(N, 9)
    inc = f.attrs('').get('restart_increment', 0)
    return d, int(np.asarray(inc).reshape(-1)[0]) if np.size(inc) else 0


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


class IncrementDriver:
    """The increment loop of DAMASK_grid (DAMASK_grid.f90:288-460) for one mechanical field,
    one increment per :meth:`step` call.

    ``solver`` provides forward/solution/materialpoint_forward/update_coords.  A step
    runs all (sub)increments of one load-case increment including the global cutback
    (time step halved up to ``N_cutback_max`` times); it raises NotConverged like
    IO_error(950).
    """
    sub_step_factor = 2

    def __init__(self, solver, loadcases: list[LoadCase], N_cutback_max: int = 3, sync=None, restart_inc: int = 0):
        self.restart_inc = restart_inc       # increments up to this one were computed before a restart
        self.solver = solver
        self.loadcases = loadcases
        self.N_cutback_max = N_cutback_max
        self.sync = sync
        self.t = 0.0
        self.Delta_t = 1.0
        self.cut_back_level = 0
        self.cut_back = False
        self.total = 0
        self._l = 0
        self._inc = 0
        self._t_0 = 0.0
        self._guess = loadcases[0].estimate_rate if loadcases else True

    @property
    def done(self) -> bool:
        return self._l >= len(self.loadcases)

    _STATE = ('t', 'Delta_t', 'cut_back_level', 'cut_back', 'total', '_l', '_inc', '_t_0', '_guess')

    def state(self) -> dict:
        """The loop's position (time, increment counters, cutback level, guess flag), so that a
        solver restored from a checkpoint taken at this point continues the same sequence."""
        return {k: getattr(self, k) for k in self._STATE}

    def set_state(self, st: dict) -> None:
        for k in self._STATE:
            setattr(self, k, st[k])

    def step(self) -> list[IncrementStats]:
        """One load-case increment with the solver's own solution call."""
        gen = self.step_requests()
        try:
            gen.send(None)
            while True:
                gen.send(self.solver.solution())
        except StopIteration as stop:
            return stop.value

    def step_requests(self):
        """The increment of :meth:`step` as a generator: it yields where the solver's solution is
        needed (after forward and materialpoint_forward), is sent that solution, and returns the
        converged (sub)increments.  A batch drives many drivers this way and solves their requests
        together."""
        if self.done:
            return []
        lc = self.loadcases[self._l]
        if self._inc == 0:
            self._t_0 = self.t
            self._guess = lc.estimate_rate
        self._inc += 1
        inc = self._inc
        self.total += 1
        out: list[IncrementStats] = []
        ssf = self.sub_step_factor
        Delta_t_prev = self.Delta_t
        self.Delta_t = lc.t * geometric_fraction(lc.r, inc, lc.N) * float(ssf) ** (-float(self.cut_back_level))
        if self.total <= self.restart_inc:
            # DAMASK_grid.f90:301-303: before the restart increment only the time advances
            self.t = self.t + self.Delta_t
            self._guess = True
            if self._inc >= lc.N:
                self._l += 1
                self._inc = 0
            return out
        step_fraction = 0
        while step_fraction < ssf ** self.cut_back_level:
            t_remaining = lc.t + self._t_0 - self.t
            self.t = self.t + self.Delta_t
            step_fraction += 1
            t0 = time.perf_counter()
            self.solver.forward(self.cut_back, self._guess, self.Delta_t, Delta_t_prev, t_remaining, lc)
            if not self.cut_back:
                self.solver.materialpoint_forward()
            sol = yield
            if self.sync is not None:
                self.sync()
            dt_wall = time.perf_counter() - t0
            if sol.converged and sol.stagConverged:
                self.solver.update_coords()
                Delta_t_prev = self.Delta_t
                self.cut_back = False
                self._guess = True
                out.append(IncrementStats(self.total, self.t, self.cut_back_level, True, sol.iterationsNeeded,
                                          sol.residualEvals, dt_wall, np.array(sol.P_av[:]).reshape(3, 3, order='F')))
            elif self.cut_back_level < self.N_cutback_max:
                self.cut_back = True
                step_fraction = (step_fraction - 1) * ssf
                self.cut_back_level += 1
                self.t = self.t - self.Delta_t
                self.Delta_t = self.Delta_t / float(ssf)
            else:
                raise NotConverged(f'increment {self.total} did not converge after {self.N_cutback_max} cutbacks')
        self.cut_back_level = max(0, self.cut_back_level - 1)
        if self._inc >= lc.N:
            self._l += 1
            self._inc = 0
        return out


STA_HEADER = 'Increment Time CutbackLevel Converged IterationsNeeded StagIterationsNeeded'


def sta_line(rec: IncrementStats) -> str:
    """One row of the job's .sta file per converged (sub)increment (DAMASK_grid.f90:394-395):
    total increment, time, cutback level, converged, iterations, staggered iterations (0 with
    the mechanical field alone)."""
    return f'{rec.inc:12d} {rec.t:24.16e} {rec.cutback_level:12d} {"T" if rec.converged else "F":>2} ' \
           f'{rec.iterations:12d} {0:12d}'


def run_load_cases(solver, loadcases: list[LoadCase], N_cutback_max: int = 3, max_increments: int | None = None,
                   on_increment=None, sync=None, restart_inc: int = 0, sta=None) -> list[IncrementStats]:
    """Run the whole load-case list (or its first ``max_increments`` increments); after a
    restart, ``restart_inc`` increments are skipped (only the time advances).  With ``sta`` (a
    path) the statistics table of DAMASK_grid.f90:268-278 is written (appended after a restart)."""
    drv = IncrementDriver(solver, loadcases, N_cutback_max, sync, restart_inc)
    stats: list[IncrementStats] = []
    fh = None
    if sta is not None:
        exists = Path(sta).exists()
        fh = open(sta, 'a' if (restart_inc and exists) else 'w')
        if not (restart_inc and exists):
            fh.write(STA_HEADER + '\n')
    try:
        while not drv.done and (max_increments is None or drv.total < max_increments):
            for rec in drv.step():
                stats.append(rec)
                if fh is not None:
                    fh.write(sta_line(rec) + '\n')
                    fh.flush()
                if on_increment is not None:
                    on_increment(rec)
    finally:
        if fh is not None:
            fh.close()
    return stats


def run_load_cases_native(solver, loadcases: list[LoadCase], N_cutback_max: int = 3,
                          max_increments: int | None = None, on_increment=None,
                          restart_inc: int = 0) -> list[IncrementStats]:
    """run_load_cases through the library's C++ increment loop (dmk_grid_run): for a
    SpectralBasic the loop calls the context directly (no interpreter between the procedures);
    any other solver offers ``native_solver()``, a dmk_grid_solver table of its procedures."""
    from .config import INCREMENT_CB, loadstep_structs
    lib = _lib.load()
    steps = loadstep_structs(loadcases)
    stats: list[IncrementStats] = []
    clock = [time.perf_counter()]

    def cb(info_p, _user):
        i = info_p.contents
        now = time.perf_counter()
        rec = IncrementStats(i.inc, i.t, i.cutback_level, bool(i.converged), i.iterations, i.residual_evals,
                             now - clock[0], np.array(i.P_av[:]).reshape(3, 3, order='F'))
        clock[0] = now
        stats.append(rec)
        if on_increment is not None:
            on_increment(rec)
        return 0

    cfn = INCREMENT_CB(cb)
    nmax = int(max_increments or 0)
    if isinstance(solver, SpectralBasic):
        # (SpectralBasic.total_counters / total_ms are kept by its Python solution() only)
        rc = lib.dmk_grid_run_ctx(solver.ctx, steps, len(loadcases), N_cutback_max, restart_inc, nmax, cfn, None)
    else:
        table = solver.native_solver()
        rc = lib.dmk_grid_run(C.byref(table), steps, len(loadcases), N_cutback_max, restart_inc, nmax, cfn, None)
    if rc == -7:
        raise NotConverged(lib.dmk_last_error().decode())
    _lib.check(rc)
    return stats


def read_sta(path) -> list[tuple]:
    """Rows of a .sta file: (increment, time, cutback level, converged, iterations, staggered)."""
    rows = []
    for line in Path(path).read_text().splitlines()[1:]:
        p = line.split()
        rows.append((int(p[0]), float(p[1]), int(p[2]), p[3] == 'T', int(p[4]), int(p[5])))
    return rows
