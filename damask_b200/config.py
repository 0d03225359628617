"""material.yaml / numerics.yaml / load.yaml in DAMASK's key layout.

The keys and defaults restate the reference readers:

* phase (one phase, Hooke + phenopowerlaw slip):
  ``phase_mechanical_elastic.f90:22-84``, ``phase_mechanical_plastic_phenopowerlaw.f90:76-295``;
* numerics: ``grid_mech_spectral_basic.f90:130-136`` (solver.grid.mechanical),
  ``spectral_utilities.f90:176-224`` (solver.grid.FFT), ``phase_mechanical.f90:281-295``
  (phase.mechanical), ``DAMASK_grid.f90:145-148`` (solver.grid);
* load cases: ``DAMASK_grid.f90:472-689`` (``parse_and_print_load_cases``), with
  ``'x'`` marking a component that is not prescribed (``get_masked_tensor`` :692-718).

The values are packed into the plain C structs of the C-ABI (``include/damask_b200.h``).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np


class PhaseStruct(C.Structure):
    _fields_ = [('lattice', C.c_int), ('n_families', C.c_int), ('N_sl', C.c_int * 4),
                ('C11', C.c_double), ('C12', C.c_double), ('C44', C.c_double),
                ('dot_gamma_0', C.c_double * 4), ('n', C.c_double * 4), ('a', C.c_double * 4),
                ('h_0', C.c_double * 4), ('xi_0', C.c_double * 4), ('xi_inf', C.c_double * 4),
                ('c_1', C.c_double * 4), ('c_2', C.c_double * 4), ('f_sat', C.c_double * 4),
                ('n_h', C.c_int), ('h_sl_sl', C.c_double * 64),
                ('n_nonschmid', C.c_int), ('a_nonschmid', C.c_double * 6),
                ('atol_xi', C.c_double), ('atol_gamma', C.c_double)]


class NumericsStruct(C.Structure):
    _fields_ = [('N_iter_min', C.c_int), ('N_iter_max', C.c_int),
                ('eps_abs_div', C.c_double), ('eps_rel_div', C.c_double),
                ('eps_abs_P', C.c_double), ('eps_rel_P', C.c_double),
                ('update_gamma', C.c_int), ('divergence_correction', C.c_int), ('derivative', C.c_int),
                ('r_cutback_min', C.c_double), ('r_cutback', C.c_double), ('r_increase', C.c_double),
                ('eps_rel_state', C.c_double), ('N_iter_state_max', C.c_int),
                ('N_iter_Lp_max', C.c_int), ('r_linesearch_Lp', C.c_double), ('eps_rel_Lp', C.c_double),
                ('eps_abs_Lp', C.c_double), ('f_update_jacobi_Lp', C.c_int),
                ('N_iter_Li_max', C.c_int), ('r_linesearch_Li', C.c_double), ('eps_rel_Li', C.c_double),
                ('eps_abs_Li', C.c_double), ('f_update_jacobi_Li', C.c_int),
                ('snes_type', C.c_int), ('anderson_m', C.c_int),
                ('solver', C.c_int), ('alpha', C.c_double), ('beta', C.c_double),
                ('eps_abs_curl', C.c_double), ('eps_rel_curl', C.c_double), ('snes_max_it', C.c_int)]


class BCStruct(C.Structure):
    _fields_ = [('values', C.c_double * 9), ('mask', C.c_int * 9), ('type', C.c_int)]


class RestartStruct(C.Structure):
    """dmk_restart (include/damask_b200.h)."""
    _fields_ = [('F', C.POINTER(C.c_double)), ('F_lastinc', C.POINTER(C.c_double)),
                ('F_phase', C.POINTER(C.c_double)), ('F_p', C.POINTER(C.c_double)),
                ('L_p', C.POINTER(C.c_double)), ('omega_plastic', C.POINTER(C.c_double)),
                ('P_aim', C.c_double * 9), ('F_aim', C.c_double * 9), ('F_aim_lastinc', C.c_double * 9),
                ('F_aimDot', C.c_double * 9), ('C_volAvg', C.c_double * 81), ('C_volAvgLastInc', C.c_double * 81),
                ('C_minMaxAvg', C.c_double * 81), ('F_tau', C.POINTER(C.c_double)),
                ('F_tau_lastinc', C.POINTER(C.c_double))]


class LoadStepStruct(C.Structure):
    """dmk_loadstep (include/damask_b200.h)."""
    _fields_ = [('deformation', BCStruct), ('stress', BCStruct), ('q_rot', C.c_double * 4), ('t', C.c_double),
                ('N', C.c_int), ('r', C.c_double), ('f_out', C.c_int), ('f_restart', C.c_int),
                ('estimate_rate', C.c_int)]


class IncrementInfoStruct(C.Structure):
    """dmk_increment_info (include/damask_b200.h)."""
    _fields_ = [('inc', C.c_int), ('t', C.c_double), ('cutback_level', C.c_int), ('converged', C.c_int),
                ('iterations', C.c_int), ('residual_evals', C.c_int), ('load_step', C.c_int),
                ('step_inc', C.c_int), ('P_av', C.c_double * 9)]


class SolutionStruct(C.Structure):
    _fields_ = [('iterationsNeeded', C.c_int), ('converged', C.c_int), ('stagConverged', C.c_int),
                ('residualEvals', C.c_int), ('err_div', C.c_double), ('err_BC', C.c_double),
                ('P_av', C.c_double * 9)]


INCREMENT_CB = C.CFUNCTYPE(C.c_int, C.POINTER(IncrementInfoStruct), C.c_void_p)
BATCH_INCREMENT_CB = C.CFUNCTYPE(C.c_int, C.c_int, C.POINTER(IncrementInfoStruct), C.c_void_p)
FORWARD_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double,
                         C.POINTER(BCStruct), C.POINTER(BCStruct), C.POINTER(C.c_double))
SOLUTION_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.POINTER(SolutionStruct))
CTX_FN = C.CFUNCTYPE(C.c_int, C.c_void_p)


class GridSolverStruct(C.Structure):
    """dmk_grid_solver: the five plugin procedures as function pointers."""
    _fields_ = [('ctx', C.c_void_p), ('forward', FORWARD_FN), ('solution', SOLUTION_FN),
                ('update_coords', CTX_FN), ('materialpoint_forward', CTX_FN)]


def loadstep_structs(loadcases) -> C.Array:
    arr = (LoadStepStruct * len(loadcases))()
    for s, lc in zip(arr, loadcases):
        s.deformation, s.stress = lc.deformation_bc(), lc.stress_bc()
        s.q_rot[:] = [float(x) for x in lc.q_rot]
        s.t, s.N, s.r = float(lc.t), int(lc.N), float(lc.r)
        s.f_out, s.f_restart, s.estimate_rate = int(lc.f_out), int(lc.f_restart), int(bool(lc.estimate_rate))
    return arr


LATTICES = {'cF': 0, 'cI': 1}
SOLVERS = {'spectral_basic': 0, 'spectral_polarization': 1}
# solver.grid.FFT.derivative (spectral_utilities.f90:198-209)
DERIVATIVES = {'continuous': 0, 'central_difference': 1, 'FWBW_difference': 2}
BC_TYPES = {'L': 1, 'dot_F': 2, 'F_dot': 2, 'F': 3, 'P': 4, 'dot_P': 5, 'P_dot': 5}


@dataclass
class Phase:
    lattice: str
    C_11: float
    C_12: float
    C_44: float
    N_sl: list[int]
    dot_gamma_0_sl: list[float]
    n_sl: list[float]
    a_sl: list[float]
    h_0_sl_sl: list[float]
    xi_0_sl: list[float]
    xi_inf_sl: list[float]
    h_sl_sl: list[float]
    c_1: list[float] | None = None
    c_2: list[float] | None = None
    f_sat_sl_tw: list[float] | None = None
    a_nonschmid: list[float] = field(default_factory=list)
    atol_xi: float = 1.0
    atol_gamma: float = 1.0e-6

    @property
    def n_slip(self) -> int:
        return int(sum(self.N_sl))

    @classmethod
    def from_dict(cls, phase: dict) -> 'Phase':
        mech = phase['mechanical']
        el, pl = mech['elastic'], mech['plastic']
        if el.get('type') != 'Hooke':
            raise ValueError(f"unsupported elasticity {el.get('type')}")
        if pl.get('type') != 'phenopowerlaw':
            raise ValueError(f"unsupported plasticity {pl.get('type')}")
        if pl.get('N_tw'):
            raise ValueError('twinning systems are not on this path')
        if phase['lattice'] not in LATTICES:
            raise ValueError(f"unsupported lattice {phase['lattice']}")

        def c(v):
            return float(v[0]) if isinstance(v, (list, tuple)) else float(v)
        ns = pl.get('a_non-Schmid', [])
        return cls(lattice=phase['lattice'], C_11=c(el['C_11']), C_12=c(el['C_12']), C_44=c(el['C_44']),
                   N_sl=[int(v) for v in pl['N_sl']],
                   dot_gamma_0_sl=[float(v) for v in pl['dot_gamma_0_sl']],
                   n_sl=[float(v) for v in pl['n_sl']], a_sl=[float(v) for v in pl['a_sl']],
                   h_0_sl_sl=[float(v) for v in pl['h_0_sl-sl']],
                   xi_0_sl=[float(v) for v in pl['xi_0_sl']],
                   xi_inf_sl=[float(v) for v in pl['xi_inf_sl']],
                   h_sl_sl=[float(v) for v in pl['h_sl-sl']],
                   c_1=pl.get('c_1'), c_2=pl.get('c_2'), f_sat_sl_tw=pl.get('f_sat_sl-tw'),
                   a_nonschmid=[float(v) for v in (ns[0] if ns else [])],
                   atol_xi=float(pl.get('atol_xi', 1.0)), atol_gamma=float(pl.get('atol_gamma', 1.0e-6)))

    def to_struct(self) -> PhaseStruct:
        nf = len(self.N_sl)
        if nf > 4 or len(self.h_sl_sl) > 64 or len(self.a_nonschmid) > 6:
            raise ValueError('phase definition exceeds the C-ABI limits')
        for name in ('dot_gamma_0_sl', 'n_sl', 'a_sl', 'h_0_sl_sl', 'xi_0_sl', 'xi_inf_sl'):
            if len(getattr(self, name)) != nf:
                raise ValueError(f'{name} needs one value per slip family')
        s = PhaseStruct()
        s.lattice = LATTICES[self.lattice]
        s.n_families = nf
        for f in range(nf):
            s.N_sl[f] = self.N_sl[f]
            s.dot_gamma_0[f] = self.dot_gamma_0_sl[f]
            s.n[f] = self.n_sl[f]
            s.a[f] = self.a_sl[f]
            s.h_0[f] = self.h_0_sl_sl[f]
            s.xi_0[f] = self.xi_0_sl[f]
            s.xi_inf[f] = self.xi_inf_sl[f]
            s.c_1[f] = float(self.c_1[f]) if self.c_1 else 0.0
            s.c_2[f] = float(self.c_2[f]) if self.c_2 else 1.0
            s.f_sat[f] = float(self.f_sat_sl_tw[f]) if self.f_sat_sl_tw else 0.0
        s.C11, s.C12, s.C44 = self.C_11, self.C_12, self.C_44
        s.n_h = len(self.h_sl_sl)
        for i, v in enumerate(self.h_sl_sl):
            s.h_sl_sl[i] = v
        s.n_nonschmid = len(self.a_nonschmid)
        for i, v in enumerate(self.a_nonschmid):
            s.a_nonschmid[i] = v
        s.atol_xi, s.atol_gamma = self.atol_xi, self.atol_gamma
        return s


@dataclass
class Numerics:
    N_iter_min: int = 1
    N_iter_max: int = 100
    eps_abs_div: float = 1.0e-4
    eps_rel_div: float = 5.0e-4
    eps_abs_P: float = 1.0e3
    eps_rel_P: float = 1.0e-3
    update_gamma: bool = False
    divergence_correction: str = 'grid+size'
    # solver.grid.FFT.memory_efficient / FFTW_plan_mode (spectral_utilities.f90:176, :210-223):
    # accepted and validated; Gamma_hat is always evaluated on the fly (both settings give the same
    # operator) and cuFFT has no planner modes
    memory_efficient: bool = True
    FFTW_plan_mode: str = 'FFTW_MEASURE'
    derivative: str = 'continuous'
    N_cutback_max: int = 3
    r_cutback_min: float = 1.0e-3
    r_cutback: float = 0.25
    r_increase: float = 1.5
    eps_rel_state: float = 1.0e-6
    N_iter_state_max: int = 20
    N_iter_Lp_max: int = 40
    r_linesearch_Lp: float = 0.5
    eps_rel_Lp: float = 1.0e-6
    eps_abs_Lp: float = 1.0e-8
    f_update_jacobi_Lp: int = 1
    N_iter_Li_max: int = 40
    r_linesearch_Li: float = 0.5
    eps_rel_Li: float | None = None
    eps_abs_Li: float | None = None
    f_update_jacobi_Li: int | None = None
    PETSc_options: str = ''
    anderson_m: int = 8
    # spectral_polarization only (grid_mech_spectral_polarization.f90:137-148)
    solver: str = 'spectral_basic'
    alpha: float = 1.0
    beta: float = 1.0
    eps_abs_curl: float = 1.0e-10
    eps_rel_curl: float = 5.0e-4

    @property
    def snes_type(self) -> int:
        """0 = Richardson (``-snes_type nrichardson``); 1 = Anderson-accelerated fixed point
        (the reference's default ``-snes_type ngmres``, and ``anderson``)."""
        toks = ('-snes_type ngmres ' + self.PETSc_options).split()
        kind = 'ngmres'
        for i, t in enumerate(toks[:-1]):
            if t == '-snes_type':
                kind = toks[i + 1]
        if kind == 'nrichardson':
            return 0
        if kind in ('ngmres', 'anderson'):
            return 1
        raise ValueError(f'unsupported -snes_type {kind}')

    @property
    def snes_max_it(self) -> int:
        """PETSc's ``-snes_max_it`` from PETSc_options (PETSc's default 50)."""
        toks = self.PETSc_options.split()
        n = 50
        for i, t in enumerate(toks[:-1]):
            if t == '-snes_max_it':
                n = int(toks[i + 1])
        return n

    @classmethod
    def from_dict(cls, d: dict | None) -> 'Numerics':
        d = d or {}
        grid = d.get('solver', {}).get('grid', {})
        mech = grid.get('mechanical', {})
        fft = grid.get('FFT', {})
        pm = d.get('phase', {}).get('mechanical', {})
        pl = pm.get('plastic', {})
        eig = pm.get('eigen', {})
        n = cls()
        for k_yaml, k in (('N_iter_min', 'N_iter_min'), ('N_iter_max', 'N_iter_max'),
                          ('eps_abs_div(P)', 'eps_abs_div'), ('eps_rel_div(P)', 'eps_rel_div'),
                          ('eps_abs_P', 'eps_abs_P'), ('eps_rel_P', 'eps_rel_P'), ('update_gamma', 'update_gamma')):
            if k_yaml in mech:
                setattr(n, k, mech[k_yaml])
        for k_yaml, k in (('alpha', 'alpha'), ('beta', 'beta'), ('eps_abs_curl(F)', 'eps_abs_curl'),
                          ('eps_rel_curl(F)', 'eps_rel_curl')):
            if k_yaml in mech:
                setattr(n, k, float(mech[k_yaml]))
        if 'PETSc_options' in mech:
            n.PETSc_options = str(mech['PETSc_options'])
        if 'anderson_m' in mech:
            n.anderson_m = int(mech['anderson_m'])
        if 'divergence_correction' in fft:
            n.divergence_correction = fft['divergence_correction']
        if 'derivative' in fft:
            n.derivative = fft['derivative']
        if 'memory_efficient' in fft:
            n.memory_efficient = bool(fft['memory_efficient'])
        if 'FFTW_plan_mode' in fft:
            n.FFTW_plan_mode = str(fft['FFTW_plan_mode'])
        if 'N_cutback_max' in grid:
            n.N_cutback_max = int(grid['N_cutback_max'])
        for k in ('r_cutback_min', 'r_cutback', 'r_increase', 'eps_rel_state', 'N_iter_state_max'):
            if k in pm:
                setattr(n, k, pm[k])
        for k in ('N_iter_Lp_max', 'r_linesearch_Lp', 'eps_rel_Lp', 'eps_abs_Lp', 'f_update_jacobi_Lp'):
            if k in pl:
                setattr(n, k, pl[k])
        for k in ('N_iter_Li_max', 'r_linesearch_Li', 'eps_rel_Li', 'eps_abs_Li', 'f_update_jacobi_Li'):
            if k in eig:
                setattr(n, k, eig[k])
        if pl.get('integrator_state', 'FPI') != 'FPI':
            raise ValueError('only the FPI state integrator is on this path')
        return n

    def validate(self) -> None:
        bad = []
        if self.eps_abs_div <= 0: bad.append('eps_abs_div(P)')
        if self.eps_rel_div <= 0: bad.append('eps_rel_div(P)')
        if self.eps_abs_P <= 0: bad.append('eps_abs_P')
        if self.eps_rel_P <= 0: bad.append('eps_rel_P')
        if self.N_iter_max < 1: bad.append('N_iter_max')
        if self.N_iter_min > self.N_iter_max or self.N_iter_min < 1: bad.append('N_iter_min')
        if self.N_iter_Lp_max < 1: bad.append('N_iter_Lp_max')
        if self.N_iter_state_max < 1: bad.append('N_iter_state_max')
        if self.derivative not in DERIVATIVES: bad.append('derivative')
        if self.divergence_correction not in ('none', 'size', 'grid+size', 'size+grid'):
            bad.append('divergence_correction')
        if self.FFTW_plan_mode not in ('FFTW_ESTIMATE', 'FFTW_MEASURE', 'FFTW_PATIENT', 'FFTW_EXHAUSTIVE'):
            bad.append('FFTW_plan_mode')
        if not 1 <= self.anderson_m <= 32: bad.append('anderson_m')
        if self.solver not in SOLVERS: bad.append('solver')
        if self.solver == 'spectral_polarization':
            if self.eps_abs_curl <= 0: bad.append('eps_abs_curl(F)')
            if self.eps_rel_curl <= 0: bad.append('eps_rel_curl(F)')
            if not 0.0 < self.alpha <= 2.0: bad.append('alpha')
            if not 0.0 <= self.beta <= 2.0: bad.append('beta')
        self.snes_type
        if bad:
            raise ValueError('invalid numerics: ' + ' '.join(bad))

    def to_struct(self) -> NumericsStruct:
        self.validate()
        s = NumericsStruct()
        s.N_iter_min, s.N_iter_max = int(self.N_iter_min), int(self.N_iter_max)
        s.eps_abs_div, s.eps_rel_div = self.eps_abs_div, self.eps_rel_div
        s.eps_abs_P, s.eps_rel_P = self.eps_abs_P, self.eps_rel_P
        s.update_gamma = int(bool(self.update_gamma))
        s.divergence_correction = {'none': 0, 'size': 1, 'grid+size': 2, 'size+grid': 2}[self.divergence_correction]
        s.derivative = DERIVATIVES[self.derivative]
        s.r_cutback_min, s.r_cutback, s.r_increase = self.r_cutback_min, self.r_cutback, self.r_increase
        s.eps_rel_state, s.N_iter_state_max = self.eps_rel_state, int(self.N_iter_state_max)
        s.N_iter_Lp_max, s.r_linesearch_Lp = int(self.N_iter_Lp_max), self.r_linesearch_Lp
        s.eps_rel_Lp, s.eps_abs_Lp, s.f_update_jacobi_Lp = self.eps_rel_Lp, self.eps_abs_Lp, int(self.f_update_jacobi_Lp)
        s.N_iter_Li_max, s.r_linesearch_Li = int(self.N_iter_Li_max), self.r_linesearch_Li
        s.eps_rel_Li = self.eps_rel_Lp if self.eps_rel_Li is None else self.eps_rel_Li
        s.eps_abs_Li = self.eps_abs_Lp if self.eps_abs_Li is None else self.eps_abs_Li
        s.f_update_jacobi_Li = int(self.f_update_jacobi_Lp if self.f_update_jacobi_Li is None else self.f_update_jacobi_Li)
        s.snes_type = self.snes_type
        s.snes_max_it = self.snes_max_it
        s.anderson_m = int(self.anderson_m)
        s.solver = SOLVERS[self.solver]
        s.alpha, s.beta = float(self.alpha), float(self.beta)
        s.eps_abs_curl, s.eps_rel_curl = float(self.eps_abs_curl), float(self.eps_rel_curl)
        return s


def mechanical_solver(load: dict) -> str:
    """The grid mechanical solver a load file selects (``solver: mechanical:``,
    DAMASK_grid.f90:171-206); this path provides spectral_basic and spectral_polarization."""
    name = load.get('solver', {}).get('mechanical', 'spectral_basic')
    if name not in SOLVERS:
        raise ValueError(f"unsupported mechanical solver '{name}'")
    return name


def masked_tensor(rows) -> tuple[np.ndarray, np.ndarray]:
    """3x3 values and mask (True where 'x') from a nested YAML list (DAMASK_grid.f90:692-718)."""
    vals = np.zeros((3, 3))
    mask = np.zeros((3, 3), bool)
    for i in range(3):
        for j in range(3):
            v = rows[i][j]
            if isinstance(v, str) and v.strip() == 'x':
                mask[i, j] = True
            else:
                vals[i, j] = float(v)
    return vals, mask


def bc_struct(kind: str | None, values: np.ndarray | None, mask: np.ndarray | None) -> BCStruct:
    s = BCStruct()
    s.type = BC_TYPES.get(kind, 0) if kind else 0
    if values is None:
        values = np.zeros((3, 3))
        mask = np.ones((3, 3), bool)
    for j in range(3):
        for i in range(3):
            s.values[3 * j + i] = float(values[i, j])
            s.mask[3 * j + i] = int(bool(mask[i, j]))
    return s


def axis_angle_to_quaternion(ax) -> np.ndarray:
    """tRotation%fromAxisAngle(ax, degrees=.true.) with P = -1 (rotations.f90:192-213, :670-686)."""
    ax = np.asarray(ax, float)
    angle = np.radians(ax[3])
    if abs(np.linalg.norm(ax[:3]) - 1.0) > 2.220446049250313e-16 * 2 or angle < 0 or angle > np.pi:
        raise ValueError('invalid load-case rotation R')
    if abs(angle) <= np.finfo(float).tiny * 10:
        return np.array([1.0, 0.0, 0.0, 0.0])
    c, s = np.cos(angle * 0.5), np.sin(angle * 0.5)
    return np.array([c, ax[0] * s, ax[1] * s, ax[2] * s])


@dataclass
class LoadCase:
    deformation_type: str
    deformation: np.ndarray
    deformation_mask: np.ndarray
    stress_type: str | None
    stress: np.ndarray
    stress_mask: np.ndarray
    t: float
    N: int
    r: float = 1.0
    f_out: int = 1
    f_restart: int = 2 ** 31 - 1
    estimate_rate: bool = True
    q_rot: np.ndarray = field(default_factory=lambda: np.array([1.0, 0.0, 0.0, 0.0]))

    def deformation_bc(self) -> BCStruct:
        return bc_struct(self.deformation_type, self.deformation, self.deformation_mask)

    def stress_bc(self) -> BCStruct:
        return bc_struct(self.stress_type, self.stress, self.stress_mask)


def parse_load(load: dict) -> list[LoadCase]:
    cases = []
    for step in load['loadstep']:
        bc = step.get('boundary_condition', step.get('boundary_conditions'))
        mech = bc['mechanical']
        dtype = dvals = dmask = None
        stype, svals, smask = None, np.zeros((3, 3)), np.ones((3, 3), bool)
        q = np.array([1.0, 0.0, 0.0, 0.0])
        for key, val in mech.items():
            if key in ('L', 'dot_F', 'F_dot', 'F'):
                if dtype is not None:
                    raise ValueError('only one of L, dot_F, or F allowed in mechanical BC')
                dtype = 'dot_F' if key == 'F_dot' else key
                dvals, dmask = masked_tensor(val)
            elif key in ('P', 'dot_P', 'P_dot'):
                if stype is not None:
                    raise ValueError('only one of P or dot_P allowed in mechanical BC')
                stype = 'dot_P' if key == 'P_dot' else key
                svals, smask = masked_tensor(val)
            elif key == 'R':
                q = axis_angle_to_quaternion(val)
        if dtype is None:
            raise ValueError('load case is incomplete: L, F_dot/dot_F, or F missing')
        disc = step['discretization']
        f_out = step.get('f_out', 1)
        cases.append(LoadCase(dtype, dvals, dmask, stype, svals, smask,
                              t=float(disc['t']), N=int(disc['N']), r=float(disc.get('r', 1.0)),
                              f_out=2 ** 31 - 1 if f_out == 'none' else int(f_out),
                              f_restart=int(step.get('f_restart', 2 ** 31 - 1)),
                              estimate_rate=bool(step.get('estimate_rate', True)), q_rot=q))
    return cases


def geometric_fraction(r: float, i: int, N: int) -> float:
    """math_geometricFraction, math.f90:1222-1234."""
    if abs(r - 1.0) <= 1.0e-9:
        return 1.0 / N
    return (1.0 - r) * r ** i / (r - r ** (N + 1))
