"""Gradients of a stress-strain misfit with respect to the phenopowerlaw parameters, through the
hand-written adjoint of the grid solver's increments, behind a ``torch.autograd.Function``.

Forward (:meth:`IncrementSequence.run`): the increments of a load case on one CUDA context of
the basic spectral scheme (FP64), with a device checkpoint of the complete state every ``k``
increments (``dmk_checkpoint_save``); the volume-averaged stress <P> of every increment is the
output.

Backward (:meth:`IncrementSequence.gradient`): for each block of ``k`` increments, last block
first, the block is recomputed from its checkpoint and the linearization point of every
increment is recorded on the device (``dmk_adj_record``); then the block's increments are
reversed (``dmk_adj_step``): per increment, the local implicit-function adjoint of the
constitutive update (the converged Lp Newton and state fixed point of
``phase_mechanical.f90:379-676``, with the sensitivities of the phenopowerlaw kinetics and
hardening, ``phase_mechanical_plastic_phenopowerlaw.f90:303-399,449-488``) and the transposed
equilibrium problem solved with the solver's Gamma operator (``spectral_utilities.f90:436-501``).
The state cotangent stays on the device from increment to increment; xi_0 receives the
cotangent of the initial state (``dmk_adj_finish``).

The derivative is that of the exactly converged equations: compare it with finite differences
of forward runs whose tolerances are tight enough (:func:`gradient_numerics`).
"""
from __future__ import annotations

import copy

import numpy as np
import torch

from .config import Numerics, Phase
from .grid import IncrementDriver, SpectralBasic

THETA = ('xi_0', 'xi_inf', 'h_0', 'n', 'a')
_PHASE_KEYS = {'xi_0': 'xi_0_sl', 'xi_inf': 'xi_inf_sl', 'h_0': 'h_0_sl_sl', 'n': 'n_sl', 'a': 'a_sl'}
MAX_FAMILIES = 4


def phase_with(phase: Phase, theta) -> Phase:
    """A copy of `phase` with the parameters (xi_0, xi_inf, h_0, n, a) of theta: shape (5,) for the
    same values in every slip family, or (5, n_families)."""
    th = np.asarray(theta, dtype=float)
    nf = len(phase.N_sl)
    if th.ndim == 1:
        th = np.repeat(th[:, None], nf, axis=1)
    if th.shape != (5, nf):
        raise ValueError(f'theta must have shape (5,) or (5, {nf})')
    p = copy.deepcopy(phase)
    for i, name in enumerate(THETA):
        setattr(p, _PHASE_KEYS[name], [float(x) for x in th[i]])
    return p


def theta_of(phase: Phase) -> np.ndarray:
    """(5, n_families) parameters of a phase."""
    return np.array([getattr(phase, _PHASE_KEYS[name]) for name in THETA], dtype=float)


def gradient_numerics(num: Numerics | None = None) -> Numerics:
    """Numerics whose converged values obey the equations the adjoint differentiates to ~1e-11
    relative, so that central differences of forward runs at a relative step of 1e-6 resolve
    derivatives to ~1e-5: divergence and stress-BC tolerances 1e-11 relative (absolute floors
    below them), Lp Newton 1e-11 relative with no absolute floor (the Newton residual's rounding
    floor lies near 1e-12), state iteration 1e-12 relative (more state iterations allowed),
    Anderson history 30 and up to 300 fixed-point iterations (-snes_max_it 300, N_iter_max 300)."""
    n = copy.deepcopy(num) if num is not None else Numerics()
    n.eps_rel_div, n.eps_abs_div = 1.0e-11, 1.0e-12
    n.eps_rel_P, n.eps_abs_P = 1.0e-11, 1.0e-6
    n.eps_rel_Lp, n.eps_abs_Lp = 1.0e-11, 1.0e-30
    n.eps_rel_state, n.N_iter_state_max = 1.0e-12, 100
    n.anderson_m = 30
    n.PETSc_options = (n.PETSc_options + ' -snes_max_it 300').strip()
    n.N_iter_max = 300
    return n


def gradient_phase(phase: Phase) -> Phase:
    """The phase with absolute state tolerances below the relative ones of gradient_numerics."""
    p = copy.deepcopy(phase)
    p.atol_xi, p.atol_gamma = 1.0e-9, 1.0e-18
    return p


class IncrementSequence:
    """The first `n_increments` increments of a load case with device checkpoints every `k`,
    and their adjoint.  One CUDA context per forward run (kept for the backward pass)."""

    def __init__(self, rve, phase: Phase, loadcases, numerics: Numerics, n_increments: int, k: int = 10,
                 device: int = 0):
        self.rve, self.phase, self.loadcases, self.numerics = rve, phase, loadcases, numerics
        self.n, self.k, self.device = int(n_increments), int(k), device
        self.solver = None
        self.krylov_iterations: list[int] = []

    def close(self) -> None:
        if self.solver is not None:
            self.solver.close()
            self.solver = None

    def _step(self, i: int):
        recs = self.drv.step()
        if len(recs) != 1 or recs[0].cutback_level != 0:
            raise RuntimeError(f'increment {i + 1} was cut back; the adjoint covers increments without cutback')
        return recs[0]

    def run(self, theta) -> np.ndarray:
        """<P> (n, 3, 3) of the increments at the parameters theta."""
        self.close()
        ph = phase_with(self.phase, theta)
        self.theta = np.asarray(theta, dtype=float)
        self.solver = SpectralBasic(self.rve.cells, self.rve.size, self.rve.material, self.rve.quaternions, ph,
                                    self.numerics, precision='fp64', device=self.device)
        self.drv = IncrementDriver(self.solver, self.loadcases)
        self.snapshots = []
        self.P_av = np.zeros((self.n, 3, 3))
        for i in range(self.n):
            if i % self.k == 0:
                self.solver.checkpoint_save(i // self.k)
                self.snapshots.append(self.drv.state())
            self.P_av[i] = self._step(i).P_av
        return self.P_av.copy()

    def gradient(self, dL_dPav) -> np.ndarray:
        """dL/dtheta (5, n_families) for dL/d<P> (n, 3, 3) of the last run."""
        g = np.asarray(dL_dPav, dtype=float).reshape(self.n, 3, 3)
        s = self.solver
        s.adj_begin(self.k)
        tb = np.zeros(5 * MAX_FAMILIES)
        self.krylov_iterations = []
        self.recompute_deviation = 0.0
        for b in reversed(range(len(self.snapshots))):
            s.checkpoint_restore(b)
            self.drv.set_state(self.snapshots[b])
            n0, n1 = b * self.k, min(self.n, (b + 1) * self.k)
            for i in range(n0, n1):
                P = self._step(i).P_av
                self.recompute_deviation = max(self.recompute_deviation,
                                               float(np.abs(P - self.P_av[i]).max() / np.abs(self.P_av[i]).max()))
                s.adj_record(i - n0)
            for i in reversed(range(n0, n1)):
                self.krylov_iterations.append(s.adj_step(i - n0, g[i], tb))
        s.adj_finish(tb)
        return tb.reshape(5, MAX_FAMILIES)[:, :len(self.phase.N_sl)].copy()


class StressCurve(torch.autograd.Function):
    """<P>(theta) of an IncrementSequence as a differentiable function of the parameters theta
    ((5,) or (5, n_families), float64): forward runs the increments, backward the adjoint."""

    @staticmethod
    def forward(ctx, theta: torch.Tensor, seq: IncrementSequence) -> torch.Tensor:
        P = seq.run(theta.detach().cpu().numpy())
        ctx.seq = seq
        ctx.shape = tuple(theta.shape)
        ctx.dtype = theta.dtype
        return torch.from_numpy(P)

    @staticmethod
    def backward(ctx, grad: torch.Tensor):
        g = ctx.seq.gradient(grad.detach().cpu().numpy())
        if len(ctx.shape) == 1:
            g = g.sum(axis=1)
        return torch.from_numpy(g).to(ctx.dtype), None


def stress_curve(theta: torch.Tensor, seq: IncrementSequence) -> torch.Tensor:
    """Differentiable <P> (n, 3, 3) of the increments of `seq` at theta."""
    return StressCurve.apply(theta, seq)
