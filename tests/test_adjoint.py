"""The hand-written adjoint of increments (dmk_adj_*, damask_b200.adjoint).

CPU: the local implicit-function Jacobian D = d(P, Fp, xi)/d(F, Fp0, xi0, theta) of one voxel
(host build of the same code as the device kernel) against central differences of the oracle's
constitutive update of that voxel, an independent restatement of integrateStress and
integrateStateFPI (phase_mechanical.f90:379-676).

GPU: device checkpoints restore bit for bit; the gradient of a stress-strain misfit with respect
to (xi_0, xi_inf, h_0, n, a) from the adjoint against central differences (relative step 1e-6) of
the FP64 forward on the GPU and of the oracle's forward, within 1e-4 relative per parameter; the
autograd path; and configuration 3 (32^3, 50 grains, 50 increments, checkpoints every 10).
"""
import copy

import numpy as np
import pytest

from damask_b200 import synthetic, workloads
from damask_b200.adjoint import (THETA, IncrementSequence, gradient_numerics, gradient_phase, phase_with,
                                 stress_curve, theta_of)

STEP = 1.0e-6          # relative step of the central differences
TOL = 1.0e-4           # relative agreement of adjoint and central differences, per parameter


# ----------------------------------------------------------------------------------- CPU
def _local_point(oracle_lib, phase, F, q, num):
    """One-voxel oracle: the increment-start state (Fp0 = orientation, xi0 = xi_0), its
    constitutive response at F over dt = 1 and the converged Lp, xi."""
    o = oracle_lib.OracleSpectralBasic((1, 1, 1), workloads.SIZE_1MM, np.zeros(1), q[None, :], phase, num, threads=1)
    Fp0 = o.get_field('F_p')[0]
    P, _, _, _, st = o.constitutive_response(F.reshape(1, 9), 1.0)
    assert st == 0
    assert o.counters()[1] == 1         # one substep: the increment is the local model's implicit function
    out = (P[0], o.get_field('F_p')[0], o.get_field('xi_sl')[0], o.get_field('L_p')[0])
    o.close()
    return Fp0, out


def _z(out):
    P, Fp, xi, _ = out
    return np.concatenate([P, Fp, xi])


@pytest.mark.parametrize('which', ['fcc12', 'bcc24'])
def test_local_jacobian_against_oracle_differences(oracle_lib, which):
    import ctypes as C
    from damask_b200 import _lib
    base = workloads.fcc_al() if which == 'fcc12' else workloads.bcc_24()
    phase = gradient_phase(base)
    num = gradient_numerics(workloads.numerics_default())
    q = np.array([0.8, 0.2, -0.4, 0.4])
    q /= np.linalg.norm(q)
    # plastic (|Lp| ~ 1e-3/s) and one substep for every perturbed input: the bcc-24 Lp Newton from
    # Lp = 0 needs substeps beyond ~0.3 % strain in one step of 1 s, with a result ~1 % apart
    E = np.array([[4.0e-3, 1.0e-3, 0.0], [0.5e-3, -1.5e-3, 0.0], [0.0, 0.2e-3, -1.8e-3]])
    F = (np.eye(3) + (1.0 if which == 'fcc12' else 0.5) * E).reshape(-1, order='F')
    Fp0, out = _local_point(oracle_lib, phase, F, q, num)
    ns, nf = phase.n_slip, len(phase.N_sl)
    xi0 = np.concatenate([[x] * n for x, n in zip(phase.xi_0_sl, phase.N_sl)])
    point = np.concatenate([F, Fp0, xi0, out[3], out[2]])
    nz, nx = 18 + ns, 18 + ns + 4 * nf
    D = np.zeros(nz * nx)
    lib = _lib.load()
    ps = phase.to_struct()
    dp = C.POINTER(C.c_double)
    _lib.check(lib.dmk_adj_local_jacobian(C.byref(ps), 1.0, point.ctypes.data_as(dp), D.ctypes.data_as(dp)))
    D = D.reshape(nz, nx)
    z0 = _z(out)
    assert np.abs(out[3]).max() > 1e-5                        # plastic: the kinetics contribute
    scale = np.maximum(np.abs(z0), 1e-3 * np.abs(z0).max())  # per output row

    # agreement within 1e-5 of the column's largest entry plus the differences' own noise: the
    # converged outputs carry ~1e-12 relative noise from the tolerances, which a central difference
    # of step h turns into 1e-11 / (2 h) (with a factor 10 of margin) in these row-scaled units
    def check(col_fd, col_ad, what, h):
        err = np.abs(col_fd - col_ad) / scale
        ref = np.abs(col_fd) / scale
        assert err.max() <= 1e-5 * ref.max() + 1e-11 / (2 * h), (what, err.max(), ref.max())

    # F columns
    for k in range(9):
        h = 1.0e-7
        zp = _z(_local_point(oracle_lib, phase, F + h * np.eye(9)[k], q, num)[1])
        zm = _z(_local_point(oracle_lib, phase, F - h * np.eye(9)[k], q, num)[1])
        check((zp - zm) / (2 * h), D[:, k], f'F[{k}]', h)
    # theta columns (xi_inf, h_0, n, a of each family) and xi_0 (the sum over its systems' xi0 columns)
    th = theta_of(phase)
    for p, name in enumerate(THETA):
        for f in range(nf):
            d = STEP * th[p, f]
            tp, tm = th.copy(), th.copy()
            tp[p, f] += d
            tm[p, f] -= d
            zp = _z(_local_point(oracle_lib, phase_with(phase, tp), F, q, num)[1])
            zm = _z(_local_point(oracle_lib, phase_with(phase, tm), F, q, num)[1])
            fd = (zp - zm) / (2 * d)
            if name == 'xi_0':
                lo = sum(phase.N_sl[:f])
                ad = D[:, 18 + lo:18 + lo + phase.N_sl[f]].sum(axis=1)
            else:
                ad = D[:, 18 + ns + (p - 1) * nf + f]
            check(fd, ad, f'{name}[{f}]', d)


# ----------------------------------------------------------------------------------- GPU
def _misfit(P, target):
    """Sum over increments of ((<P_xx> - target) / 1 MPa)^2 and its derivative with respect to <P>."""
    r = (P[:, 0, 0] - target) / 1.0e6
    g = np.zeros_like(P)
    g[:, 0, 0] = 2.0 * r / 1.0e6
    return float((r * r).sum()), g


def _central_differences(run, theta, target):
    out = np.zeros_like(theta)
    for idx in np.ndindex(theta.shape):
        d = STEP * theta[idx]
        tp, tm = theta.copy(), theta.copy()
        tp[idx] += d
        tm[idx] -= d
        out[idx] = (_misfit(run(tp), target)[0] - _misfit(run(tm), target)[0]) / (2 * d)
    return out


def _problem(cells, grains, seed, n, base=None):
    rve = synthetic.voronoi_rve(cells, workloads.SIZE_1MM, grains, seed)
    phase = gradient_phase(base or workloads.fcc_al())
    num = gradient_numerics(workloads.numerics_default())
    return rve, phase, workloads.tension_x(float(n), n), num


THETA_STAR = np.array([40.0e6, 80.0e6, 100.0e6, 20.0, 2.0])   # the target curve's parameters
THETA_0 = np.array([31.0e6, 63.0e6, 75.0e6, 20.0, 2.25])       # where the gradient is taken


@pytest.mark.gpu
def test_checkpoint_restore_is_bit_exact(gpu):
    from damask_b200.grid import IncrementDriver, SpectralBasic
    rve, phase, lcs, num = _problem((8, 8, 8), 6, 0, 10)
    s = SpectralBasic(rve.cells, rve.size, rve.material, rve.quaternions, phase, num)
    drv = IncrementDriver(s, lcs)
    for _ in range(3):
        drv.step()
    s.checkpoint_save(0)
    st = drv.state()
    ref = [drv.step()[0].P_av for _ in range(3)]
    fields = {k: s.get_field(k) for k in ('P', 'F', 'F_p', 'L_p', 'xi_sl', 'gamma_sl')}
    s.checkpoint_restore(0)
    drv.set_state(st)
    again = [drv.step()[0].P_av for _ in range(3)]
    for a, b in zip(ref, again):
        assert np.array_equal(a, b)
    for k, v in fields.items():
        assert np.array_equal(s.get_field(k), v), k
    s.close()


@pytest.mark.gpu
@pytest.mark.parametrize('case', ['fcc8', 'bcc8'])
def test_adjoint_against_gpu_central_differences(gpu, case):
    """Two blocks of three increments (k = 3) on an 8^3 RVE: the recomputation from checkpoints and
    the state cotangent across blocks are exercised."""
    base = workloads.fcc_al() if case == 'fcc8' else workloads.bcc_24()
    rve, phase, lcs, num = _problem((8, 8, 8), 6, 1, 6, base)
    theta0 = theta_of(phase)
    tstar = theta0 * np.array([1.25, 1.2, 1.3, 1.0, 0.9])[:, None]
    seq = IncrementSequence(rve, phase, lcs, num, 6, k=3)
    target = seq.run(tstar)[:, 0, 0]
    L, g = _misfit(seq.run(theta0), target)
    grad = seq.gradient(g)
    assert seq.recompute_deviation == 0.0
    fd = _central_differences(seq.run, theta0, target)
    seq.close()
    rel = np.abs(grad - fd) / np.abs(fd)
    print(f'{case}: adjoint {grad.ravel()} central differences {fd.ravel()} rel {rel.ravel()}; '
          f'Krylov iterations {seq.krylov_iterations}')
    assert rel.max() < TOL


@pytest.mark.gpu
def test_adjoint_against_oracle_central_differences(gpu, oracle_lib):
    """The FP64 reference gradient: central differences of the oracle's forward (CPU restatement of
    the reference), against the GPU adjoint, on a 6^3 RVE over four increments."""
    from damask_b200.grid import run_load_cases
    rve, phase, lcs, num = _problem((6, 6, 6), 4, 5, 4)
    theta0 = THETA_0.copy()

    def oracle_run(theta):
        o = oracle_lib.OracleSpectralBasic(rve.cells, rve.size, rve.material, rve.quaternions,
                                           phase_with(phase, theta), num)
        st = run_load_cases(o, lcs, max_increments=4)
        o.close()
        return np.array([s.P_av for s in st])

    target = oracle_run(THETA_STAR)[:, 0, 0]
    seq = IncrementSequence(rve, phase, lcs, num, 4, k=2)
    P = seq.run(theta0)
    assert np.abs(P - oracle_run(theta0)).max() / np.abs(P).max() < 1e-9
    grad = seq.gradient(_misfit(P, target)[1])[:, 0]
    seq.close()
    fd = _central_differences(oracle_run, theta0, target)
    rel = np.abs(grad - fd) / np.abs(fd)
    print(f'adjoint {grad} oracle central differences {fd} rel {rel}')
    assert rel.max() < TOL


@pytest.mark.gpu
def test_autograd_function(gpu):
    import torch
    rve, phase, lcs, num = _problem((6, 6, 6), 4, 3, 3)
    seq = IncrementSequence(rve, phase, lcs, num, 3, k=2)
    target = torch.from_numpy(seq.run(THETA_STAR)[:, 0, 0])
    theta = torch.tensor(THETA_0, dtype=torch.float64, requires_grad=True)
    P = stress_curve(theta, seq)
    loss = (((P[:, 0, 0] - target) / 1.0e6) ** 2).sum()
    loss.backward()
    direct = seq.gradient(_misfit(P.detach().numpy(), target.numpy())[1])[:, 0]
    seq.close()
    assert np.allclose(theta.grad.numpy(), direct, rtol=1e-12, atol=0.0)


@pytest.mark.gpu
def test_configuration_3_adjoint_against_central_differences(gpu):
    """32^3, 50 Voronoi grains (seed 2), fcc, uniaxial tension to 5 % in 50 increments; target curve
    from the forward at (xi_0, xi_inf, h_0, n, a) = (40 MPa, 80 MPa, 100 MPa, 20, 2.0); gradient at
    (31 MPa, 63 MPa, 75 MPa, 20, 2.25); checkpoints every 10 increments; central differences at a
    relative step of 1e-6."""
    rve, phase, lcs, num = workloads.make('grid32_fcc_50g')
    phase = gradient_phase(phase)
    num = gradient_numerics(num)
    seq = IncrementSequence(rve, phase, lcs, num, 50, k=10)
    target = seq.run(THETA_STAR)[:, 0, 0]
    L, g = _misfit(seq.run(THETA_0), target)
    grad = seq.gradient(g)[:, 0]
    fd = _central_differences(lambda t: seq.run(t), THETA_0, target)
    seq.close()
    rel = np.abs(grad - fd) / np.abs(fd)
    print(f'configuration 3: loss {L:.6e}; adjoint {grad}; central differences {fd}; rel {rel}; '
          f'Krylov iterations per increment {seq.krylov_iterations}')
    assert rel.max() < TOL
