"""The oracle (CPU FP64 restatement) against the reference's golden vectors and the
invariants its own self-tests check (spectral_utilities.f90:974-1108, math.f90:1240-1410)."""
import numpy as np
import pytest

from damask_b200 import synthetic, workloads
from damask_b200.config import Numerics
from damask_b200.grid import run_load_cases

from conftest import rel


def small_oracle(oracle_lib, cells=(4, 4, 4), grains=3, seed=0, phase=None, num=None, size=workloads.SIZE_1MM,
                 init=True):
    rve = synthetic.voronoi_rve(cells, size, grains, seed)
    return oracle_lib.OracleSpectralBasic(rve.cells, rve.size, rve.material, rve.quaternions,
                                          phase or workloads.fcc_al(), num or workloads.numerics_default(),
                                          threads=2, init=init)


def test_seeds_and_rotations_match_reference(golden):
    rng = np.random.default_rng(0)
    s = synthetic.seeds_from_random([1.0e-3] * 3, 20, rng)
    q = synthetic.rotations_from_random(20, rng)
    assert np.array_equal(s, golden['seeds_0'])
    assert np.allclose(q, golden['quats_0'], rtol=0, atol=1e-15)


def test_fft_matches_numpy(oracle_lib):
    x = np.random.default_rng(1).normal(size=(6, 5, 8)) + 1j * np.random.default_rng(2).normal(size=(6, 5, 8))
    assert rel(oracle_lib.fft3(x, -1), np.fft.fftn(x)) < 1e-13
    assert rel(oracle_lib.fft3(x, +1), np.fft.ifftn(x) * x.size) < 1e-13


def test_divergence_rms_matches_reference_numpy(golden, oracle_lib):
    """utilities_divergenceRMS with divergence_correction 'size' is the RMS of the
    spectral divergence field computed by the reference's python/damask/grid.py."""
    f = golden['div_field']                        # [x, y, z, 3, 3]
    num = workloads.numerics_default()
    num.divergence_correction = 'size'
    o = small_oracle(oracle_lib, cells=f.shape[:3], size=tuple(golden['div_size']), num=num, init=False)
    P = f.transpose(2, 1, 0, 4, 3).reshape(-1, 9)   # voxel-major, x fastest; column-major tensor
    assert rel(o.divergence_rms(P), golden['div_rms']) < 1e-12


def numerics_with(derivative):
    n = workloads.numerics_default()
    n.derivative = derivative
    return n


@pytest.mark.parametrize('derivative', ['continuous', 'central_difference', 'FWBW_difference'])
def test_divergence_of_constant_field_vanishes(oracle_lib, derivative):
    o = small_oracle(oracle_lib, cells=(5, 4, 6), init=False, num=numerics_with(derivative))
    P = np.tile(np.random.default_rng(3).normal(size=9) * 1e8, (o.N, 1))
    assert o.divergence_rms(P) < 5e-14 * 1e8


@pytest.mark.parametrize('derivative', ['continuous', 'central_difference', 'FWBW_difference'])
def test_gamma_convolution_of_constant_field_is_aim(oracle_lib, derivative):
    o = small_oracle(oracle_lib, cells=(4, 6, 5), num=numerics_with(derivative))
    field = np.tile(np.random.default_rng(4).normal(size=9), (o.N, 1))
    aim = np.random.default_rng(5).normal(size=9)
    out = o.gamma_convolution(field, aim)
    assert np.abs(out - aim).max() < 1e-13


def test_gamma_is_projection_of_compatible_part(oracle_lib):
    """Gamma applied to C_ref : grad(u) returns grad(u) (Gamma^0 C^0 is the projector on
    compatible fields); the C2R of the unnormalised transform carries the 1/N of C_ref."""
    o = small_oracle(oracle_lib, cells=(8, 8, 8))
    C = o.aims()['C_minMaxAvg'].reshape(3, 3, 3, 3, order='F')
    n = 8
    x = (np.arange(n) + 0.5) / n * 1.0e-3
    X, Y, Z = np.meshgrid(x, x, x, indexing='ij')
    k = 2 * np.pi / 1.0e-3
    # displacement u = a sin(k x) + b cos(2 k y) with gradient H = du/dX
    H = np.zeros((n, n, n, 3, 3))
    a, b = np.array([1e-4, 2e-4, -1e-4]), np.array([-3e-5, 1e-4, 5e-5])
    H[..., :, 0] = a[None, None, None, :] * (k * np.cos(k * X))[..., None]
    H[..., :, 1] = b[None, None, None, :] * (-2 * k * np.sin(2 * k * Y))[..., None]
    tau = np.einsum('ijkl,xyzkl->xyzij', C, H)
    field = tau.transpose(2, 1, 0, 4, 3).reshape(-1, 9)
    out = o.gamma_convolution(field, np.zeros(9))
    expect = H.transpose(2, 1, 0, 4, 3).reshape(-1, 9)
    assert rel(out, expect) < 1e-12


def test_hooke_small_strain(oracle_lib):
    """At dt = 0 the response is elastic: P ~= C : eps for a small symmetric strain (cubic C)."""
    ph = workloads.fcc_al()
    o = small_oracle(oracle_lib, cells=(2, 2, 2), grains=1, phase=ph)
    eps = np.array([[1e-5, 2e-6, 0], [2e-6, -3e-6, 1e-6], [0, 1e-6, 4e-6]])
    F = np.tile((np.eye(3) + eps).reshape(-1, order='F'), (o.N, 1))
    P, P_av, Cv, Cm, st = o.constitutive_response(F, 0.0)
    assert st == 0
    C = Cv.reshape(3, 3, 3, 3, order='F')
    lin = np.einsum('ijkl,kl->ij', C, eps)
    assert rel(P_av.reshape(3, 3, order='F'), lin) < 2e-5     # geometric nonlinearity ~ |eps|


def _fd_tangent(o, F0, dt, h):
    fd = np.zeros((3, 3, 3, 3))
    for k in range(3):
        for l in range(3):
            Fp, Fm = F0.copy(), F0.copy()
            Fp[k, l] += h
            Fm[k, l] -= h
            Pp = o.constitutive_response(np.tile(Fp.reshape(-1, order='F'), (o.N, 1)), dt)[0][0].reshape(3, 3, order='F')
            Pm = o.constitutive_response(np.tile(Fm.reshape(-1, order='F'), (o.N, 1)), dt)[0][0].reshape(3, 3, order='F')
            fd[:, :, k, l] = (Pp - Pm) / (2 * h)
    return fd


@pytest.mark.parametrize('dt,F_pert,tol', [
    # elastic (dt = 0): the tangent is exact
    (0.0, [[1e-4, 1e-5, 0], [0, -3e-5, 2e-5], [1e-5, 0, -3e-5]], 1e-6),
    # plastic: phase_mechanical_dPdF holds the slip resistance fixed and the Lp Newton stops at
    # eps_rel_Lp = 1e-6, so central differences agree to about 1e-3
    (1.0, [[4e-3, 1e-4, 0], [0, -1.2e-3, 2e-4], [1e-4, 0, -1.3e-3]], 5e-3)])
def test_tangent_matches_finite_differences(oracle_lib, dt, F_pert, tol):
    o = small_oracle(oracle_lib, cells=(1, 1, 2), grains=1, phase=workloads.fcc_al())
    F0 = np.eye(3) + np.array(F_pert)
    P, *_, st = o.constitutive_response(np.tile(F0.reshape(-1, order='F'), (o.N, 1)), dt)
    assert st == 0
    D = o.dPdF(dt)[0].reshape(3, 3, 3, 3, order='F')
    fd = _fd_tangent(o, F0, dt, 1e-7 if dt == 0.0 else 1e-8)
    if dt > 0:
        assert np.abs(P[0]).max() > 5e7                      # plastic flow at this strain
    assert rel(D, fd) < tol


@pytest.mark.parametrize('snes', ['', '-snes_type nrichardson'])
def test_small_run_converges(oracle_lib, snes):
    num = workloads.numerics_default()
    num.PETSc_options = snes
    o = small_oracle(oracle_lib, cells=(6, 6, 6), grains=4, num=num)
    stats = run_load_cases(o, workloads.tension_x(60.0, 60), max_increments=4)
    assert len(stats) == 4 and all(s.converged for s in stats)
    Pxx = [s.P_av[0, 0] for s in stats]
    assert all(b > a for a, b in zip(Pxx, Pxx[1:]))          # hardening under tension
    assert abs(stats[-1].P_av[1, 1]) < 1e3 + 1e-3 * Pxx[-1]   # lateral stress BC held


def test_state_loop_bound_is_honoured(oracle_lib):
    """N_iter_Lp_max = 1 makes integrateStress fail (STATUS_..._LP_MAXIT) in the plastic range;
    the substep cutback then fails below r_cutback_min and the solution reports no convergence."""
    num = workloads.numerics_default()
    num.N_iter_Lp_max = 1
    o = small_oracle(oracle_lib, cells=(2, 2, 2), grains=2, num=num)
    F = np.tile((np.eye(3) + np.diag([5e-3, -2e-3, -2e-3])).reshape(-1, order='F'), (o.N, 1))
    *_, st = o.constitutive_response(F, 1.0)
    assert st != 0


def test_orientation_output(oracle_lib):
    """crystallite_orientations: O is the rotational part of Fe.  At init Fe is the
    inverse lattice orientation, so O returns the input quaternions; a right stretch
    Fe U (U symmetric positive definite) leaves it unchanged."""
    rve = synthetic.voronoi_rve((3, 3, 2), workloads.SIZE_1MM, 4, 5)
    o = oracle_lib.OracleSpectralBasic(rve.cells, rve.size, rve.material, rve.quaternions, workloads.fcc_al(),
                                       workloads.numerics_default(), threads=2)
    q = rve.quaternions[rve.material]
    q = q * np.sign(q[:, :1])
    assert np.abs(o.get_field('O') - q).max() < 1e-13
    Fe = o.get_field('F_e').reshape(-1, 3, 3, order='C')           # per voxel: column-major 3x3
    U = np.array([[1.02, 0.003, -0.001], [0.003, 0.99, 0.002], [-0.001, 0.002, 1.005]])
    Fe_m = np.transpose(Fe, (0, 2, 1))                              # as matrices
    Fs = np.transpose(Fe_m @ U, (0, 2, 1)).reshape(-1, 9)
    o.set_field('F_e', Fs)
    assert np.abs(o.get_field('O') - q).max() < 1e-12
    o.close()


def voxel_tensors(F: np.ndarray) -> np.ndarray:
    """(x, y, z, 3, 3) -> (N, 9): column-major 3x3 per voxel, x fastest."""
    return np.transpose(F, (0, 1, 2, 4, 3)).reshape(F.shape[:3] + (9,)).reshape(-1, 9, order='F')


@pytest.mark.parametrize('case', ['odd', 'smooth'])
def test_update_coords_matches_reference_python(golden, oracle_lib, case):
    """utilities_updateCoords against the reference's Python form (coordinates_point/_node)."""
    F = golden[f'coords_{case}_F']
    cells = F.shape[:3]
    o = oracle_lib.OracleSpectralBasic(cells, tuple(golden[f'coords_{case}_size']), np.zeros(int(np.prod(cells))),
                                       np.array([[1.0, 0, 0, 0]]), workloads.fcc_al(), init=False, threads=1)
    o.set_field('F_solver', voxel_tensors(F))
    o.update_coords()
    ip, nodes = o.get_coords()
    o.close()
    assert rel(ip, golden[f'coords_{case}_ip'].reshape(-1, 3, order='F')) < 1e-13
    assert rel(nodes, golden[f'coords_{case}_nodes'].reshape(-1, 3, order='F')) < 1e-13


def test_coordinates_start_undeformed_and_follow_uniform_F(oracle_lib):
    """Before any update the coordinates are IPcoordinates0 / nodes0; a uniform F maps them
    affinely (no fluctuation) and the displacements are (F - I) x0."""
    from damask_b200.grid import coordinates0, displacements
    cells, size = (4, 3, 2), (1.0e-3, 2.0e-3, 3.0e-3)
    o = oracle_lib.OracleSpectralBasic(cells, size, np.zeros(24), np.array([[1.0, 0, 0, 0]]), workloads.fcc_al(),
                                       init=False, threads=1)
    ip0, n0 = coordinates0(cells, size)
    ip, nodes = o.get_coords()
    assert np.array_equal(ip, ip0) and np.array_equal(nodes, n0)
    Fu = np.array([[1.1, 0.02, 0.0], [0.0, 0.95, 0.01], [0.03, 0.0, 1.0]])
    o.set_field('F_solver', np.tile(Fu.T.reshape(-1), (24, 1)))
    o.update_coords()
    ip, nodes = o.get_coords()
    o.close()
    up, un = displacements(cells, size, ip, nodes)
    assert rel(up, ip0 @ (Fu - np.eye(3)).T) < 1e-12
    assert rel(un, n0 @ (Fu - np.eye(3)).T) < 1e-12


def test_central_difference_divergence_matches_finite_differences(oracle_lib):
    """With derivative: central_difference the reference's frequencies are
    i sin(2 pi k / n) / (2 L / n) (spectral_utilities.f90:808-850), half the symbol of the usual
    central difference, so the spectral divergence is sum_j (P(x + h_j) - P(x - h_j)) / (4 h_j);
    with divergence_correction 'size' no rescaling applies (:181-197), and the RMS follows
    Parseval (:650-691)."""
    cells, size = (6, 5, 7), (1.0e-3, 0.8e-3, 1.4e-3)
    num = numerics_with('central_difference')
    num.divergence_correction = 'size'
    o = oracle_lib.OracleSpectralBasic(cells, size, np.zeros(int(np.prod(cells))), np.array([[1.0, 0, 0, 0]]),
                                       workloads.fcc_al(), num, init=False, threads=1)
    P = np.random.default_rng(9).normal(size=cells + (3, 3))
    h = np.asarray(size) / np.asarray(cells)
    div = sum((np.roll(P[..., :, j], -1, axis=j) - np.roll(P[..., :, j], 1, axis=j)) / (4 * h[j]) for j in range(3))
    voxels = np.transpose(P, (0, 1, 2, 4, 3)).reshape(cells + (9,)).reshape(-1, 9, order='F')
    rms = np.sqrt(np.mean(np.sum(div ** 2, axis=-1)))
    assert abs(o.divergence_rms(voxels) - rms) < 1e-12 * rms
    o.close()


@pytest.mark.parametrize('cells', [(6, 5, 7), (4, 6, 8)])
def test_fwbw_divergence_matches_staggered_differences(oracle_lib, cells):
    """With derivative: FWBW_difference the frequencies are (e^{i t_d} - 1) prod_{e != d} (e^{i t_e} + 1)
    / (4 L_d / n_d) (spectral_utilities.f90:823-849).  conj(-xi) multiplies the spectrum by the
    backward difference along d and the sum of the two neighbours along the other directions,
    so the divergence is the edge-averaged difference sum_j B_j A_e A_f P(:, j) / (4 h_j) on the
    staggered grid (B x = x(n - 1) - x(n), A x = x(n - 1) + x(n)), and its RMS follows Parseval."""
    size = (1.0e-3, 0.8e-3, 1.4e-3)
    num = numerics_with('FWBW_difference')
    num.divergence_correction = 'size'
    o = oracle_lib.OracleSpectralBasic(cells, size, np.zeros(int(np.prod(cells))), np.array([[1.0, 0, 0, 0]]),
                                       workloads.fcc_al(), num, init=False, threads=1)
    P = np.random.default_rng(11).normal(size=cells + (3, 3))
    h = np.asarray(size) / np.asarray(cells)

    def back(x, ax):
        return np.roll(x, 1, axis=ax) - x

    def both(x, ax):
        return np.roll(x, 1, axis=ax) + x

    div = 0.0
    for j in range(3):
        d = back(P[..., :, j], j)
        for e in range(3):
            if e != j:
                d = both(d, e)
        div = div + d / (4 * h[j])
    voxels = np.transpose(P, (0, 1, 2, 4, 3)).reshape(cells + (9,)).reshape(-1, 9, order='F')
    rms = np.sqrt(np.mean(np.sum(div ** 2, axis=-1)))
    assert abs(o.divergence_rms(voxels) - rms) < 1e-12 * rms
    o.close()


@pytest.mark.parametrize('derivative', ['continuous', 'central_difference', 'FWBW_difference'])
@pytest.mark.parametrize('cells', [(5, 6, 7), (6, 4, 8)])
def test_gamma_c_gamma_is_gamma(oracle_lib, derivative, cells):
    """Gamma_hat C_ref Gamma_hat = Gamma_hat point by point for any wave vector (the acoustic
    tensor K = C_ref : conj(xi) (x) xi cancels against its inverse), so convolving C : Gamma(tau)
    again reproduces Gamma(tau); with the complex FWBW frequencies this exercises the complex
    inverse of spectral_utilities.f90:356-395."""
    o = small_oracle(oracle_lib, cells=cells, num=numerics_with(derivative))
    C = o.aims()['C_minMaxAvg'].reshape(3, 3, 3, 3, order='F')
    tau = np.random.default_rng(12).normal(size=(o.N, 9)) * 1e8
    g1 = o.gamma_convolution(tau, np.zeros(9))
    H = g1.reshape(-1, 3, 3).transpose(0, 2, 1)                   # [v, i, j]
    tau2 = np.einsum('ijkl,vkl->vij', C, H).transpose(0, 2, 1).reshape(-1, 9)
    g2 = o.gamma_convolution(tau2, np.zeros(9))
    assert rel(g2, g1) < 1e-11
    o.close()


def test_update_coords_inverts_gradients_of_purely_imaginary_frequencies(oracle_lib):
    """utilities_updateCoords (spectral_utilities.f90:899-909) forms u_hat = F_hat xi / sum(conj(-xi) xi).
    For a gradient F_hat = u_hat (x) xi that is u_hat sum(xi^2) / (-|xi|^2): u itself when xi is purely
    imaginary (continuous, central difference), but not for the complex FWBW frequencies.  The
    restatement keeps the reference's formula for all three (odd grid, so no Nyquist terms)."""
    from damask_b200.grid import displacements
    cells, size = (5, 7, 3), (1.0e-3, 2.0e-3, 1.5e-3)
    rng = np.random.default_rng(6)
    u = rng.normal(size=cells + (3,)) * 1e-6
    u -= u.mean(axis=(0, 1, 2))
    h = np.asarray(size) / np.asarray(cells)
    k = [np.fft.fftfreq(n, d=s / n) * 2 * np.pi for n, s in zip(cells, size)]
    uh, K = np.fft.fftn(u, axes=(0, 1, 2)), np.meshgrid(*k, indexing='ij')
    spectral = np.stack([np.stack([np.real(np.fft.ifftn(1j * K[j] * uh[..., i], axes=(0, 1, 2))) for j in range(3)],
                                  -1) for i in range(3)], -2)
    staggered = np.zeros(cells + (3, 3))
    for j in range(3):
        d = np.roll(u, -1, axis=j) - u
        for e in range(3):
            if e != j:
                d = np.roll(d, -1, axis=e) + d
        staggered[..., :, j] = d / (4 * h[j])
    err = {}
    for derivative, grad in (('continuous', spectral), ('FWBW_difference', staggered)):
        F = np.transpose(np.eye(3) + grad, (0, 1, 2, 4, 3)).reshape(cells + (9,)).reshape(-1, 9, order='F')
        o = oracle_lib.OracleSpectralBasic(cells, size, np.zeros(int(np.prod(cells))), np.array([[1.0, 0, 0, 0]]),
                                           workloads.fcc_al(), numerics_with(derivative), init=False, threads=1)
        o.set_field('F_solver', F)
        o.update_coords()
        up, _ = displacements(cells, size, *o.get_coords())
        o.close()
        ref = u.transpose(2, 1, 0, 3).reshape(-1, 3)
        err[derivative] = np.abs(up - ref).max() / np.abs(ref).max()
    assert err['continuous'] < 1e-12
    assert err['FWBW_difference'] > 0.1


@pytest.mark.parametrize('derivative', ['continuous', 'central_difference', 'FWBW_difference'])
@pytest.mark.parametrize('cells', [(5, 6, 7), (6, 4, 8)])
def test_gamma_output_is_curl_free(oracle_lib, derivative, cells):
    """Gamma_hat : tau_hat = (K^-1 tau_hat conj(xi)) (x) xi is a gradient for the same first-derivative
    frequencies that utilities_curlRMS uses (spectral_utilities.f90:697-757), so its curl RMS vanishes
    for each of the three derivatives, including the complex FWBW ones."""
    o = small_oracle(oracle_lib, cells=cells, num=numerics_with(derivative))
    tau = np.random.default_rng(13).normal(size=(o.N, 9)) * 1e8
    g = o.gamma_convolution(tau, np.zeros(9))
    F = g + np.eye(3).reshape(-1)
    assert o.curl_rms(F) < 1e-12 * np.abs(g).max()
    assert o.curl_rms(F + 1e-3 * np.abs(g).max() * np.random.default_rng(14).normal(size=F.shape)) > 1e-6 * np.abs(g).max()
    o.close()
