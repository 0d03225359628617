"""The spectral polarization solver (grid_mech_spectral_polarization.f90) and its curl
criterion (utilities_curlRMS, spectral_utilities.f90:695-757).

CPU: the oracle's two solvers reproduce the reference's cross-solver consistency test
(tests/integration/test_grid_mech_consistency.py: same job with each grid solver, every output
within rtol 1e-5, atol 1e-2), and the curl criterion vanishes on compatible fields.
GPU: the CUDA polarization solver against the oracle at 1e-9 with equal iteration counts.
"""
import json
from pathlib import Path

import numpy as np
import pytest

from damask_b200 import config, synthetic, workloads
from damask_b200.grid import run_load_cases

from conftest import assert_fields, rel

GOLD = Path(__file__).resolve().parent / 'golden' / 'golden_mech_consistency.npz'
TOL = 1e-9


def consistency_inputs():
    g = np.load(GOLD)
    phase = config.Phase.from_dict(json.loads(str(g['phase_json'])))
    lcs = config.parse_load(json.loads(str(g['load_json'])))
    return tuple(int(c) for c in g['cells']), tuple(float(s) for s in g['size']), g['material'], g['quaternions'], \
        phase, lcs


def run_outputs(solver, lcs):
    """Fields of the phase outputs (F, F_e, F_p, L_p, O) at the f_out increments."""
    rec = {}

    def cb(r):
        if r.converged and r.inc % lcs[0].f_out == 0:
            rec[r.inc] = {k: solver.get_field(k).copy() for k in ('F', 'F_e', 'F_p', 'L_p', 'O')}

    stats = run_load_cases(solver, lcs, on_increment=cb)
    return rec, stats


def test_oracle_solvers_pass_reference_consistency_test(oracle_lib):
    cells, size, mat, q, phase, lcs = consistency_inputs()
    out = {}
    for name in ('spectral_basic', 'spectral_polarization'):
        num = config.Numerics()
        num.solver = name
        o = oracle_lib.OracleSpectralBasic(cells, size, mat, q, phase, num, threads=4)
        out[name], stats = run_outputs(o, lcs)
        o.close()
        assert len(stats) == 100 and all(s.converged for s in stats)
    a, b = out['spectral_basic'], out['spectral_polarization']
    assert sorted(a) == list(range(10, 101, 10))
    for inc in a:
        for k in a[inc]:
            x, y = a[inc][k], b[inc][k]
            close = np.logical_or(np.isclose(x, y, rtol=1e-5, atol=1e-2), np.isclose(y, x, rtol=1e-5, atol=1e-2))
            assert close.all(), (inc, k)


def test_curl_of_compatible_field_vanishes(oracle_lib):
    """F = I + grad u of a periodic u (spectral gradient, so exactly compatible) has zero curl;
    a random field does not."""
    cells, size = (8, 6, 5), (1.0e-3, 2.0e-3, 1.5e-3)
    o = oracle_lib.OracleSpectralBasic(cells, size, np.zeros(240), np.array([[1.0, 0, 0, 0]]), workloads.fcc_al(),
                                       init=False, threads=1)
    rng = np.random.default_rng(5)
    u = rng.normal(size=cells + (3,)) * 1e-6
    k = [np.fft.fftfreq(n, d=s / n) * 2 * np.pi for n, s in zip(cells, size)]
    for d, n in enumerate(cells):
        if n % 2 == 0:
            k[d][n // 2] = 0.0            # first derivative without the Nyquist frequency
    uh = np.fft.fftn(u, axes=(0, 1, 2))
    K = np.meshgrid(*k, indexing='ij')
    grad = np.stack([np.stack([np.real(np.fft.ifftn(1j * K[j] * uh[..., i], axes=(0, 1, 2))) for j in range(3)], -1)
                     for i in range(3)], -2)
    F = np.eye(3) + grad
    voxels = np.transpose(F, (0, 1, 2, 4, 3)).reshape(cells + (9,)).reshape(-1, 9, order='F')
    assert o.curl_rms(voxels) < 1e-12 * np.abs(grad).max()
    assert o.curl_rms(voxels + 1e-3 * rng.normal(size=voxels.shape)) > 1e-5
    o.close()


@pytest.mark.parametrize('cells', [(8, 6, 5), (5, 7, 3)])
def test_curl_of_fwbw_gradient_vanishes(oracle_lib, cells):
    """With derivative: FWBW_difference (spectral_utilities.f90:823-849) the compatible fields are
    the staggered gradients G_ij = D_j A_e A_f u_i / (4 h_j) (D x = x(n + 1) - x(n) along j,
    A x = x(n + 1) + x(n) along the two other directions): their spectra are u_hat (x) xi, whose
    curl vanishes; the same field is not curl-free for the continuous frequencies."""
    size = (1.0e-3, 2.0e-3, 1.5e-3)
    rng = np.random.default_rng(6)
    u = rng.normal(size=cells + (3,)) * 1e-6
    h = np.asarray(size) / np.asarray(cells)
    grad = np.zeros(cells + (3, 3))
    for j in range(3):
        d = np.roll(u, -1, axis=j) - u
        for e in range(3):
            if e != j:
                d = np.roll(d, -1, axis=e) + d
        grad[..., :, j] = d / (4 * h[j])
    voxels = np.transpose(np.eye(3) + grad, (0, 1, 2, 4, 3)).reshape(cells + (9,)).reshape(-1, 9, order='F')
    res = {}
    for derivative in ('FWBW_difference', 'continuous'):
        num = workloads.numerics_default()
        num.derivative = derivative
        o = oracle_lib.OracleSpectralBasic(cells, size, np.zeros(int(np.prod(cells))), np.array([[1.0, 0, 0, 0]]),
                                           workloads.fcc_al(), num, init=False, threads=1)
        res[derivative] = o.curl_rms(voxels)
        o.close()
    assert res['FWBW_difference'] < 1e-12 * np.abs(grad).max()
    assert res['continuous'] > 1e-3 * np.abs(grad).max()


def test_polarization_numerics_validation():
    num = config.Numerics()
    num.solver = 'spectral_polarization'
    num.alpha = 2.5
    with pytest.raises(ValueError, match='alpha'):
        num.to_struct()
    num.alpha, num.eps_abs_curl = 1.0, 0.0
    with pytest.raises(ValueError, match='eps_abs_curl'):
        num.to_struct()
    assert config.mechanical_solver({'solver': {'mechanical': 'spectral_polarization'}}) == 'spectral_polarization'
    with pytest.raises(ValueError):
        config.mechanical_solver({'solver': {'mechanical': 'FEM'}})


# ------------------------------------------------------------------------------- GPU
def gpu_pair(oracle_lib, cells, grains, seed=0, phase=None, snes='ngmres', derivative='continuous',
             update_gamma=False):
    from damask_b200.grid import SpectralPolarization
    rve = synthetic.voronoi_rve(cells, workloads.SIZE_1MM, grains, seed)
    phase = phase or workloads.fcc_al()
    num = workloads.numerics_default()
    num.solver = 'spectral_polarization'
    num.derivative = derivative
    num.update_gamma = update_gamma
    if snes == 'nrichardson':
        num.PETSc_options = '-snes_type nrichardson'
    g = SpectralPolarization(rve.cells, rve.size, rve.material, rve.quaternions, phase, num)
    o = oracle_lib.OracleSpectralBasic(rve.cells, rve.size, rve.material, rve.quaternions, phase, num, threads=4)
    return g, o


@pytest.mark.gpu
@pytest.mark.parametrize('case', ['fcc16_anderson', 'fcc8_richardson', 'bcc8_anderson', 'fcc9_fwbw', 'fcc8_central',
                                  'fcc8_update_gamma'])
def test_polarization_parity(gpu, oracle_lib, case):
    if case == 'fcc16_anderson':
        g, o = gpu_pair(oracle_lib, (16, 16, 16), 20)
        n = 3
    elif case == 'fcc8_richardson':
        g, o = gpu_pair(oracle_lib, (8, 8, 8), 6, snes='nrichardson')
        n = 3
    elif case == 'fcc9_fwbw':
        g, o = gpu_pair(oracle_lib, (9, 7, 5), 6, seed=2, derivative='FWBW_difference')
        n = 3
    elif case == 'fcc8_central':
        g, o = gpu_pair(oracle_lib, (8, 6, 10), 6, seed=4, derivative='central_difference')
        n = 3
    elif case == 'fcc8_update_gamma':
        # Gamma and the polarization scales re-based on C_minMaxAvg every solution (:291-295)
        g, o = gpu_pair(oracle_lib, (8, 8, 8), 6, seed=5, update_gamma=True)
        n = 3
    else:
        g, o = gpu_pair(oracle_lib, (8, 8, 8), 10, seed=3, phase=workloads.bcc_24())
        n = 2
    lcs = workloads.tension_x(60.0, 60)
    sg = run_load_cases(g, lcs, max_increments=n)
    so = run_load_cases(o, lcs, max_increments=n)
    assert [s.iterations for s in sg] == [s.iterations for s in so]
    assert all(s.converged for s in sg)
    for a, b in zip(sg, so):
        assert rel(a.P_av, b.P_av) < TOL
    for name in ('P', 'F', 'F_p', 'L_p', 'S', 'xi_sl', 'gamma_sl', 'F_tau', 'F_tau_lastinc'):
        assert_fields(g, o, [name], TOL)
    assert rel(g.aims()['C_volAvg'], o.aims()['C_volAvg']) < TOL
    # the difference schemes' |xi|^2 is ~1e-32 at Nyquist points of even grids (sin(pi) rounds to
    # 1.2e-16), where utilities_updateCoords divides by it: coordinates there are rounding noise
    if g.numerics.derivative == 'continuous' or all(n % 2 == 1 for n in g.cells):
        for a, b in zip(g.get_coords(), o.get_coords()):
            assert rel(a, b) < TOL
    g.close()


@pytest.mark.gpu
@pytest.mark.parametrize('cells', [(8, 6, 4), (5, 7, 9), (2, 3, 4)])
def test_curl_rms_parity(gpu, oracle_lib, cells):
    from damask_b200.grid import SpectralBasic
    rve = synthetic.voronoi_rve(cells, workloads.SIZE_1MM, 2, 0)
    g = SpectralBasic(rve.cells, rve.size, rve.material, rve.quaternions, workloads.fcc_al(),
                      workloads.numerics_default())
    o = oracle_lib.OracleSpectralBasic(rve.cells, rve.size, rve.material, rve.quaternions, workloads.fcc_al(),
                                       workloads.numerics_default(), init=False, threads=1)
    F = np.tile(np.eye(3).reshape(-1), (g.N, 1)) + 0.05 * np.random.default_rng(4).normal(size=(g.N, 9))
    assert rel(g.curl_rms(F), o.curl_rms(F)) < 1e-12
    g.close()
