"""CUDA path (libdamask_b200.so, through the C-ABI) against the oracle on the same inputs.

Tolerances: FP64 results within 1e-9 relative (per voxel, relative to the field's
maximum) with equal fixed-point iteration counts; the mixed-precision form within
1e-5 relative in the volume-averaged stress.
"""
import numpy as np
import pytest

from damask_b200 import synthetic, workloads
from damask_b200.grid import SpectralBasic, run_load_cases

from conftest import assert_fields, rel

pytestmark = pytest.mark.gpu

TOL = 1e-9


def partial_families(lattice):
    """Active slip-system sums without compiled kernels: cF N_sl [6] (run as 12) and cI
    N_sl [12,12,12] (run as 48), padded with inert systems."""
    from damask_b200.config import Phase
    if lattice == 'cF':
        d = {'lattice': 'cF', 'mechanical': {
            'elastic': {'type': 'Hooke', 'C_11': 106.75e9, 'C_12': 60.41e9, 'C_44': 28.34e9},
            'plastic': {'type': 'phenopowerlaw', 'N_sl': [6], 'a_sl': [2.25], 'dot_gamma_0_sl': [0.001],
                        'h_0_sl-sl': [75e6], 'h_sl-sl': [1, 1, 1.4, 1.4, 1.4, 1.4, 1.4], 'n_sl': [20],
                        'xi_0_sl': [31e6], 'xi_inf_sl': [63e6]}}}
    else:
        d = {'lattice': 'cI', 'mechanical': {
            'elastic': {'type': 'Hooke', 'C_11': 233.3e9, 'C_12': 135.5e9, 'C_44': 118.0e9},
            'plastic': {'type': 'phenopowerlaw', 'N_sl': [12, 12, 12], 'a_sl': [2.0] * 3,
                        'dot_gamma_0_sl': [0.001] * 3, 'h_0_sl-sl': [1e9] * 3, 'h_sl-sl': [1, 1.4, 1, 1.4] + [1.4] * 24,
                        'n_sl': [20] * 3, 'xi_0_sl': [95e6, 97e6, 97e6], 'xi_inf_sl': [222e6, 412e6, 412e6]}}}
    return Phase.from_dict(d)


def pair(oracle_lib, cells, grains, seed=0, phase=None, num=None, size=workloads.SIZE_1MM, precision='fp64'):
    rve = synthetic.voronoi_rve(cells, size, grains, seed)
    phase = phase or workloads.fcc_al()
    num = num or workloads.numerics_default()
    g = SpectralBasic(rve.cells, rve.size, rve.material, rve.quaternions, phase, num, precision=precision)
    o = oracle_lib.OracleSpectralBasic(rve.cells, rve.size, rve.material, rve.quaternions, phase, num, threads=4)
    return g, o


def test_init_sweep(gpu, oracle_lib):
    g, o = pair(oracle_lib, (8, 8, 8), 5)
    for name in ('F_p', 'F_e', 'xi_sl'):
        assert rel(g.get_field(name), o.get_field(name)) < 1e-14
    ag, ao = g.aims(), o.aims()
    assert rel(ag['C_minMaxAvg'], ao['C_minMaxAvg']) < 1e-12
    assert rel(ag['C_volAvg'], ao['C_volAvg']) < 1e-12
    g.close()


@pytest.mark.parametrize('phase', [workloads.fcc_al(), workloads.bcc_24(), workloads.bcc_48(),
                                   partial_families('cF'), partial_families('cI')],
                         ids=['fcc12', 'bcc24', 'bcc48', 'fcc6_padded', 'bcc36_padded'])
def test_constitutive_response_and_tangent(gpu, oracle_lib, phase):
    """utilities_constitutiveResponse and phase_mechanical_dPdF in the plastic range."""
    g, o = pair(oracle_lib, (6, 5, 4), 4, phase=phase)
    rng = np.random.default_rng(11)
    F = np.eye(3) + np.diag([4e-3, -1.5e-3, -1.5e-3])
    Fs = np.tile(F.reshape(-1, order='F'), (g.N, 1)) + 2e-4 * rng.normal(size=(g.N, 9))
    Pg, Pavg, Cvg, Cmg, stg = g.constitutive_response(Fs, 1.0)
    Po, Pavo, Cvo, Cmo, sto = o.constitutive_response(Fs, 1.0)
    assert stg == sto == 0
    assert np.abs(Po).max() > 5e7                 # plastic
    assert rel(Pg, Po) < TOL and rel(Pavg, Pavo) < TOL
    assert rel(Cvg, Cvo) < TOL and rel(Cmg, Cmo) < TOL
    for name in ('F_p', 'L_p', 'S', 'xi_sl', 'gamma_sl', 'F_e'):
        assert_fields(g, o, [name], TOL)
    assert rel(g.dPdF(1.0), o.dPdF(1.0)) < TOL
    it = g.iteration_counts()
    assert it[:, 0].min() >= 1 and it[:, 1].min() >= 1 and np.all(it[:, 3] == 0)
    g.close()


def test_failure_status_matches(gpu, oracle_lib):
    num = workloads.numerics_default()
    num.N_iter_Lp_max = 1
    g, o = pair(oracle_lib, (2, 2, 2), 2, num=num)
    F = np.tile((np.eye(3) + np.diag([5e-3, -2e-3, -2e-3])).reshape(-1, order='F'), (g.N, 1))
    stg = g.constitutive_response(F, 1.0)[-1]
    sto = o.constitutive_response(F, 1.0)[-1]
    assert stg != 0 and sto != 0
    g.close()


def test_spectral_operators(gpu, oracle_lib, golden):
    num = workloads.numerics_default()
    num.divergence_correction = 'size'
    f = golden['div_field']
    g, o = pair(oracle_lib, f.shape[:3], 3, num=num, size=tuple(golden['div_size']))
    P = f.transpose(2, 1, 0, 4, 3).reshape(-1, 9)
    assert rel(g.divergence_rms(P), golden['div_rms']) < 1e-12      # reference python/damask/grid.py
    aim = np.random.default_rng(2).normal(size=9)
    assert rel(g.gamma_convolution(P, aim), o.gamma_convolution(P, aim)) < 1e-12
    g.close()


def run_both(g, o, n):
    sg = run_load_cases(g, workloads.tension_x(60.0, 60), max_increments=n)
    so = run_load_cases(o, workloads.tension_x(60.0, 60), max_increments=n)
    return sg, so


@pytest.mark.parametrize('case', ['fcc16_anderson', 'fcc8_richardson', 'bcc8_anderson', 'bcc48_anderson',
                                  'bcc36_padded'])
def test_solver_parity(gpu, oracle_lib, case):
    """grid_mechanical_spectral_basic_{forward,solution} + materialpoint_forward over several
    increments of uniaxial tension: per-voxel fields within 1e-9, identical iteration counts."""
    num = workloads.numerics_default()
    if case == 'fcc16_anderson':
        g, o, n = *pair(oracle_lib, (16, 16, 16), 20), 3
    elif case == 'fcc8_richardson':
        num.PETSc_options = '-snes_type nrichardson'
        g, o, n = *pair(oracle_lib, (8, 8, 8), 6, num=num), 3
    elif case == 'bcc36_padded':
        g, o, n = *pair(oracle_lib, (8, 8, 8), 10, seed=3, phase=partial_families('cI')), 2
    elif case == 'bcc48_anderson':
        # all three cI families, N_sl [12,12,24]
        g, o, n = *pair(oracle_lib, (8, 8, 8), 10, seed=3, phase=workloads.bcc_48()), 2
    else:
        g, o, n = *pair(oracle_lib, (8, 8, 8), 10, seed=3, phase=workloads.bcc_24()), 2
    sg, so = run_both(g, o, n)
    assert [s.iterations for s in sg] == [s.iterations for s in so]
    for a, b in zip(sg, so):
        assert rel(a.P_av, b.P_av) < TOL
    for name in ('P', 'F', 'F_p', 'L_p', 'S', 'xi_sl', 'gamma_sl', 'O'):
        assert_fields(g, o, [name], TOL)
    assert rel(g.aims()['C_volAvg'], o.aims()['C_volAvg']) < TOL
    # coordinates of the last updateCoords (after every converged increment)
    for a, b in zip(g.get_coords(), o.get_coords()):
        assert rel(a, b) < TOL
    g.close()


@pytest.mark.parametrize('derivative', ['continuous', 'FWBW_difference'])
def test_mixed_precision_within_1e5(gpu, oracle_lib, derivative):
    """FP32 FFT/Gamma/field update with the FP64 correction sweep: <P> within 1e-5 of FP64 (the
    FP32 instantiations of both Gamma kernels)."""
    rve = synthetic.voronoi_rve((16, 16, 16), workloads.SIZE_1MM, 12, 3)
    ph, num = workloads.bcc_24(), workloads.numerics_default()
    num.derivative = derivative
    res = {}
    for prec in ('fp64', 'mixed'):
        s = SpectralBasic(rve.cells, rve.size, rve.material, rve.quaternions, ph, num, precision=prec)
        res[prec] = (run_load_cases(s, workloads.tension_x(100.0, 100), max_increments=3), s.get_field('P'))
        s.close()
    for a, b in zip(res['mixed'][0], res['fp64'][0]):
        assert rel(a.P_av, b.P_av) < 1e-5
    assert rel(res['mixed'][1], res['fp64'][1]) < 1e-5


def test_field_access_roundtrip(gpu, oracle_lib):
    g, _ = pair(oracle_lib, (4, 3, 2), 2)
    F = np.tile(np.eye(3).reshape(-1, order='F'), (g.N, 1)) + 1e-3 * np.arange(g.N * 9).reshape(g.N, 9) / g.N
    g.set_field('F_solver', F)
    assert np.array_equal(g.get_field('F_solver'), F)
    assert g.get_field('xi_sl').shape == (g.N, 12)
    assert np.array_equal(g.get_field('F_i'), np.tile(np.eye(3).reshape(-1), (g.N, 1)))
    g.close()


def test_stress_field_as_first_read(gpu, oracle_lib):
    """dmk_get_field(S) as the first field read of a context: its staging buffer is
    allocated on demand, as for every other field.  After the initial sweep S is the
    rounding residue of Fe^T Fe - I for a rotation Fe (~1e-5 Pa), so the two agree to
    an absolute 1e-3 Pa, far below any stress of the path."""
    g, o = pair(oracle_lib, (4, 3, 2), 2)
    Sg, So = g.get_field('S'), o.get_field('S')
    assert np.isfinite(Sg).all() and np.abs(Sg - So).max() < 1e-3
    g.close()


@pytest.mark.parametrize('case', ['odd', 'smooth'])
def test_update_coords_golden(gpu, oracle_lib, golden, case):
    """utilities_updateCoords on the device against the reference's Python form."""
    from test_oracle import voxel_tensors
    F = golden[f'coords_{case}_F']
    cells = F.shape[:3]
    g = SpectralBasic(cells, tuple(golden[f'coords_{case}_size']), np.zeros(int(np.prod(cells))),
                      np.array([[1.0, 0, 0, 0]]), workloads.fcc_al(), workloads.numerics_default())
    g.set_field('F_solver', voxel_tensors(F))
    g.update_coords()
    ip, nodes = g.get_coords()
    g.close()
    assert rel(ip, golden[f'coords_{case}_ip'].reshape(-1, 3, order='F')) < 1e-13
    assert rel(nodes, golden[f'coords_{case}_nodes'].reshape(-1, 3, order='F')) < 1e-13


@pytest.mark.parametrize("cells", [(8, 6, 4), (5, 7, 9), (6, 3, 2), (16, 16, 16)])
def test_update_coords_random_field(gpu, oracle_lib, cells):
    """Random F fields (content at every frequency, Nyquist included on even edges): device and
    oracle coordinates agree, and before the first update both are the undeformed ones."""
    from damask_b200.grid import coordinates0
    size = (1.0e-3, 2.0e-3, 1.5e-3)
    N = int(np.prod(cells))
    g, o = pair(oracle_lib, cells, 1, size=size)
    ip0, n0 = coordinates0(cells, size)
    for a, b in zip(g.get_coords(), (ip0, n0)):
        assert rel(a, b) < 1e-15
    F = np.tile(np.eye(3).reshape(-1), (N, 1)) + 0.05 * np.random.default_rng(11).normal(size=(N, 9))
    for s in (g, o):
        s.set_field('F_solver', F)
        s.update_coords()
    for a, b in zip(g.get_coords(), o.get_coords()):
        assert rel(a, b) < 1e-12
    g.close()


@pytest.mark.parametrize('cells', [(16, 16, 1), (1, 16, 16), (16, 1, 16)])
@pytest.mark.parametrize('solver', ['spectral_basic', 'spectral_polarization'])
def test_quasi_2d_grids(gpu, oracle_lib, cells, solver):
    """One-cell-thick grids (the reference halves the divergence and curl sums for cells(1) = 1)."""
    num = workloads.numerics_default()
    num.solver = solver
    g, o = pair(oracle_lib, cells, 8, seed=2, num=num)
    sg, so = run_both(g, o, 3)
    assert [s.iterations for s in sg] == [s.iterations for s in so]
    assert all(s.converged for s in sg)
    for a, b in zip(sg, so):
        assert rel(a.P_av, b.P_av) < TOL
    for name in ('P', 'F', 'F_p', 'xi_sl', 'gamma_sl'):
        assert_fields(g, o, [name], TOL)
    for a, b in zip(g.get_coords(), o.get_coords()):
        assert rel(a, b) < TOL
    g.close()


LOADS = {
    'simple_shear': {'dot_F': [[0, 1.0e-3, 0], [0, 0, 0], [0, 0, 0]]},
    'L_tension': {'L': [[1.0e-3, 0, 0], [0, 'x', 0], [0, 0, 'x']], 'P': [['x', 'x', 'x'], ['x', 0, 'x'], ['x', 'x', 0]]},
    'F_target': {'F': [[1.02, 0, 0], [0, 'x', 0], [0, 0, 'x']], 'P': [['x', 'x', 'x'], ['x', 0, 'x'], ['x', 'x', 0]]},
    'dot_P_xx': {'dot_F': [['x', 0, 0], [0, 0, 0], [0, 0, 0]], 'dot_P': [[2.0e6, 'x', 'x'], ['x', 'x', 'x'], ['x', 'x', 'x']]},
    'rotated_tension': {'dot_F': [[1.0e-3, 0, 0], [0, 'x', 0], [0, 0, 'x']],
                        'P': [['x', 'x', 'x'], ['x', 0, 'x'], ['x', 'x', 0]], 'R': [0.0, 0.6, 0.8, 35.0]},
}


@pytest.mark.parametrize('load', sorted(LOADS))
def test_boundary_condition_types(gpu, oracle_lib, load):
    """Deformation BCs L / dot_F / F, stress BCs P / dot_P and the load-case rotation R
    (DAMASK_grid.f90:472-689; forward grid_mech_spectral_basic.f90:284-355)."""
    from damask_b200.config import parse_load
    lcs = parse_load({'loadstep': [{'boundary_conditions': {'mechanical': LOADS[load]},
                                    'discretization': {'t': 10.0, 'N': 10}}]})
    g, o = pair(oracle_lib, (8, 8, 8), 5, seed=4)
    sg = run_load_cases(g, lcs, max_increments=3)
    so = run_load_cases(o, lcs, max_increments=3)
    assert [s.iterations for s in sg] == [s.iterations for s in so]
    assert all(s.converged for s in sg)
    for a, b in zip(sg, so):
        assert rel(a.P_av, b.P_av) < TOL
    for name in ('P', 'F', 'xi_sl'):
        assert_fields(g, o, [name], TOL)
    for k in ('F_aim', 'P_aim'):
        assert rel(g.aims()[k], o.aims()[k]) < TOL, k
    g.close()


def test_displacements_of_the_converged_field(gpu, oracle_lib):
    """After the reference's tests/integration/test_grid_displacements.py: at the end of a two-step
    load (tension, then shear) on a random two-orientation grid, the cell-centre displacements the
    solver reports equal the displacement field of its converged F (computed here by the oracle's
    restatement of utilities_updateCoords, which matches the reference's
    damask.grid.displacement_point)."""
    from damask_b200.config import parse_load
    from damask_b200.grid import displacements
    rng = np.random.default_rng(8)
    cells = tuple(int(c) for c in rng.integers(5, 12, 3))
    size = tuple(float(x) for x in rng.random(3) + 1.0)
    mat = rng.integers(0, 2, int(np.prod(cells))).astype(np.int32)
    q = np.array([[1.0, 0, 0, 0], [0.0, 0.6, 0.8, 0.0]])
    lcs = parse_load({'loadstep': [
        {'boundary_conditions': {'mechanical': {'dot_F': [[1.0e-3, 0, 0], [0, 'x', 0], [0, 0, 'x']],
                                                'P': [['x', 'x', 'x'], ['x', 0, 'x'], ['x', 'x', 0]]}},
         'discretization': {'t': 10, 'N': 40}, 'f_out': 4},
        {'boundary_conditions': {'mechanical': {'dot_F': [[0, 0, 0], [1.0e-3, 0, 0], [0, 0, 0]]}},
         'discretization': {'t': 40, 'N': 80}, 'f_out': 20}]})
    g = SpectralBasic(cells, size, mat, q, workloads.fcc_al(), workloads.numerics_default())
    stats = run_load_cases(g, lcs)
    assert len(stats) >= 120 and all(s.converged for s in stats)
    ip, nodes = g.get_coords()
    F = g.get_field('F')
    g.close()
    o = oracle_lib.OracleSpectralBasic(cells, size, mat, q, workloads.fcc_al(), init=False, threads=1)
    o.set_field('F_solver', F)
    o.update_coords()
    ip_o, nodes_o = o.get_coords()
    o.close()
    u_p, _ = displacements(cells, size, ip, nodes)
    u_o, _ = displacements(cells, size, ip_o, nodes_o)
    assert np.allclose(u_p, u_o, rtol=1e-5, atol=1e-8)
    assert rel(ip, ip_o) < 1e-12 and rel(nodes, nodes_o) < 1e-12


def test_fp64_peak_probe(gpu):
    """The FP64 FMA probe behind the bench's FP64 roofline gives a plausible B200 figure."""
    import ctypes as C
    from damask_b200 import _lib
    out = C.c_double()
    _lib.check(_lib.load().dmk_fp64_peak(0, C.byref(out)))
    assert 10.0 < out.value < 80.0


@pytest.mark.parametrize('option', ['update_gamma', 'divergence_correction_none', 'divergence_correction_size',
                                    'central_difference', 'FWBW_difference'])
def test_numerics_options(gpu, oracle_lib, option):
    """update_gamma (Gamma re-based on C_minMaxAvg every solution, spectral_utilities.f90:356-395)
    and the divergence_correction modes (scaledGeomSize, :181-197) on a non-cubic RVE."""
    num = workloads.numerics_default()
    if option == 'update_gamma':
        num.update_gamma = True
    elif option in ('central_difference', 'FWBW_difference'):
        num.derivative = option                    # utilities_getFreqDerivative, :808-850
    else:
        num.divergence_correction = option.split('_')[-1]
    g, o = pair(oracle_lib, (8, 6, 10), 6, seed=5, num=num, size=(1.0e-3, 0.75e-3, 1.25e-3))
    sg, so = run_both(g, o, 3)
    assert [s.iterations for s in sg] == [s.iterations for s in so]
    for a, b in zip(sg, so):
        assert rel(a.P_av, b.P_av) < TOL
    for name in ('P', 'F', 'xi_sl'):
        assert_fields(g, o, [name], TOL)
    g.close()


@pytest.mark.parametrize('cells', [(5, 6, 7), (6, 4, 8), (1, 6, 5), (5, 7, 3)])
def test_fwbw_spectral_operators(gpu, oracle_lib, cells):
    """The complex FWBW frequencies (spectral_utilities.f90:823-849) in every spectral operator:
    divergence RMS, Gamma convolution (complex inverse of the acoustic tensor), curl RMS and, on
    grids without a Nyquist index (even edges give near-zero |xi|^2 at points other than k = 0),
    the coordinate update."""
    num = workloads.numerics_default()
    num.derivative = 'FWBW_difference'
    size = (1.0e-3, 0.8e-3, 1.2e-3)
    g, o = pair(oracle_lib, cells, 3, num=num, size=size)
    rng = np.random.default_rng(21)
    P = rng.normal(size=(g.N, 9)) * 1e8
    aim = rng.normal(size=9)
    assert rel(g.divergence_rms(P), o.divergence_rms(P)) < 1e-12
    assert rel(g.gamma_convolution(P, aim), o.gamma_convolution(P, aim)) < 1e-12
    F = np.tile(np.eye(3).reshape(-1), (g.N, 1)) + 0.05 * rng.normal(size=(g.N, 9))
    assert rel(g.curl_rms(F), o.curl_rms(F)) < 1e-12
    if all(n % 2 == 1 for n in cells):
        for s in (g, o):
            s.set_field('F_solver', F)
            s.update_coords()
        for a, b in zip(g.get_coords(), o.get_coords()):
            assert rel(a, b) < 1e-12
    g.close()


@pytest.mark.parametrize('cells', [(64, 32, 64), (64, 64, 48)])
def test_two_and_three_voxel_chunks(gpu, oracle_lib, cells):
    """Contexts of 2^17 and 3 * 2^16 voxels split their constitutive passes into two and three
    chunks on their own streams; results as the oracle's."""
    g, o = pair(oracle_lib, cells, 30, seed=6)
    sg, so = run_both(g, o, 1)
    assert [s.iterations for s in sg] == [s.iterations for s in so]
    assert rel(sg[0].P_av, so[0].P_av) < TOL
    for name in ('P', 'xi_sl', 'gamma_sl'):
        assert_fields(g, o, [name], TOL)
    g.close()
