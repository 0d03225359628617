"""Restart (grid_mech_spectral_basic.f90:198-235,378-416; grid_mech_spectral_polarization.f90:
236-268,400-438; phase_mechanical.f90:1248-1280): a run resumed from the restart data of
increment k continues like the uninterrupted run, for both solvers."""
import numpy as np
import pytest

from damask_b200 import synthetic, workloads
from damask_b200.grid import IncrementDriver, SpectralBasic, load_restart, save_restart


@pytest.mark.gpu
@pytest.mark.parametrize('solver', ['spectral_basic', 'spectral_polarization'])
def test_restart_resumes_the_run(gpu, tmp_path, solver):
    rve = synthetic.voronoi_rve((8, 8, 8), workloads.SIZE_1MM, 6, 1)
    num = workloads.numerics_default()
    num.solver = solver
    args = (rve.cells, rve.size, rve.material, rve.quaternions, workloads.fcc_al(), num)
    lcs = workloads.tension_x(60.0, 60)
    a = SpectralBasic(*args)
    drv = IncrementDriver(a, lcs)
    for _ in range(4):
        drv.step()
    save_restart(tmp_path / 'job_restart.hdf5', a.restart_write(), drv.total)
    ref = [r for _ in range(3) for r in drv.step()]
    xi_a, P_a = a.get_field('xi_sl'), a.get_field('P')
    a.close()

    data, inc = load_restart(tmp_path / 'job_restart.hdf5')
    assert inc == 4
    b = SpectralBasic(*args)
    b.restart_read(data)
    drv_b = IncrementDriver(b, lcs, restart_inc=inc)
    res = [r for _ in range(7) for r in drv_b.step()]
    assert [r.inc for r in res] == [r.inc for r in ref] == [5, 6, 7]
    # the resumed run starts its first Newton from the Lp of a dt = 0 sweep and S0 = 0 (as the
    # reference), so it reaches the same fixed point within the solver tolerances
    for x, y in zip(res, ref):
        assert abs(x.iterations - y.iterations) <= 1
        assert np.abs(x.P_av - y.P_av).max() / np.abs(y.P_av).max() < 1e-3
    assert np.abs(b.get_field('xi_sl') - xi_a).max() / np.abs(xi_a).max() < 1e-4
    assert np.abs(b.get_field('P') - P_a).max() / np.abs(P_a).max() < 1e-2
    b.close()


@pytest.mark.gpu
def test_restart_rejects_mismatched_data(gpu):
    rve = synthetic.voronoi_rve((4, 4, 4), workloads.SIZE_1MM, 2, 0)
    g = SpectralBasic(rve.cells, rve.size, rve.material, rve.quaternions, workloads.fcc_al(),
                      workloads.numerics_default())
    d = g.restart_write()
    d['omega_plastic'] = d['omega_plastic'][:, :3]
    with pytest.raises(ValueError):
        g.restart_read(d)
    g.close()


@pytest.mark.gpu
def test_restart_state_of_padded_phase(gpu):
    """A phase whose active slip systems run on a larger compiled count (cF N_sl [6] on 12) writes
    and reads omega_plastic with the active systems only (xi then gamma per voxel, sizeState = 2 Ns)."""
    from test_gpu_parity import partial_families
    rve = synthetic.voronoi_rve((6, 6, 6), workloads.SIZE_1MM, 4, 2)
    ph = partial_families('cF')
    args = (rve.cells, rve.size, rve.material, rve.quaternions, ph, workloads.numerics_default())
    a = SpectralBasic(*args)
    drv = IncrementDriver(a, workloads.tension_x(60.0, 60))
    for _ in range(3):
        drv.step()
    d = a.restart_write()
    xi, ga = a.get_field('xi_sl'), a.get_field('gamma_sl')
    assert xi.shape == ga.shape == (a.N, 6) and np.abs(ga).max() > 0.0
    assert np.array_equal(d['omega_plastic'][:, :6], xi) and np.array_equal(d['omega_plastic'][:, 6:], ga)
    a.close()
    b = SpectralBasic(*args)
    b.restart_read(d)
    assert np.array_equal(b.restart_write()['omega_plastic'], d['omega_plastic'])
    b.close()


def test_restart_file_layout_and_round_trip(tmp_path):
    """<job>_restart.hdf5 holds the reference's groups and datasets (solver, phase/<name>,
    homogenization/<name>) with libhdf5's shapes for Fortran (3,3,N) arrays, and reads back
    exactly (CPU only: synthetic restart data)."""
    from damask_b200.h5read import DADF5
    rng = np.random.default_rng(4)
    N, ns = 30, 12
    d = {k: rng.normal(size=(N, 9)) for k in ('F', 'F_lastinc', 'F_phase', 'F_p', 'L_p')}
    d['omega_plastic'] = rng.normal(size=(N, 2 * ns))
    for k in ('P_aim', 'F_aim', 'F_aim_lastinc', 'F_aimDot'):
        d[k] = rng.normal(size=9)
    for k in ('C_volAvg', 'C_volAvgLastInc', 'C_minMaxAvg'):
        d[k] = rng.normal(size=81)
    p = tmp_path / 'job_restart.hdf5'
    save_restart(p, d, 17, phase_name='Aluminum', homogenization_name='SX')
    f = DADF5(p)
    assert sorted(f.keys('')) == ['homogenization', 'phase', 'solver']
    assert sorted(f.keys('solver')) == sorted(['F', 'F_lastinc', 'P_aim', 'F_aim', 'F_aim_lastinc', 'F_aimDot',
                                               'C_volAvg', 'C_volAvgLastInc', 'C_minMaxAvg'])
    assert sorted(f.keys('phase/Aluminum')) == sorted(['omega_plastic', 'F', 'F_p', 'F_i', 'L_p', 'L_i'])
    assert f.keys('homogenization') == ['SX']
    assert f.read('solver/F').shape == (N, 3, 3) and f.read('solver/C_volAvg').shape == (3, 3, 3, 3)
    assert f.read('phase/Aluminum/omega_plastic').shape == (N, 2 * ns)
    # Fortran order: F(i,j,e) is element [e, j, i]
    assert f.read('solver/F')[3, 2, 1] == d['F'][3, 1 + 3 * 2]
    back, inc = load_restart(p, phase_name='Aluminum')
    assert inc == 17
    for k, v in d.items():
        assert np.array_equal(back[k], v), k
