"""Restart (grid_mech_spectral_basic.f90:198-235,378-416; grid_mech_spectral_polarization.f90:
236-268,400-438; phase_mechanical.f90:1248-1280): a run resumed from the restart data of
increment k continues like the uninterrupted run, for both solvers."""
import numpy as np
import pytest

from damask_b200 import synthetic, workloads
from damask_b200.grid import IncrementDriver, SpectralBasic, load_restart, save_restart

pytestmark = pytest.mark.gpu


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
    save_restart(tmp_path / 'r.npz', a.restart_write(), drv.total)
    ref = [r for _ in range(3) for r in drv.step()]
    xi_a, P_a = a.get_field('xi_sl'), a.get_field('P')
    a.close()

    data, inc = load_restart(tmp_path / 'r.npz')
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


def test_restart_rejects_mismatched_data(gpu):
    rve = synthetic.voronoi_rve((4, 4, 4), workloads.SIZE_1MM, 2, 0)
    g = SpectralBasic(rve.cells, rve.size, rve.material, rve.quaternions, workloads.fcc_al(),
                      workloads.numerics_default())
    d = g.restart_write()
    d['omega_plastic'] = d['omega_plastic'][:, :3]
    with pytest.raises(ValueError):
        g.restart_read(d)
    g.close()


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
