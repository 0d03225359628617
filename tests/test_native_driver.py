"""The C++ increment loop (dmk_grid_run, DAMASK_grid.f90:288-460) against the Python restatement
of the same loop: identical increments, times, cutback levels, iterations and results, driving the
oracle (CPU) through its procedure table and the CUDA context directly (GPU)."""
import numpy as np
import pytest

from damask_b200 import synthetic, workloads
from damask_b200.config import parse_load
from damask_b200.grid import NotConverged, run_load_cases, run_load_cases_native

from test_loadcase_semantics import LOADCASES


def same(a, b):
    assert [(r.inc, r.cutback_level, r.iterations, r.residual_evals) for r in a] == \
        [(r.inc, r.cutback_level, r.iterations, r.residual_evals) for r in b]
    for x, y in zip(a, b):
        assert x.t == y.t
        assert np.array_equal(x.P_av, y.P_av)


def oracle(oracle_lib, cells=(6, 6, 6), num=None):
    rve = synthetic.voronoi_rve(cells, workloads.SIZE_1MM, 4, 3)
    return oracle_lib.OracleSpectralBasic(rve.cells, rve.size, rve.material, rve.quaternions, workloads.fcc_al(),
                                          num or workloads.numerics_default(), threads=2)


@pytest.mark.parametrize('k', [0, 2, 3, 5, 7])
def test_native_loop_equals_python_loop(oracle_lib, k):
    lcs = parse_load({'loadstep': LOADCASES[k]})
    a, b = oracle(oracle_lib), oracle(oracle_lib)
    same(run_load_cases_native(a, lcs, max_increments=25), run_load_cases(b, lcs, max_increments=25))
    assert np.array_equal(a.get_field('F'), b.get_field('F'))
    a.close(), b.close()


def test_native_loop_cutbacks_and_restart_skip(oracle_lib):
    """N_iter_max = 2 forces cutbacks (and finally IO_error 950); restart_inc skips increments."""
    num = workloads.numerics_default()
    num.N_iter_max = 6
    lcs = workloads.tension_x(60.0, 60)
    outs = []
    for run in (run_load_cases_native, run_load_cases):
        o = oracle(oracle_lib, num=num)
        try:
            run(o, lcs, max_increments=6)
            outs.append(None)
        except NotConverged as e:
            outs.append(str(e).split(' did not')[0])
        o.close()
    assert outs[0] == outs[1]
    a, b = oracle(oracle_lib), oracle(oracle_lib)
    same(run_load_cases_native(a, lcs, max_increments=6, restart_inc=3),
         run_load_cases(b, lcs, max_increments=6, restart_inc=3))
    a.close(), b.close()


@pytest.mark.gpu
def test_native_loop_drives_the_context(gpu):
    from damask_b200.grid import SpectralBasic
    rve = synthetic.voronoi_rve((16, 16, 16), workloads.SIZE_1MM, 20, 0)
    args = (rve.cells, rve.size, rve.material, rve.quaternions, workloads.fcc_al(), workloads.numerics_default())
    a, b = SpectralBasic(*args), SpectralBasic(*args)
    lcs = workloads.tension_x(60.0, 60)
    same(run_load_cases_native(a, lcs, max_increments=5), run_load_cases(b, lcs, max_increments=5))
    assert np.array_equal(a.get_field('P'), b.get_field('P'))
    for x, y in zip(a.get_coords(), b.get_coords()):
        assert np.array_equal(x, y)
    a.close(), b.close()
