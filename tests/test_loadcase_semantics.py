"""Load-case semantics of the grid driver and solvers, after the reference's
tests/integration/test_grid_parse_loadcase.py: the volume-averaged F at every output increment
matches the analytic target of the deformation boundary conditions (L: true rate, dot_F:
engineering rate, F: final value; geometric time steps r; several load steps; f_out including
'none') within atol 1e-2 on the deformation-controlled components, and the averaged P matches the
prescribed stress (P: ramp to the value, dot_P: rate) within max(1e-3 max|P|, 1e3) on the
stress-controlled ones.  The reference's 2x2x2 single-grain grid and orientation; the phenopowerlaw
Al of this path instead of its J2 material (the targets do not depend on the material).

CPU: the oracle.  GPU: both solvers."""
import numpy as np
import pytest

from damask_b200 import workloads
from damask_b200.config import parse_load

rng = np.random.default_rng(20)
s = float((1 + rng.random()) * 1e-3)
LOADCASES = [
    [{'boundary_conditions': {'mechanical': {'dot_F': [[0, s, 0], [0, 0, 0], ['x', 'x', 'x']],
                                             'P': [['x', 'x', 'x'], ['x', 'x', 'x'], [0, 0, 0]]}},
      'discretization': {'t': 100, 'N': 100}, 'f_out': int(rng.integers(2, 50))}],
    [{'boundary_conditions': {'mechanical': {'dot_F': [['x', 0, 0], [s, 'x', 0], [0, 0, 'x']],
                                             'P': [[0, 'x', 'x'], ['x', 0, 'x'], ['x', 'x', 0]]}},
      'discretization': {'t': 100, 'N': 100, 'r': 1.0}, 'f_out': 10}],
    [{'boundary_conditions': {'mechanical': {'dot_F': [['x', 0, 0], [0, 0, s], [0, 0, 'x']],
                                             'P': [[0, 'x', 'x'], ['x', 'x', 'x'], ['x', 'x', 0]]}},
      'discretization': {'t': 20, 'N': 20, 'r': 1.1}}],
    [{'boundary_conditions': {'mechanical': {'P': [[0, 0, 0], ['x', 'x', 'x'], ['x', 'x', 'x']],
                                             'L': [['x', 'x', 'x'], [0, 0, 0], [1e-3, 0, s]]}},
      'discretization': {'t': 20, 'N': 20, 'r': 0.95}}],
    [{'boundary_conditions': {'mechanical': {'F': [[1.1, 0, 0], [0, float(np.sqrt(1 / 1.1)), 0],
                                                   [0, 0, float(np.sqrt(1 / 1.1))]]}},
      'discretization': {'t': 50, 'N': 30}}],
    [{'boundary_conditions': {'mechanical': {'dot_F': [['x', 0, 0], [0, 0, 0], [0, 0, 'x']],
                                             'P': [[4e7, 'x', 'x'], ['x', 'x', 'x'], ['x', 'x', 0]]}},
      'discretization': {'t': 40, 'N': 200}},
     {'boundary_conditions': {'mechanical': {'dot_F': [['x', 0, 0], [1e-2, 0, 0], [0, 0, 'x']],
                                             'P': [[1e2, 'x', 'x'], ['x', 'x', 'x'], ['x', 'x', 0]]}},
      'discretization': {'t': 40, 'N': 200}}],
    [{'boundary_conditions': {'mechanical': {'dot_F': [['x', 0, 'x'], [0, -1e-3, 2e-3], [0, 0, 0]],
                                             'dot_P': [[0, 'x', 0], ['x', 'x', 'x'], ['x', 'x', 'x']]}},
      'discretization': {'t': 30, 'N': 150}, 'f_out': int(rng.integers(4, 40))}],
    [{'boundary_conditions': {'mechanical': {'dot_F': [['x', 0, 0], [0, 0, -s], [0, 0, 'x']],
                                             'P': [[1e7, 'x', 'x'], ['x', 'x', 'x'], ['x', 'x', 0]]}},
      'discretization': {'t': 20, 'N': 60}, 'f_out': 8},
     {'boundary_conditions': {'mechanical': {'dot_F': [['x', 0, 0], [0, 0, -s], [0, 0, 'x']],
                                             'P': [[1e7, 'x', 'x'], ['x', 'x', 'x'], ['x', 'x', 0]]}},
      'discretization': {'t': 20, 'N': 20}, 'f_out': 'none'},
     {'boundary_conditions': {'mechanical': {'dot_F': [['x', 0, 0], [s, 'x', 0], [0, 0, 'x']],
                                             'P': [[0, 'x', 'x'], ['x', 0, 'x'], ['x', 'x', 0]]}},
      'discretization': {'t': 100, 'N': 100, 'r': 1.1}, 'f_out': 100}],
]


def masked(lst):
    return np.array([[0.0 if v == 'x' else float(v) for v in row] for row in lst])


def time_inc(d):
    if 'r' not in d or np.isclose(d['r'], 1.0):
        return [d['t'] / d['N']] * d['N']
    r = d['r']
    return [d['t'] * (r ** i - r ** (i + 1)) / (1.0 - r ** d['N']) for i in range(d['N'])]


def targets(loadcase):
    """Analytic averaged F, P and the stress mask at the output increments."""
    F, P, M = [np.eye(3)], [np.zeros((3, 3))], [np.zeros((3, 3), bool)]
    incs, count = [0], 0
    for step in loadcase:
        bc, dts = step['boundary_conditions']['mechanical'], time_inc(step['discretization'])
        f = step.get('f_out', 1)
        if f != 'none':
            incs += list(range(count + f, count + len(dts) + 1, f))
        count += len(dts)
        if 'P' in bc or 'dot_P' in bc:
            key = 'P' if 'P' in bc else 'dot_P'
            m = np.array(bc[key]) != 'x'
            v = masked(bc[key])
            rate = (v - P[-1]) / sum(dts) if key == 'P' else v
        else:
            m, rate = np.zeros((3, 3), bool), np.zeros((3, 3))
        for dt in dts:
            P.append(P[-1] + rate * dt)
            M.append(m)
        if 'L' in bc:
            for dt in dts:
                F.append(F[-1] + masked(bc['L']) @ F[-1] * dt)
        elif 'dot_F' in bc:
            for dt in dts:
                F.append(F[-1] + masked(bc['dot_F']) * dt)
        else:
            r = (masked(bc['F']) - F[-1]) / sum(dts)
            for dt in dts:
                F.append(F[-1] + r * dt)
    return incs, F, P, M


def run(solver, loadcase):
    from damask_b200.grid import run_load_cases
    lcs = parse_load({'loadstep': loadcase})
    incs = targets(loadcase)[0]
    out = {0: (solver.get_field('F').mean(0), solver.get_field('P').mean(0))}

    def cb(rec):
        if rec.converged and rec.inc in incs:
            out[rec.inc] = (solver.get_field('F').mean(0), solver.get_field('P').mean(0))

    stats = run_load_cases(solver, lcs, on_increment=cb)
    assert all(st.converged for st in stats)
    return out


def check(out, loadcase):
    incs, F, P, M = targets(loadcase)
    assert sorted(out) == incs
    for i in incs:
        Fc, Pc = out[i][0].reshape(3, 3, order='F'), out[i][1].reshape(3, 3, order='F')
        m = M[i]
        assert np.all(np.abs(Fc - F[i])[~m] <= 1e-2), i
        if m.any():
            assert np.all(np.abs(Pc - P[i])[m] < max(np.abs(Pc).max() * 1e-3, 1e3)), i


def grid():
    return (2, 2, 2), (1.0, 1.0, 1.0), np.zeros(8, np.int32), \
        np.array([[0.06817485875515444, 0.03985506619537109, -0.5032054951163741, 0.8605509816489446]])


@pytest.mark.parametrize('k', range(len(LOADCASES)))
def test_loadcase_targets_oracle(oracle_lib, k):
    cells, size, mat, q = grid()
    o = oracle_lib.OracleSpectralBasic(cells, size, mat, q, workloads.fcc_al(), workloads.numerics_default(), threads=1)
    check(run(o, LOADCASES[k]), LOADCASES[k])
    o.close()


@pytest.mark.gpu
@pytest.mark.parametrize('solver', ['spectral_basic', 'spectral_polarization'])
@pytest.mark.parametrize('k', range(len(LOADCASES)))
def test_loadcase_targets_gpu(gpu, k, solver):
    from damask_b200.grid import SpectralBasic
    cells, size, mat, q = grid()
    num = workloads.numerics_default()
    num.solver = solver
    g = SpectralBasic(cells, size, mat, q, workloads.fcc_al(), num)
    check(run(g, LOADCASES[k]), LOADCASES[k])
    g.close()
