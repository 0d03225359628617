"""End-to-end runs of the workloads the path is specified on (synthetic inputs generated with
the reference's own recipe: uniform seeds, Gaussian quaternions, periodic Voronoi).

* 16^3, 20 grains (seed 0), fcc, tension to 6 % in 60 increments — the configuration the
  reference's CPU path runs: the FP64 CUDA path and the oracle over all 60 increments, equal
  fixed-point iteration counts, <P> within 1e-9 at every increment, fields within 1e-9 at the end.
* 64^3, 200 grains (seed 1), fcc, tension to 10 % in 100 increments: FP64 against the mixed
  form (FP32 FFT/Gamma/field update, FP64 constitutive update and correction sweep), <P>
  within 1e-5 at every increment; the first two increments of the FP64 form against the oracle.
"""
import numpy as np
import pytest

from damask_b200 import workloads
from damask_b200.grid import SpectralBasic, run_load_cases

from conftest import rel

pytestmark = pytest.mark.gpu


def test_grid16_fcc_full_run(gpu, oracle_lib):
    rve, phase, lcs, num = workloads.make('grid16_fcc_20g')
    g = SpectralBasic(rve.cells, rve.size, rve.material, rve.quaternions, phase, num)
    o = oracle_lib.OracleSpectralBasic(rve.cells, rve.size, rve.material, rve.quaternions, phase, num, threads=8)
    sg = run_load_cases(g, lcs)
    so = run_load_cases(o, lcs)
    assert len(sg) == len(so) == 60
    assert [s.iterations for s in sg] == [s.iterations for s in so]
    for a, b in zip(sg, so):
        assert rel(a.P_av, b.P_av) < 1e-9, a.inc
    for name in ('P', 'F', 'F_p', 'L_p', 'xi_sl', 'gamma_sl', 'O'):
        assert rel(g.get_field(name), o.get_field(name)) < 1e-9, name
    for a, b in zip(g.get_coords(), o.get_coords()):
        assert rel(a, b) < 1e-9
    g.close()


def test_grid64_fcc_mixed_against_fp64(gpu, oracle_lib):
    rve, phase, lcs, num = workloads.make('grid64_fcc_200g')
    runs = {}
    for precision in ('fp64', 'mixed'):
        g = SpectralBasic(rve.cells, rve.size, rve.material, rve.quaternions, phase, num, precision=precision)
        runs[precision] = run_load_cases(g, lcs)
        g.close()
    assert len(runs['fp64']) == len(runs['mixed']) == 100
    errs = [rel(m.P_av, f.P_av) for m, f in zip(runs['mixed'], runs['fp64'])]
    assert max(errs) < 1e-5
    o = oracle_lib.OracleSpectralBasic(rve.cells, rve.size, rve.material, rve.quaternions, phase, num, threads=8)
    so = run_load_cases(o, lcs, max_increments=2)
    for a, b in zip(runs['fp64'][:2], so):
        assert a.iterations == b.iterations
        assert rel(a.P_av, b.P_av) < 1e-9
