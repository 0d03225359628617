"""The batched workload: many independent RVEs of uneven size on one GPU (damask_b200/batch.py)."""
import numpy as np
import pytest

from damask_b200 import workloads

from conftest import rel


def test_batched_jobs_generator():
    jobs = workloads.batched_jobs(40, seed=4)
    edges = {j[0].cells[0] for j in jobs}
    assert edges <= {8, 12, 16, 24, 32} and len(edges) >= 4
    assert all(j[0].cells == (j[0].cells[0],) * 3 for j in jobs)
    assert all(5 <= len(j[0].quaternions) <= 100 for j in jobs)
    kinds = {('shear' if j[2][0].stress_type is None else 'tension') for j in jobs}
    assert kinds == {'shear', 'tension'}
    for j in jobs:
        lc = j[2][0]
        assert lc.N == 40 and lc.t == 40.0
        assert abs(np.linalg.norm(lc.q_rot) - 1.0) < 1e-12
    again = workloads.batched_jobs(40, seed=4)
    assert all(np.array_equal(a[0].material, b[0].material) for a, b in zip(jobs, again))


@pytest.mark.gpu
def test_batch_equals_standalone_runs(gpu):
    """RVEs run concurrently (3 host threads, own streams) give the results of standalone runs."""
    from damask_b200.batch import BatchRunner
    from damask_b200.grid import SpectralBasic, run_load_cases
    jobs = workloads.batched_jobs(6, seed=11)
    fields = {}

    def keep(k, s):
        fields[k] = s.get_field('P').copy()

    br = BatchRunner(jobs, threads=3, max_increments=3)
    br.run(on_finish=keep)
    for k, (rve, phase, lcs, num) in enumerate(jobs):
        s = SpectralBasic(rve.cells, rve.size, rve.material, rve.quaternions, phase, num)
        ref = run_load_cases(s, lcs, max_increments=3)
        assert [r.iterations for r in br.results[k]] == [r.iterations for r in ref]
        for a, b in zip(br.results[k], ref):
            assert rel(a.P_av, b.P_av) < 1e-12
        assert rel(fields[k], s.get_field('P')) < 1e-12
        assert br.updates[k] == sum(r.residual_evals for r in ref) * s.N
        s.close()
