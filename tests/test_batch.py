"""The batched workload: many independent RVEs of uneven size on one GPU (damask_b200/batch.py):
the library's batch (shared launches, dmk_batch_*) and the host-thread runner, each against
standalone runs of the same RVEs."""
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


def _standalone(job, n):
    from damask_b200.grid import SpectralBasic, run_load_cases
    rve, phase, lcs, num = job
    s = SpectralBasic(rve.cells, rve.size, rve.material, rve.quaternions, phase, num)
    stats = run_load_cases(s, lcs, max_increments=n)
    return s, stats


@pytest.mark.gpu
def test_device_batch_equals_standalone_runs(gpu):
    """Eight RVEs of four edge sizes in one batch of the library: per fixed-point iteration one CUDA
    graph evaluates the constitutive update of every active RVE, one cuFFT plan pair per edge size
    transforms them, batched kernels form aim, Gamma, convergence test and Anderson step.  The
    members differ in what a batch must keep per RVE: one runs the Richardson iteration, one the
    FWBW_difference derivative, one Anderson depth 12 (two chunks of inner products), one a
    shorter load case with twice the time step (it leaves the batch early, so later calls solve
    subsets).  Each RVE matches its standalone run: fixed-point iterations and residual
    evaluations per increment, constitutive counters, <P> per increment within 1e-12 and the fields
    within 1e-10: the batched cuFFT plans (9 x RVEs transforms per plan instead of 9) may round
    differently, and the fixed point carries last-bit differences of the residual into the fields
    (measured 1.1e-11 for the P field of a 32^3 member)."""
    from damask_b200.batch import DeviceBatch
    jobs = workloads.batched_jobs(8, seed=11)
    jobs[1][3].PETSc_options = '-snes_type nrichardson'
    jobs[2][3].derivative = 'FWBW_difference'
    jobs[3][3].anderson_m = 12
    rve, phase, _, num = jobs[4]
    jobs[4] = (rve, phase, workloads.tension_along([1.0, 2.0, 2.0], 4.0, 2), num)
    assert len({j[0].cells for j in jobs}) >= 3
    n = 4
    db = DeviceBatch(jobs, max_increments=n)
    db.run()
    st = db.stats()
    assert st['graphs'] >= st['iterations'] > 0 and st['passes'] > 0
    errs = {}
    for k, job in enumerate(jobs):
        s, ref = _standalone(job, n)
        got = db.results[k]
        assert len(got) == len(ref) == (2 if k == 4 else n)
        assert [r.iterations for r in got] == [r.iterations for r in ref], k
        assert [r.residual_evals for r in got] == [r.residual_evals for r in ref], k
        for a, b in zip(got, ref):
            assert rel(a.P_av, b.P_av) < 1e-12, (k, a.inc)
        g = db.solvers[k]
        assert np.array_equal(g.total_counters[:3], s.total_counters[:3]), (k, g.total_counters, s.total_counters)
        errs[k] = {name: rel(g.get_field(name), s.get_field(name)) for name in ('P', 'F', 'F_p', 'xi_sl', 'gamma_sl')}
        s.close()
    db.close()
    print('field differences batch vs standalone:', errs)
    assert max(max(e.values()) for e in errs.values()) < 1e-10, errs


@pytest.mark.gpu
def test_device_batch_native_loop_equals_python_loop(gpu):
    """The library's batched increment loop (dmk_batch_run) takes the steps of the Python loop over
    the same batch: the same converged increments, iteration counts and results, bit for bit."""
    from damask_b200.batch import DeviceBatch
    jobs = workloads.batched_jobs(5, seed=3)
    a = DeviceBatch(jobs, max_increments=3)
    a.run()
    b = DeviceBatch(jobs, max_increments=3)
    b.run_native()
    assert not b.failed
    for k in range(len(jobs)):
        key = lambda r: (r.inc, r.t, r.cutback_level, r.iterations, r.residual_evals)
        assert [key(r) for r in a.results[k]] == [key(r) for r in b.results[k]]
        for x, y in zip(a.results[k], b.results[k]):
            assert np.array_equal(x.P_av, y.P_av)
        assert np.array_equal(a.solvers[k].get_field('P'), b.solvers[k].get_field('P'))
        assert np.array_equal(a.solvers[k].get_coords()[1], b.solvers[k].get_coords()[1])
    assert a.updates == b.updates
    a.close()
    b.close()


@pytest.mark.gpu
def test_device_batch_cutbacks_match_standalone(gpu):
    """A member whose fixed point is capped at 8 iterations (-snes_max_it 8) fails increments and
    cuts back while the others go on: both batched loops (Python and dmk_batch_run) reproduce its
    standalone sequence of (sub)increments, time steps and cutback levels, and every member's
    results."""
    from damask_b200.batch import DeviceBatch
    jobs = workloads.batched_jobs(4, seed=7)
    jobs[1][3].PETSc_options = '-snes_max_it 8'
    n = 4
    refs = [_standalone(job, n) for job in jobs]
    assert any(r.cutback_level > 0 for r in refs[1][1]), 'the capped member must cut back'
    for native in (False, True):
        db = DeviceBatch(jobs, max_increments=n)
        db.run_native() if native else db.run()
        for k, (s, ref) in enumerate(refs):
            key = lambda r: (r.inc, round(r.t, 12), r.cutback_level, r.iterations, r.residual_evals)
            assert [key(r) for r in db.results[k]] == [key(r) for r in ref], (native, k)
            for a, b in zip(db.results[k], ref):
                assert rel(a.P_av, b.P_av) < 1e-12, (native, k, a.inc)
        db.close()
    for s, _ in refs:
        s.close()


@pytest.mark.gpu
def test_device_batch_mixed_form(gpu):
    """The mixed form in a batch: FP32 spectral passes (cuFFT R2C/C2R plans per edge size) with the
    FP64 correction pass of dmk_mech_solution for the members whose FP32 pass meets the tolerance.
    Against standalone mixed runs: equal fixed-point iteration counts and <P> within 1e-6 (the FP32
    transforms of the batched plans round differently from the per-RVE ones); against the batch's
    FP64 form: <P> within 1e-5, the mixed form's bound."""
    from damask_b200.batch import DeviceBatch
    from damask_b200.grid import SpectralBasic, run_load_cases
    jobs = workloads.batched_jobs(6, seed=5)
    n = 3
    mixed = DeviceBatch(jobs, max_increments=n, precision='mixed')
    mixed.run_native()
    fp64 = DeviceBatch(jobs, max_increments=n)
    fp64.run_native()
    worst = 0.0
    for k, (rve, phase, lcs, num) in enumerate(jobs):
        s = SpectralBasic(rve.cells, rve.size, rve.material, rve.quaternions, phase, num, precision='mixed')
        ref = run_load_cases(s, lcs, max_increments=n)
        got = mixed.results[k]
        assert [r.iterations for r in got] == [r.iterations for r in ref], k
        for a, b, c in zip(got, ref, fp64.results[k]):
            assert rel(a.P_av, b.P_av) < 1e-6, (k, a.inc)
            worst = max(worst, rel(a.P_av, c.P_av))
        s.close()
    assert worst < 1e-5
    print(f'mixed batch vs FP64 batch: <P> within {worst:.2e}')
    mixed.close()
    fp64.close()
