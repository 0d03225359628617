"""Host-side logic: input formats, the increment driver, the C-ABI surface, multi-rank reductions."""
import ctypes as C
import os
import re
import socket
from pathlib import Path

import numpy as np
import pytest
import yaml

from damask_b200 import _lib, config, workloads
from damask_b200.config import Numerics, Phase, parse_load
from damask_b200.grid import NotConverged, run_load_cases

ROOT = Path(__file__).resolve().parent.parent

LOAD = """
solver:
  mechanical: spectral_basic
loadstep:
  - boundary_conditions:
      mechanical:
        dot_F: [[1.0e-3, 0, 0], [0, x, 0], [0, 0, x]]
        P: [[x, x, x], [x, 0, x], [x, x, 0]]
    discretization: {t: 10, N: 40}
    f_out: 4
  - boundary_conditions:
      mechanical:
        F: [[1.1, 0, 0], [0, 1, 0], [0, 0, 1]]
        R: [0, 0, 1, 90]
    discretization: {t: 60, N: 60, r: 1.05}
    estimate_rate: false
    f_out: none
"""


def test_parse_load_cases():
    lc = parse_load(yaml.safe_load(LOAD))
    assert len(lc) == 2
    a, b = lc
    assert a.deformation_type == 'dot_F' and a.stress_type == 'P'
    assert a.deformation_mask[1, 1] and a.deformation_mask[2, 2] and not a.deformation_mask[0, 0]
    assert not a.stress_mask[1, 1] and a.stress_mask[0, 0]
    assert a.t == 10 and a.N == 40 and a.f_out == 4 and a.estimate_rate
    assert b.deformation_type == 'F' and b.stress_type is None and not b.estimate_rate
    assert b.f_out == 2 ** 31 - 1 and b.r == 1.05
    # R: 90 degrees about z, tRotation%fromAxisAngle with P = -1
    assert np.allclose(b.q_rot, [np.cos(np.pi / 4), 0, 0, np.sin(np.pi / 4)])
    bc = a.deformation_bc()
    assert bc.type == 2 and bc.values[0] == 1e-3 and bc.mask[4] == 1


def test_geometric_fraction_sums_to_one():
    for r in (1.0, 1.05, 0.9):
        assert abs(sum(config.geometric_fraction(r, i, 37) for i in range(1, 38)) - 1.0) < 1e-12


def test_numerics_from_yaml_and_validation():
    n = Numerics.from_dict({'solver': {'grid': {'N_cutback_max': 2, 'mechanical': {
        'N_iter_min': 2, 'eps_rel_div(P)': 1e-4, 'PETSc_options': '-snes_type nrichardson'}}},
        'phase': {'mechanical': {'N_iter_state_max': 10, 'plastic': {'N_iter_Lp_max': 20}}}})
    assert n.N_iter_min == 2 and n.eps_rel_div == 1e-4 and n.N_cutback_max == 2
    assert n.N_iter_state_max == 10 and n.N_iter_Lp_max == 20 and n.snes_type == 0
    s = n.to_struct()
    assert s.eps_rel_Li == n.eps_rel_Lp and s.snes_type == 0
    assert Numerics().snes_type == 1          # reference default -snes_type ngmres -> accelerated
    with pytest.raises(ValueError):
        Numerics(N_iter_min=5, N_iter_max=2).to_struct()
    with pytest.raises(ValueError):
        Numerics(PETSc_options='-snes_type newtonls').to_struct()
    # solver.grid.FFT keys (spectral_utilities.f90:176-223)
    n = Numerics.from_dict({'solver': {'grid': {'FFT': {'memory_efficient': False, 'FFTW_plan_mode': 'FFTW_PATIENT',
                                                        'derivative': 'FWBW_difference'}}}})
    assert not n.memory_efficient and n.FFTW_plan_mode == 'FFTW_PATIENT' and n.to_struct().derivative == 2
    for bad in ({'FFTW_plan_mode': 'FFTW_WISDOM_ONLY'}, {'divergence_correction': 'grid'}, {'derivative': 'FWBW'}):
        with pytest.raises(ValueError, match=list(bad)[0]):
            Numerics.from_dict({'solver': {'grid': {'FFT': bad}}}).to_struct()


def test_phase_rejects_unsupported():
    d = yaml.safe_load("""
lattice: cF
mechanical:
  elastic: {type: Hooke, C_11: 1e11, C_12: 6e10, C_44: 3e10}
  plastic: {type: dislotwin}
""")
    with pytest.raises(ValueError):
        Phase.from_dict(d)


class FakeSolver:
    """Scripted solver: fails the solutions listed in `fail_at` (call index)."""

    def __init__(self, fail_at):
        self.fail_at = set(fail_at)
        self.calls = []
        self.n = 0

    def forward(self, cutBack, guess, dt, dt_old, t_rem, lc):
        self.calls.append(('forward', cutBack, guess, round(dt, 12), round(dt_old, 12)))

    def materialpoint_forward(self):
        self.calls.append(('mp_forward',))

    def solution(self):
        from damask_b200.config import SolutionStruct
        s = SolutionStruct()
        s.converged = int(self.n not in self.fail_at)
        s.stagConverged = 1
        s.iterationsNeeded = 3
        s.residualEvals = 4
        self.n += 1
        return s

    def update_coords(self):
        pass


def test_driver_cutback_semantics():
    """DAMASK_grid.f90:288-460: a failed increment halves Delta_t (cutBack=.true., no
    materialpoint_forward), the substeps of the level complete it, and the next
    increment starts one cutback level lower."""
    lc = workloads.tension_x(4.0, 4)
    s = FakeSolver(fail_at=[1])
    stats = run_load_cases(s, lc, max_increments=3)
    forwards = [c for c in s.calls if c[0] == 'forward']
    assert forwards[0] == ('forward', False, True, 1.0, 1.0)      # inc 1, guess from estimate_rate
    assert forwards[1] == ('forward', False, True, 1.0, 1.0)      # inc 2 first try
    assert forwards[2] == ('forward', True, True, 0.5, 1.0)       # cut back: dt/2, no mp_forward
    assert forwards[3] == ('forward', False, True, 0.5, 0.5)      # second substep
    assert forwards[4] == ('forward', False, True, 1.0, 0.5)      # inc 3 back at level 0
    assert [st.t for st in stats] == [1.0, 1.5, 2.0, 3.0]
    assert sum(1 for c in s.calls if c[0] == 'mp_forward') == 4


def test_driver_restart_skips_computed_increments():
    """DAMASK_grid.f90:301-303: increments up to the restart increment only advance the
    time; the first computed increment then starts with guess = .true. and the previous
    increment's Delta_t."""
    lc = workloads.tension_x(4.0, 4)
    s = FakeSolver(fail_at=[])
    stats = run_load_cases(s, lc, restart_inc=2)
    forwards = [c for c in s.calls if c[0] == 'forward']
    assert len(forwards) == 2 and s.n == 2
    assert forwards[0] == ('forward', False, True, 1.0, 1.0)
    assert [st.inc for st in stats] == [3, 4] and [st.t for st in stats] == [3.0, 4.0]


def test_driver_gives_up_after_max_cutbacks():
    s = FakeSolver(fail_at=range(1, 100))
    with pytest.raises(NotConverged):
        run_load_cases(s, workloads.tension_x(4.0, 4), N_cutback_max=3)
    assert s.n == 5          # first increment + 4 tries of the second (levels 0..3)


def test_library_exports_every_declared_symbol():
    header = (ROOT / 'include' / 'damask_b200.h').read_text()
    names = set(re.findall(r'\b(dmk_[A-Za-z0-9_]+)\s*\(', header))
    assert len(names) >= 20
    lib = C.CDLL(str(_lib.LIB_PATH))
    missing = [n for n in sorted(names) if not hasattr(lib, n)]
    assert not missing, missing
    assert set(_lib.EXPORTS) <= names


def test_product_path_has_no_fallback(monkeypatch, tmp_path):
    """Without the CUDA library the product raises instead of computing elsewhere."""
    monkeypatch.setattr(_lib, '_lib', None)
    with pytest.raises(RuntimeError, match='no CPU fallback'):
        _lib.load(tmp_path / 'missing.so')


def _free_port():
    s = socket.socket()
    s.bind(('127.0.0.1', 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank_main(rank, world, port, q):
    os.environ.update(MASTER_ADDR='127.0.0.1', MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import datetime
    import sys
    import torch.distributed as dist
    sys.path.insert(0, str(ROOT))
    import bench
    dist.init_process_group('gloo', rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    bench.barrier(world)
    mx = bench.allreduce_max(10.0 + rank, world)
    sm = bench.allreduce_sum(100.0 * (rank + 1), world)
    dist.destroy_process_group()
    q.put((rank, mx, sm))


def test_replica_reductions_two_ranks():
    """bench.py reports updates summed over replicas and the time of the slowest replica."""
    import multiprocessing as mp
    ctx = mp.get_context('spawn')
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
    assert res == [(0, 11.0, 300.0), (1, 11.0, 300.0)]


def test_plugin_object_interface():
    """SpectralBasic (GPU) and the oracle offer the plugin procedures the driver calls and
    the accessors the tests use."""
    from damask_b200.grid import SpectralBasic
    from oracle.oracle import OracleSpectralBasic
    common = ('forward', 'solution', 'materialpoint_forward', 'update_coords', 'get_field', 'set_field',
              'aims', 'counters', 'constitutive_response', 'gamma_convolution', 'divergence_rms', 'dPdF', 'close')
    for cls in (SpectralBasic, OracleSpectralBasic):
        missing = [m for m in common if not callable(getattr(cls, m, None))]
        assert not missing, (cls.__name__, missing)
    for m in ('restart_write', 'restart_read', 'timer_start', 'timer_stop', 'launches', 'iteration_counts'):
        assert callable(getattr(SpectralBasic, m, None)), m


def test_sta_file(oracle_lib, tmp_path):
    """The statistics table of the driver (DAMASK_grid.f90:268-278, 394-395): header, one row per
    converged increment, appended after a restart."""
    from damask_b200 import synthetic, workloads
    from damask_b200.grid import STA_HEADER, read_sta, run_load_cases
    rve = synthetic.voronoi_rve((4, 4, 4), workloads.SIZE_1MM, 3, 0)
    o = oracle_lib.OracleSpectralBasic(rve.cells, rve.size, rve.material, rve.quaternions, workloads.fcc_al(),
                                       workloads.numerics_default(), threads=1)
    sta = tmp_path / 'job.sta'
    stats = run_load_cases(o, workloads.tension_x(60.0, 60), max_increments=3, sta=sta)
    o.close()
    assert sta.read_text().splitlines()[0] == STA_HEADER
    rows = read_sta(sta)
    assert [r[0] for r in rows] == [s.inc for s in stats] == [1, 2, 3]
    assert [r[4] for r in rows] == [s.iterations for s in stats] and all(r[3] for r in rows)
    assert abs(rows[-1][1] - 3.0) < 1e-12


def test_driver_requests_match_step():
    """IncrementDriver.step_requests (the generator a batch drives) takes the same steps as
    step(): forward / materialpoint_forward calls, cutbacks and statistics."""
    from damask_b200.grid import IncrementDriver
    lc = workloads.tension_x(4.0, 4)
    a = FakeSolver(fail_at=[1, 4])
    ref = run_load_cases(a, lc)
    b = FakeSolver(fail_at=[1, 4])
    drv = IncrementDriver(b, lc)
    got = []
    while not drv.done:
        gen = drv.step_requests()
        try:
            gen.send(None)
            while True:
                gen.send(b.solution())
        except StopIteration as stop:
            got.extend(stop.value)
    assert a.calls == b.calls
    assert [(s.inc, s.t, s.cutback_level) for s in got] == [(s.inc, s.t, s.cutback_level) for s in ref]


def test_device_batch_scheduling():
    """DeviceBatch.run with the batched solve replaced by scripted solvers: jobs with different
    cutbacks and lengths fall out of step, each request goes to its own job, every job runs its
    increments, and the jobs' call sequences equal their standalone runs."""
    from damask_b200.batch import DeviceBatch
    from damask_b200.grid import IncrementDriver
    loads = [workloads.tension_x(4.0, 4), workloads.tension_x(2.0, 2), workloads.tension_x(4.0, 4)]
    fails = [[1], [], [0, 3]]
    db = object.__new__(DeviceBatch)
    db.jobs = loads
    db.max_increments = None
    fakes = [FakeSolver(f) for f in fails]
    db.drivers = [IncrementDriver(s, lc) for s, lc in zip(fakes, loads)]
    db.results = [[] for _ in loads]
    db.batch_calls = 0
    db._gens = [None] * len(loads)
    sizes = []

    def solve(waiting):
        sizes.append(len(waiting))
        return [fakes[k].solution() for k in waiting]

    db.run(solve=solve)
    for k, (lc, f) in enumerate(zip(loads, fails)):
        s = FakeSolver(f)
        ref = run_load_cases(s, lc)
        assert fakes[k].calls == s.calls
        assert [(r.inc, r.t) for r in db.results[k]] == [(r.inc, r.t) for r in ref]
    assert db.batch_calls == len(sizes) and sizes[0] == 3 and sizes[-1] < 3
