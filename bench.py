#!/usr/bin/env python
"""Benchmark of DAMASK's grid mechanical hot path on B200.

Metric: material-point updates/s (one update = one constitutive evaluation of one
voxel inside one residual evaluation of the basic spectral scheme) on the 256^3
bcc RVE (2000 Voronoi grains, seed 3, phenopowerlaw N_sl [12,12], uniaxial
tension dot_F_xx = 1e-3/s to 10 % in 100 increments).  One step = one load
increment (forward, the fixed-point solve to convergence, materialpoint forward).

  python bench.py [--gpus N --steps K --warmup W]     # this implementation
  python bench.py --impl reference ...                  # CPU restatement (oracle) on host cores

Multi-GPU (torchrun, one rank per GPU): the path is run as independent replicas,
one RVE per GPU, with no collective in the data path ("weak" scaling).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

import numpy as np  # noqa: E402

WORKLOAD = 'grid256_bcc24_2000g'
METRIC = 'material-point updates/s at 256^3: mixed vs FP64 GPU, P within 1e-5 of FP64'
FP64_NOMINAL_TFLOPS = 37.0   # B200 FP64 (CUDA cores), datasheet figure


def constitutive_flops(ns: int, newton: float, state: float, updates: float) -> float:
    """Static FP64 FLOP count of the constitutive passes (FMA = 2):
    per residual evaluation (Newton iteration) 264 + 56 Ns; per Newton step (Woodbury
    6x6 system: assembly, QR, back-substitution; one per non-final Newton iteration)
    567 + 135 Ns; per state iteration (stress start/finish, hardening, damped update)
    455 + 86 Ns; per substep start (kinetics and hardening) 89 Ns."""
    steps = max(newton - state, 0.0)
    return newton * (264 + 56 * ns) + steps * (567 + 135 * ns) + state * (455 + 86 * ns) + updates * (89 * ns)


# DRAM bytes that one stress and one control launch move per voxel of a full pass, by slip-system
# count, from the ncu captures summarised in profiles/constitutive_passes_64cubed_bcc24.txt and
# _bcc48.txt (two passes of a 65 536-voxel chunk each; 24 systems: stress 568 B, control 2 114 B;
# 48 systems: stress 794 B, control 4 840 B); a material-point update runs one such pass per state
# iteration
TRAFFIC_BYTES_PER_PASS = {24: 2682, 48: 5634}

# the 48-system RVE's window inside the default bench line (5.7 s per increment at 256^3)
BCC48_WARMUP, BCC48_STEPS = 3, 3
# timed increments of the CPU baseline leg (after the headline's warm-up window)
CPU_STEPS = 3


def bc_bytes() -> int:
    """Host bytes passed to the device per increment: two boundary-condition structs and the rotation."""
    import ctypes
    from damask_b200.config import BCStruct
    return 2 * ctypes.sizeof(BCStruct) + 4 * 8


def constitutive_bytes(ns: int) -> int:
    """Algorithmic HBM bytes per update of the constitutive kernel (Anderson form):
    reads F, F0, Fp0, Lp (9 doubles each), S0 (6), state0 (2 Ns); writes F, P, Fp, Lp, Fe
    (9 each), S (6), state (2 Ns)."""
    return 8 * (4 * 9 + 6 + 2 * ns) + 8 * (5 * 9 + 6 + 2 * ns)


class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons during the timed region."""

    FIELDS = ('clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,'
              'clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,'
              'clocks_event_reasons.sw_power_cap')

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.proc = None
        self.lines: list[str] = []
        self._t = None

    def start(self):
        try:
            self.proc = subprocess.Popen(['nvidia-smi', '-i', str(self.gpu), f'--query-gpu={self.FIELDS}',
                                          '--format=csv,noheader,nounits', '-lms', '200'],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        self._t = threading.Thread(target=self._read, daemon=True)
        self._t.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {'sm_mhz': None, 'sm_max_mhz': None, 'reasons': ['nvidia-smi unavailable']}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self._t:
            self._t.join(timeout=2)
        sm, smax, reasons = [], [], set()
        names = ['hw_slowdown', 'hw_thermal_slowdown', 'sw_thermal_slowdown', 'sw_power_cap']
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(',')]
            if len(parts) < 7:
                continue
            try:
                sm.append(float(parts[0]))
                smax.append(float(parts[1]))
            except ValueError:
                continue
            for n, v in zip(names, parts[3:7]):
                if v.lower().startswith('active'):
                    reasons.add(n)
        return {'sm_mhz': statistics.median(sm) if sm else None, 'sm_max_mhz': max(smax) if smax else None,
                'reasons': sorted(reasons), 'samples': len(sm)}


def dist_setup():
    world = int(os.environ.get('WORLD_SIZE', '1'))
    rank = int(os.environ.get('RANK', '0'))
    local = int(os.environ.get('LOCAL_RANK', '0'))
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group('nccl', timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device('cuda', local))
    return world, rank, local


def _allreduce(x: float, world: int, op: str) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = 'cpu' if dist.get_backend() == 'gloo' else 'cuda'
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX if op == 'max' else dist.ReduceOp.SUM)
    return float(t.item())


def allreduce_max(x: float, world: int) -> float:
    """Maximum over ranks (the timed region of the slowest replica)."""
    return _allreduce(x, world, 'max')


def allreduce_sum(x: float, world: int) -> float:
    """Sum over ranks (updates of all replicas)."""
    return _allreduce(x, world, 'sum')


def barrier(world: int):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def measure_fp64_peak(device: int) -> tuple[float, str]:
    """FP64 FMA throughput of this GPU from the library's probe (dmk_fp64_peak), outside the
    timed region; the datasheet figure if the probe fails."""
    import ctypes as C
    from damask_b200 import _lib
    out = C.c_double()
    if _lib.load().dmk_fp64_peak(device, C.byref(out)) == 0 and out.value > 0:
        return out.value, 'measured (FP64 FMA probe, dmk_fp64_peak)'
    return FP64_NOMINAL_TFLOPS, 'datasheet (probe failed)'


def load_peaks() -> dict:
    p = ROOT / 'MEASURED_PEAKS.json'
    if p.exists():
        d = json.loads(p.read_text())
        return {'hbm_gbs': float(d['hbm_gbs']), 'source': 'measured'}
    return {'hbm_gbs': 6650.0, 'source': 'fallback'}


def run_gpu(precision: str, steps: int, warmup: int, world: int, rank: int, local: int, cells=None,
            solver_name: str = 'spectral_basic', workload: str = WORKLOAD, derivative: str = 'continuous') -> dict:
    from damask_b200 import workloads
    from damask_b200.grid import IncrementDriver, SpectralBasic

    import torch
    rve, phase, lcs, num = workloads.make(workload, cells)
    num.solver = solver_name
    num.derivative = derivative
    free0 = torch.cuda.mem_get_info(local)[0]
    solver = SpectralBasic(rve.cells, rve.size, rve.material, rve.quaternions, phase, num, precision=precision,
                           device=local)
    device_gb = (free0 - torch.cuda.mem_get_info(local)[0]) / 1e9
    drv = IncrementDriver(solver, lcs)
    p_av = []

    def one_step():
        c0, t0 = solver.total_counters.copy(), solver.total_ms.copy()
        recs = drv.step()
        c = solver.total_counters - c0
        tm = solver.total_ms - t0
        p_av.extend(r.P_av for r in recs)
        return recs, c, tm

    for _ in range(warmup - 1):
        one_step()
    # the last warm-up increment: the autotuner picks the stress-kernel variant and the voxel-chunk
    # count between its forward and its solution (results unchanged; basic scheme only)
    tuning = None
    if solver_name == 'spectral_basic':
        gen = drv.step_requests()
        try:
            gen.send(None)
            try:
                tuning = solver.autotune(reps=2)
            except Exception as e:                   # not enough free memory for the state copy
                tuning = {'skipped': str(e)}
            while True:
                gen.send(solver.solution())
        except StopIteration as stop:
            p_av.extend(r.P_av for r in stop.value)
    else:
        one_step()
    # timed region: inputs resident in HBM, device time on the solver's stream.  Each step is
    # timed twice from the same increment: the increment itself (value) and, end to end through
    # the public API, the increment plus the read-back of its stress field P into pinned host
    # memory (e2e; the boundary conditions enter from host memory inside the increment).
    pinned = torch.empty((solver.N, 9), dtype=torch.float64, pin_memory=True).numpy()
    barrier(world)
    clocks = ClockSampler(local)
    clocks.start()
    launches0 = solver.launches()
    upd = newton = state = evals = 0
    const_ms = ms = ms_e2e = 0.0
    for _ in range(steps):
        solver.timer_start()
        recs, c, tm = one_step()
        ms_step = solver.timer_stop()
        solver.timer_start()
        solver.get_field('P', out=pinned)
        ms_copy = solver.timer_stop()
        ms += ms_step
        ms_e2e += ms_step + ms_copy
        upd += c[0]
        state += c[1]
        newton += c[2]
        evals += c[3]
        const_ms += tm[0]
    launches = solver.launches() - launches0
    clk = clocks.stop()
    barrier(world)
    upd_e2e = upd
    out = {'updates': upd, 'ms': ms, 'newton': newton, 'state': state, 'evals': evals, 'const_ms': const_ms,
           'launches': launches, 'clocks': clk, 'updates_e2e': upd_e2e, 'ms_e2e': ms_e2e, 'N': solver.N,
           'ns': phase.n_slip, 'p_av': p_av, 'd2h_bytes': solver.N * 9 * 8, 'device_gb': device_gb,
           'tuning': tuning}
    solver.close()
    return out


def cpu_sample(steps: int = 5, warmup: int = 5, threads: int | None = None, workload: str = WORKLOAD) -> dict:
    """The CPU restatement on the same material and load, on a 48^3 cut of the workload at its
    grain density (13 grains, seed 3): `warmup` untimed increments, then `steps` timed ones
    (the increment window of the GPU figures: after the same warm-up, the same load)."""
    from damask_b200 import workloads
    from damask_b200.grid import IncrementDriver
    from damask_b200.synthetic import voronoi_rve
    from oracle.oracle import OracleSpectralBasic

    threads = threads or os.cpu_count() or 1
    cells = (48, 48, 48)
    rve = voronoi_rve(cells, workloads.SIZE_1MM, 13, 3)
    phase = workloads.PHASES[workloads.WORKLOADS[workload][3]]()
    lcs = workloads.tension_x(100.0, 100)
    o = OracleSpectralBasic(rve.cells, rve.size, rve.material, rve.quaternions, phase, workloads.numerics_default(),
                            threads=threads)
    drv = IncrementDriver(o, lcs)
    for _ in range(warmup):
        drv.step()
    t0 = time.perf_counter()
    upd = 0
    for _ in range(steps):
        for r in drv.step():
            upd += r.residual_evals * o.N
    dt = time.perf_counter() - t0
    o.close()
    return {'value': upd / dt, 'seconds': dt, 'cores': threads, 'updates': upd,
            'warmup': warmup, 'increments_timed': f'{warmup + 1}..{warmup + steps}',
            'sample': f'oracle (C++ FP64, OpenMP, {threads} threads) on a 48^3 RVE, 13 grains, same '
                      f'{phase.n_slip}-system material and tension load, increments {warmup + 1}..{warmup + steps} '
                      f'after {warmup} untimed warm-up increments'}


def _json_default(o):
    if isinstance(o, np.integer):
        return int(o)
    if isinstance(o, np.floating):
        return float(o)
    raise TypeError(type(o))


def flop_sample(increments: int) -> None:
    """The constitutive counters and the static FP64 FLOP count of the first increments of a 32^3 cut of
    the bcc-24 workload (FP64), printed as one JSON line: the run that an ncu count of the FP64
    instructions of the constitutive kernels checks the static model against."""
    from damask_b200 import workloads
    from damask_b200.grid import IncrementDriver, SpectralBasic
    rve, phase, lcs, num = workloads.make_cut(WORKLOAD, (32, 32, 32))
    s = SpectralBasic(rve.cells, rve.size, rve.material, rve.quaternions, phase, num, precision='fp64')
    drv = IncrementDriver(s, lcs)
    for _ in range(increments):
        drv.step()
    c = s.total_counters
    print(json.dumps({'workload': f'{WORKLOAD} 32^3 cut', 'increments': increments, 'updates': int(c[0]),
                      'state_iterations': int(c[1]), 'newton_iterations': int(c[2]), 'residual_evals': int(c[3]),
                      'static_fp64_flop': float(constitutive_flops(phase.n_slip, c[2], c[1], c[0]))},
                     default=_json_default), flush=True)
    s.close()


def _timed_run(solver, lcs, n=None) -> dict:
    """Wall time, device time and counters of the first n increments (all: None) of a solver."""
    from damask_b200.grid import run_load_cases
    t0 = time.perf_counter()
    st = run_load_cases(solver, lcs, max_increments=n)
    wall = time.perf_counter() - t0
    upd = sum(r.residual_evals for r in st) * solver.N
    out = {'increments': len(st), 'wall_s': wall, 's_per_increment': wall / max(1, len(st)), 'updates': upd,
           'updates_per_s': upd / wall, 'iterations': [r.iterations for r in st][:8]}
    if hasattr(solver, 'total_ms'):
        dev = float(np.sum(solver.total_ms)) * 1e-3
        out.update({'device_s': dev, 'device_updates_per_s': upd / dev if dev > 0 else None})
    return out


def config_times() -> None:
    """Times of the specified configurations other than the headline, one JSON line each: the
    16^3 fcc run (C0, 60 increments) and the 64^3 fcc run (C1, 100 increments) in FP64 and mixed on
    the GPU, with the oracle on all host cores (C0 whole, C1 its first 3 increments); the batched
    workload's first 16 RVEs on the oracle (C2; the GPU figure is the bench line's `batched` key and
    `--batch 512`); the adjoint configuration (C3: 32^3, 50 grains, 50 increments, checkpoints every
    10) forward and gradient on the GPU, and 5 increments of its forward on the oracle."""
    from damask_b200 import workloads
    from damask_b200.adjoint import IncrementSequence, gradient_numerics, gradient_phase, theta_of
    from damask_b200.grid import SpectralBasic
    from oracle.oracle import OracleSpectralBasic
    threads = os.cpu_count() or 1

    def gpu(name, precision):
        rve, phase, lcs, num = workloads.make(name)
        s = SpectralBasic(rve.cells, rve.size, rve.material, rve.quaternions, phase, num, precision=precision)
        r = _timed_run(s, lcs)
        s.close()
        return r

    def cpu(name, n):
        rve, phase, lcs, num = workloads.make(name)
        o = OracleSpectralBasic(rve.cells, rve.size, rve.material, rve.quaternions, phase, num, threads=threads)
        r = _timed_run(o, lcs, n)
        o.close()
        return dict(r, cores=threads, kind='port')

    for cfg, name, n_cpu in (('C0', 'grid16_fcc_20g', None), ('C1', 'grid64_fcc_200g', 3)):
        line = {'config': cfg, 'workload': name, 'gpu_fp64': gpu(name, 'fp64'), 'gpu_mixed': gpu(name, 'mixed'),
                'cpu': cpu(name, n_cpu)}
        print(json.dumps(line, default=_json_default), flush=True)
    # C2 on the oracle: the first 16 RVEs of the batched workload one after the other, 5 increments each
    upd, wall = 0, 0.0
    for rve, phase, lcs, num in workloads.batched_jobs(BATCH_JOBS)[:16]:
        o = OracleSpectralBasic(rve.cells, rve.size, rve.material, rve.quaternions, phase, num, threads=threads)
        r = _timed_run(o, lcs, 5)
        o.close()
        upd += r['updates']
        wall += r['wall_s']
    print(json.dumps({'config': 'C2', 'workload': 'first 16 RVEs of batched512, increments 1..5 of each, in sequence',
                      'cpu': {'updates': upd, 'wall_s': wall, 'updates_per_s': upd / wall, 'cores': threads,
                              'kind': 'port'}}, default=_json_default), flush=True)
    rve, phase, lcs, num = workloads.make('grid32_fcc_50g')
    phase, num = gradient_phase(phase), gradient_numerics(num)
    seq = IncrementSequence(rve, phase, lcs, num, 50, k=10)
    theta = theta_of(phase)
    t0 = time.perf_counter()
    curve = seq.run(theta)
    t1 = time.perf_counter()
    seq.gradient(np.ones_like(curve))
    t2 = time.perf_counter()
    seq.close()
    o = OracleSpectralBasic(rve.cells, rve.size, rve.material, rve.quaternions, phase, num, threads=threads)
    c = _timed_run(o, lcs, 5)
    o.close()
    print(json.dumps({'config': 'C3', 'workload': 'grid32_fcc_50g, 50 increments, gradient numerics',
                      'gpu_forward_s': t1 - t0, 'gpu_gradient_s': t2 - t1,
                      'cpu_forward_5_increments': dict(c, cores=threads, kind='port')}, default=_json_default),
          flush=True)


BATCH_JOBS = 512                         # RVEs of the batched workload definition
BATCH_RVES, BATCH_INCREMENTS = 128, 10   # the bounded batched sample of the default bench line


def batch_sample(n_rves: int, increments: int, local: int = 0, precision: str = 'mixed') -> dict:
    """The batched workload's first n_rves RVEs (edges 8..32, 5..100 grains, random-axis tension or
    simple shear), their first `increments` increments, as one batch of the library (mixed form, as the
    workload is specified) driven by its C++ batched increment loop: updates/s over the wall time of the
    run (the increment loops included, context set-up not)."""
    from damask_b200 import workloads
    from damask_b200.batch import DeviceBatch
    jobs = workloads.batched_jobs(BATCH_JOBS)[:n_rves]
    voxels = sum(j[0].n_cells for j in jobs)
    t0 = time.perf_counter()
    db = DeviceBatch(jobs, max_increments=increments, device=local, precision=precision)
    setup = time.perf_counter() - t0
    clocks = ClockSampler(local)
    clocks.start()
    seconds = db.run_native()
    clk = clocks.stop()
    if db.failed:
        raise RuntimeError(f'batched RVEs {db.failed} did not converge')
    st = db.stats()
    updates = sum(db.updates)
    incs = sum(len(r) for r in db.results)
    out = {'workload': f'first {n_rves} RVEs of batched{BATCH_JOBS} (edges {{8,12,16,24,32}}, 5..100 grains, '
                       'random-axis tension or simple shear 1e-3/s), '
                       + (f'increments 1..{increments} of each' if increments < 40 else 'all 40 increments'),
           'value': updates / seconds, 'unit': 'updates/s', 'seconds': seconds, 'setup_seconds': setup,
           'rves': n_rves, 'voxels': voxels, 'increments': incs, 'updates': updates,
           'batched_solutions': st['solutions'], 'graphs': st['graphs'], 'passes': st['passes'],
           'fixed_point_iterations': st['iterations'],
           'dtype': 'f64 constitutive, f32 spectral (mixed)' if precision == 'mixed' else 'f64', 'clocks': clk,
           'how': 'dmk_batch_run: one dmk_batch_solution per round of solution requests; per fixed-point '
                  'iteration one CUDA graph (constitutive passes of all active RVEs, device-side while loop), '
                  'one cuFFT plan pair per edge size, batched aim / Gamma / convergence / Anderson kernels'}
    db.close()
    return out


def run_batch(args) -> None:
    """Batched workload: independent RVEs (edges 8..32, 5..100 grains, random-axis tension or
    simple shear, 40 increments to 4 %), all increments of every RVE.  Default: one batch of the
    library (FP64, shared launches); --batch-engine threads: one context per RVE on its own streams,
    host threads issue the RVEs concurrently (mixed precision)."""
    import torch
    from damask_b200 import workloads
    from damask_b200.batch import BatchRunner
    if args.batch_engine == 'device':
        torch.cuda.synchronize()
        b = batch_sample(args.batch, 40)
        line = {'metric': 'batched RVE material-point updates/s (wall clock of the increment loops)',
                'value': b['value'], 'unit': 'updates/s', 'n_gpus': 1, 'steps': b['increments'], 'warmup': 0,
                'ms_per_step': 1e3 * b['seconds'] / max(1, b['increments']), 'higher_is_better': True,
                'scaling': 'weak', 'vs_baseline': None, 'dtype': b['dtype'], 'data': 'synthetic',
                'config': {'workload': b['workload'], 'rves': args.batch, 'voxels': b['voxels'], 'engine': 'dmk_batch'},
                'batched': b, 'clocks': b['clocks']}
        print(json.dumps(line, default=_json_default), flush=True)
        return
    jobs = workloads.batched_jobs(args.batch)
    voxels = sum(j[0].n_cells for j in jobs)
    torch.cuda.synchronize()
    clocks = ClockSampler(int(os.environ.get('LOCAL_RANK', 0)))
    clocks.start()
    br = BatchRunner(jobs, threads=args.batch_threads, precision='mixed')
    seconds = br.run()
    clk = clocks.stop()
    updates = sum(br.updates)
    incs = sum(len(r) for r in br.results)
    line = {'metric': 'batched RVE material-point updates/s (wall clock incl. context setup)',
            'value': updates / seconds, 'unit': 'updates/s', 'n_gpus': 1, 'steps': incs, 'warmup': 0,
            'ms_per_step': 1e3 * seconds / max(1, incs), 'higher_is_better': True, 'scaling': 'weak',
            'vs_baseline': None, 'dtype': 'f64 constitutive, f32 spectral (mixed)', 'data': 'synthetic',
            'config': {'workload': f'batched{args.batch}: edges {{8,12,16,24,32}}, 5..100 grains, random-axis '
                                   'tension or simple shear 1e-3/s, 40 increments to 4 %',
                       'rves': args.batch, 'voxels': voxels, 'host_threads': args.batch_threads,
                       'increments': incs},
            'seconds': seconds, 'clocks': clk}
    print(json.dumps(line, default=_json_default), flush=True)


def measure(workload, steps, warmup, world, rank, local, cells, solver, derivative, precision) -> dict:
    """Both precisions of one workload over the same increment window; the figures of a bench line."""
    res = {}
    precs = ('mixed', 'fp64') if precision == 'both' else (precision,)
    for prec in precs:
        res[prec] = run_gpu(prec, steps, warmup, world, rank, local, cells, solver, workload, derivative)
    mx = res.get('mixed', res.get('fp64'))
    fp = res.get('fp64', mx)
    ms_max = allreduce_max(mx['ms'], world)
    value = allreduce_sum(mx['updates'], world) / (ms_max * 1e-3)
    fp_ms = allreduce_max(fp['ms'], world)
    fp_value = allreduce_sum(fp['updates'], world) / (fp_ms * 1e-3)
    e2e_ms = allreduce_max(mx['ms_e2e'], world)
    e2e_value = allreduce_sum(mx['updates_e2e'], world) / (e2e_ms * 1e-3)
    # agreement of the volume-averaged stress of the mixed and FP64 runs, increment by increment
    rel = [float(np.abs(a - b).max() / np.abs(b).max()) for a, b in zip(mx['p_av'], fp['p_av'])]
    peaks = load_peaks()
    fp64_peak, fp64_source = measure_fp64_peak(local)
    ns = mx['ns']
    bpu = constitutive_bytes(ns)
    avg_launch_ms = mx['const_ms'] / max(1, mx['evals'])
    achieved_gbs = bpu * mx['N'] / (avg_launch_ms * 1e-3) / 1e9
    flops = constitutive_flops(ns, mx['newton'], mx['state'], mx['updates'])
    fp64_tflops = flops / (mx['const_ms'] * 1e-3) / 1e12
    per_pass = TRAFFIC_BYTES_PER_PASS.get(ns)
    traffic = per_pass * mx['state'] / max(1, mx['updates']) if per_pass else None
    roofline = {
        'bound': 'fp64',
        'kernel': 'constitutive update (begin + stress/control pass kernels), one evaluation of all voxels',
        'achieved': fp64_tflops, 'peak': fp64_peak, 'unit': 'TFLOP/s', 'frac': fp64_tflops / fp64_peak,
        'peak_source': fp64_source, 'nominal_peak': FP64_NOMINAL_TFLOPS,
        'flops_per_update': flops / max(1, mx['updates']),
        'flop_source': 'static FP64 count of the kernels times the counted Newton / state iterations',
        'traffic': traffic * mx['N'] if traffic else None,
        'traffic_source': f'ncu DRAM bytes of a stress and a control launch per voxel and pass at 64^3 ({ns} systems), '
                          'times the passes (state iterations) per update and the voxels of one evaluation; '
                          'the begin kernel is not included',
        'avg_launch_ms': avg_launch_ms,
        'hbm': {'achieved': achieved_gbs, 'peak': peaks['hbm_gbs'], 'unit': 'GB/s', 'frac': achieved_gbs / peaks['hbm_gbs'],
                'peak_source': peaks['source'], 'bytes_per_update': bpu},
        'fp64': {'achieved': fp64_tflops, 'peak': fp64_peak, 'unit': 'TFLOP/s', 'frac': fp64_tflops / fp64_peak},
    }
    return {'mixed': mx, 'fp64_raw': fp, 'value': value, 'ms_per_step': ms_max / steps,
            'fp64': {'value': fp_value, 'unit': 'updates/s', 'ms_per_step': fp_ms / steps},
            's_per_increment': {'mixed': ms_max / steps * 1e-3, 'fp64': fp_ms / steps * 1e-3},
            'mixed_over_fp64': value / fp_value, 'P_av_rel_err': max(rel) if rel else None,
            'roofline': roofline,
            'e2e': {'value': e2e_value, 'unit': 'updates/s', 'h2d_bytes_per_step': bc_bytes(),
                    'd2h_bytes_per_step': mx['d2h_bytes'],
                    'how': 'the same increments as value: each increment plus the read-back of its P field into '
                           'pinned host memory through dmk_get_field'},
            'iterations': {'newton_per_update': mx['newton'] / max(1, mx['updates']),
                           'state_per_update': mx['state'] / max(1, mx['updates']),
                           'residual_evals': mx['evals']}}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--gpus', type=int, default=1)
    ap.add_argument('--steps', type=int, default=3)
    ap.add_argument('--warmup', type=int, default=3)
    ap.add_argument('--impl', choices=['ours', 'reference'], default='ours')
    ap.add_argument('--cells', type=str, default=None, help='override grid (testing only)')
    ap.add_argument('--no-cpu-baseline', action='store_true')
    ap.add_argument('--no-bcc48', action='store_true', help='leave out the 48-system key of the bench line')
    ap.add_argument('--precision', choices=['both', 'mixed', 'fp64'], default='both',
                    help='run one precision only (profiling); the bench line needs both')
    ap.add_argument('--solver', choices=['spectral_basic', 'spectral_polarization'], default='spectral_basic',
                    help='grid solver (the bench line is defined for spectral_basic)')
    ap.add_argument('--batch', type=int, default=0,
                    help='measure the batched workload instead: this many independent RVEs (512 in the '
                         'workload definition), one JSON line of its own')
    ap.add_argument('--batch-threads', type=int, default=48)
    ap.add_argument('--batch-engine', choices=['device', 'threads'], default='device',
                    help='--batch: one batch of the library (shared launches) or host threads over contexts')
    ap.add_argument('--no-batched', action='store_true', help='leave out the batched key of the bench line')
    ap.add_argument('--configs', action='store_true', help='time the other specified configurations and exit')
    ap.add_argument('--flop-sample', type=int, default=0,
                    help='print the counters and static FLOP count of this many increments of a 32^3 cut and exit')
    ap.add_argument('--derivative', choices=['continuous', 'central_difference', 'FWBW_difference'],
                    default='continuous', help='solver.grid.FFT.derivative (testing and profiling only)')
    ap.add_argument('--workload', choices=['grid256_bcc24_2000g', 'grid256_bcc48_2000g'], default=WORKLOAD,
                    help='the headline bcc N_sl [12,12] RVE, or the same RVE with all three cI families (48 systems)')
    args = ap.parse_args()
    if args.flop_sample:
        return flop_sample(args.flop_sample)
    if args.configs:
        return config_times()
    if args.batch:
        return run_batch(args)
    world, rank, local = dist_setup()
    warmup = max(3, args.warmup)
    cells = tuple(int(x) for x in args.cells.split(',')) if args.cells else None

    if args.impl == 'reference':
        if rank != 0:
            return
        # the same increment window as this implementation's timed region: W untimed warm-up
        # increments, then K timed ones, on the bounded 48^3 sample
        s = cpu_sample(steps=max(1, args.steps), warmup=warmup, workload=args.workload)
        line = {'metric': METRIC, 'value': s['value'], 'unit': 'updates/s', 'n_gpus': args.gpus, 'steps': args.steps,
                'warmup': warmup, 'ms_per_step': 1e3 * s['seconds'] / max(1, args.steps), 'higher_is_better': True,
                'scaling': 'weak', 'vs_baseline': None, 'dtype': 'f64', 'data': 'synthetic',
                'impl': 'reference', 'warmup_match': True,
                'config': {'workload': f'{args.workload}: bcc phenopowerlaw RVE, tension 1e-3/s (48^3 bounded '
                                       'sample of the 256^3/2000-grain workload)', 'solver': 'Anderson fixed point',
                           'increments_timed': s['increments_timed']},
                'cpu_baseline': {'value': s['value'], 'unit': 'updates/s', 'cores': s['cores'], 'kind': 'port',
                                 'sample': s['sample']},
                'e2e': {'value': s['value'], 'unit': 'updates/s', 'h2d_bytes_per_step': 0, 'd2h_bytes_per_step': 0}}
        print(json.dumps(line, default=_json_default), flush=True)
        return

    headline = measure(args.workload, args.steps, warmup, world, rank, local, cells, args.solver, args.derivative,
                       args.precision)
    # the 48-system RVE of the same grid (all three cI families), on a short window
    b48 = None
    if args.workload == WORKLOAD and cells is None and not args.no_bcc48 and args.precision == 'both':
        b48 = measure('grid256_bcc48_2000g', BCC48_STEPS, BCC48_WARMUP, world, rank, local, None, args.solver,
                      args.derivative, 'both')
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    if rank != 0:
        return
    batched = None
    if world == 1 and cells is None and not args.no_batched:
        batched = batch_sample(BATCH_RVES, BATCH_INCREMENTS, local)
    cpu = None
    if world == 1 and not args.no_cpu_baseline:
        s = cpu_sample(steps=CPU_STEPS, warmup=warmup, workload=args.workload)
        cpu = {'value': s['value'], 'unit': 'updates/s', 'cores': s['cores'], 'kind': 'port', 'sample': s['sample']}
    mx = headline['mixed']
    line = {
        'metric': METRIC, 'value': headline['value'], 'unit': 'updates/s', 'n_gpus': world, 'steps': args.steps,
        'warmup': warmup, 'ms_per_step': headline['ms_per_step'], 'higher_is_better': True, 'scaling': 'weak',
        'vs_baseline': None, 'dtype': 'f64 constitutive, f32 spectral (mixed)', 'data': 'synthetic',
        'config': {'workload': f'{args.workload}: 256^3 grid, 2000 Voronoi grains (seed 3), bcc N_sl '
                               f'{"[12,12,24]" if "bcc48" in args.workload else "[12,12]"}, '
                               'tension dot_F_xx 1e-3/s, 100 increments to 10 %' if cells is None else
                               f'{args.workload} at {cells}',
                   'solver': f"{args.solver.replace('spectral_', '')} spectral, Anderson fixed point (m=8)"
                             + ('' if args.derivative == 'continuous' else f', derivative {args.derivative}'),
                   'precision': 'mixed',
                   'parallelism': f'replicas x{world}',
                   'l2': f'inputs larger than L2 (device memory of the context {mx["device_gb"]:.1f} GB)',
                   'increments_timed': f'{warmup + 1}..{warmup + args.steps}',
                   'tuning': {p: headline[k]['tuning'] for p, k in (('mixed', 'mixed'), ('fp64', 'fp64_raw'))
                              if headline.get(k)}},
        'fp64': headline['fp64'],
        's_per_increment': headline['s_per_increment'],
        'mixed_over_fp64': headline['mixed_over_fp64'],
        'mixed_vs_fp64_P_av_rel_err_max': headline['P_av_rel_err'],
        'roofline': headline['roofline'],
        'cpu_baseline': cpu,
        'e2e': headline['e2e'],
        'gpu_launches': mx['launches'],
        'clocks': mx['clocks'],
        'iterations': headline['iterations'],
    }
    if b48 is not None:
        line['bcc48'] = {'workload': 'grid256_bcc48_2000g: the same RVE with N_sl [12,12,24] (48 systems)',
                         'value': b48['value'], 'unit': 'updates/s', 'fp64': b48['fp64'],
                         'mixed_over_fp64': b48['mixed_over_fp64'], 'P_av_rel_err': b48['P_av_rel_err'],
                         'increments_timed': f'{BCC48_WARMUP + 1}..{BCC48_WARMUP + BCC48_STEPS}',
                         's_per_increment': b48['s_per_increment'], 'roofline_fp64': b48['roofline']['fp64'],
                         'traffic': b48['roofline']['traffic'], 'traffic_source': b48['roofline']['traffic_source'],
                         'clocks': b48['mixed']['clocks'], 'tuning': b48['mixed'].get('tuning')}
    if batched is not None:
        line['batched'] = batched
    print(json.dumps(line, default=_json_default), flush=True)


if __name__ == '__main__':
    main()
