"""Many independent RVEs on one GPU.

DeviceBatch: every RVE is a solver context and all of them form one batch of the library
(dmk_batch_*).  Each RVE's increment loop runs on the host up to the point where it needs a
solution; the solutions of all waiting RVEs are computed together, with the fixed-point iterations
of every RVE in shared launches (per iteration one CUDA graph for the constitutive evaluation of
all active RVEs, one cuFFT plan pair per edge size, batched residual and Anderson kernels).  The
RVEs never exchange data; every RVE's results are those of a standalone run.  It takes the basic
scheme (FP64 or mixed form) with one phase for all RVEs.

BatchRunner: one context per RVE on its own streams, driven by a pool of host threads (any
scheme and precision; the library calls release the interpreter lock, so the RVEs' kernel
sequences overlap on the device).
"""
from __future__ import annotations

import threading
import time
from concurrent.futures import ThreadPoolExecutor

import ctypes as C

import numpy as np

from . import _lib
from .config import LoadStepStruct, SolutionStruct
from .grid import IncrementDriver, SpectralBasic, run_load_cases, run_load_cases_native


class BatchRunner:
    """Run a list of jobs ``(rve, phase, loadcases, numerics)`` with ``threads`` host threads.

    Contexts are created lazily by the thread that runs the job and closed when it finishes, so
    at most ``threads`` RVEs hold device memory at a time."""

    def __init__(self, jobs, threads: int = 16, precision: str = 'fp64', max_increments: int | None = None,
                 solver_class=SpectralBasic, native: bool = True):
        self.jobs = list(jobs)
        self.threads = max(1, int(threads))
        self.precision = precision
        self.max_increments = max_increments
        self.solver_class = solver_class
        self.native = native              # the C++ increment loop: one library call per RVE
        self.results = [None] * len(self.jobs)
        self.updates = [0] * len(self.jobs)
        self._lock = threading.Lock()

    def _run_one(self, k: int, on_finish=None):
        rve, phase, lcs, num = self.jobs[k]
        s = self.solver_class(rve.cells, rve.size, rve.material, rve.quaternions, phase, num, precision=self.precision)
        try:
            run = run_load_cases_native if self.native else run_load_cases
            stats = run(s, lcs, max_increments=self.max_increments)
            # material-point updates of the converged solutions (cut-back attempts not counted)
            total = sum(r.residual_evals for r in stats) * s.N
            if on_finish is not None:
                on_finish(k, s)
        finally:
            s.close()
        with self._lock:
            self.results[k] = stats
            self.updates[k] = total
        return k

    def run(self, on_finish=None) -> float:
        """Run every job; returns the wall time in seconds.  ``on_finish(k, solver)`` is called in
        the worker thread before job k's context is closed (to read its fields)."""
        t0 = time.perf_counter()
        with ThreadPoolExecutor(max_workers=self.threads) as ex:
            for f in [ex.submit(self._run_one, k, on_finish) for k in range(len(self.jobs))]:
                f.result()
        return time.perf_counter() - t0


class DeviceBatch:
    """Run the jobs ``(rve, phase, loadcases, numerics)`` as one batch of the library.

    All contexts are created up front (they hold device memory until :meth:`close`).  ``run``
    advances every job's increment loop (``IncrementDriver.step_requests``) to its next solution
    request, solves all requests with one ``dmk_batch_solution`` call, hands each job its solution
    and repeats until every job has run its increments (all, or ``max_increments``).  Jobs may
    cut back and so fall out of step with the others; each request is solved at its own job's
    increment and time step."""

    def __init__(self, jobs, max_increments: int | None = None, N_cutback_max: int = 3, device: int = 0,
                 precision: str = 'fp64'):
        self.jobs = list(jobs)
        self.max_increments = max_increments
        self.lib = _lib.load()
        self.solvers = [SpectralBasic(rve.cells, rve.size, rve.material, rve.quaternions, phase, num,
                                      precision=precision, device=device) for rve, phase, _, num in self.jobs]
        self.drivers = [IncrementDriver(s, lcs, N_cutback_max) for s, (_, _, lcs, _) in zip(self.solvers, self.jobs)]
        self.results = [[] for _ in self.jobs]
        self.updates = [0] * len(self.jobs)   # material-point updates of the converged (sub)increments
        self.failed: list[int] = []
        self.batch_calls = 0
        self.device_ms = 0.0              # device time of the batched solutions (dmk_batch_stats)
        ctxs = (C.c_void_p * len(self.solvers))(*[s.ctx.value for s in self.solvers])
        h = C.c_void_p()
        _lib.check(self.lib.dmk_batch_create(C.byref(h), ctxs, len(self.solvers)))
        self.handle = h
        self._gens = [None] * len(self.jobs)

    def _advance(self, k: int, sol) -> bool:
        """Drive job k until it requests a solution (True) or has run its increments (False)."""
        while True:
            g = self._gens[k]
            try:
                if g is None:
                    d = self.drivers[k]
                    if d.done or (self.max_increments is not None and d.total >= self.max_increments):
                        return False
                    g = self._gens[k] = d.step_requests()
                    g.send(None)
                else:
                    g.send(sol)
                return True
            except StopIteration as stop:
                self.results[k].extend(stop.value or [])
                self._gens[k] = None
                sol = None

    def solve(self, waiting: list[int]):
        """One dmk_batch_solution call for the jobs in ``waiting``; their solution states."""
        which = (C.c_int * len(waiting))(*waiting)
        outs = (SolutionStruct * len(waiting))()
        _lib.check(self.lib.dmk_batch_solution(self.handle, which, len(waiting), outs))
        self.device_ms += self.stats()['solution_ms_last']
        for j, k in enumerate(waiting):
            s = self.solvers[k]
            c = s.counters()
            s.total_counters += c
            if outs[j].converged:
                self.updates[k] += int(c[0])
        return [outs[j] for j in range(len(waiting))]

    def run(self, solve=None) -> float:
        """Run every job; returns the wall time in seconds.  ``solve(waiting)`` replaces the
        library call (it returns one solution state per listed job)."""
        solve = solve or self.solve
        t0 = time.perf_counter()
        waiting = [k for k in range(len(self.jobs)) if self._advance(k, None)]
        while waiting:
            outs = solve(waiting)
            self.batch_calls += 1
            waiting = [k for k, sol in zip(waiting, outs) if self._advance(k, sol)]
        return time.perf_counter() - t0

    def run_native(self, N_cutback_max: int = 3) -> float:
        """Run every job through the library's C++ batched increment loop (dmk_batch_run): no
        interpreter between the members' calls; the results and updates as :meth:`run` (the solvers'
        ``total_counters`` are not kept).  Returns the wall time in seconds.  A job that does not
        converge after the cutbacks stops; its index goes to ``failed``."""
        from .config import BATCH_INCREMENT_CB, loadstep_structs
        from .grid import IncrementStats
        n = len(self.jobs)
        steps = [loadstep_structs(lcs) for _, _, lcs, _ in self.jobs]
        arr = (C.POINTER(LoadStepStruct) * n)(*[C.cast(s, C.POINTER(LoadStepStruct)) for s in steps])
        counts = (C.c_int * n)(*[len(lcs) for _, _, lcs, _ in self.jobs])
        status = (C.c_int * n)()
        clock = [time.perf_counter()]

        def cb(k, info_p, _user):
            i = info_p.contents
            now = time.perf_counter()
            self.results[k].append(IncrementStats(i.inc, i.t, i.cutback_level, bool(i.converged), i.iterations,
                                                  i.residual_evals, now - clock[0],
                                                  np.array(i.P_av[:]).reshape(3, 3, order='F')))
            clock[0] = now
            self.updates[k] += i.residual_evals * self.solvers[k].N
            return 0

        cfn = BATCH_INCREMENT_CB(cb)
        t0 = time.perf_counter()
        _lib.check(self.lib.dmk_batch_run(self.handle, arr, counts, N_cutback_max, int(self.max_increments or 0), cfn,
                                          None, status))
        seconds = time.perf_counter() - t0
        self.failed = [k for k in range(n) if status[k] != 0]
        return seconds

    def stats(self) -> dict:
        """Device ms of the constitutive graphs and of the whole last batched solution, graphs
        launched, constitutive passes, fixed-point iterations and batched solutions so far, and the
        host ms of the last solution's set-up, iterations, and tangents with counters."""
        out = np.zeros(9)
        _lib.check(self.lib.dmk_batch_stats(self.handle, out.ctypes.data_as(C.POINTER(C.c_double))))
        return {'const_ms_last': out[0], 'solution_ms_last': out[1], 'graphs': int(out[2]), 'passes': int(out[3]),
                'iterations': int(out[4]), 'solutions': int(out[5]), 'host_ms_last': out[6:9].tolist()}

    def close(self) -> None:
        if getattr(self, 'handle', None):
            self.lib.dmk_batch_destroy(self.handle)
            self.handle = None
        for s in getattr(self, 'solvers', []):
            s.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
