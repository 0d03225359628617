"""Many independent RVEs on one GPU.

Each RVE is its own solver context (its fields, cuFFT plans and CUDA streams); a pool of host
threads drives the RVEs' increment loops.  The library calls release the interpreter lock, so
the RVEs' kernel sequences are issued concurrently on their own streams and overlap on the
device, which keeps the GPU busy although a single small RVE (8^3 ... 32^3 cells) is bound by
launch latency.  RVEs never exchange data; every RVE's results are those of a standalone run.
"""
from __future__ import annotations

import threading
import time
from concurrent.futures import ThreadPoolExecutor

from .grid import SpectralBasic, run_load_cases, run_load_cases_native


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
