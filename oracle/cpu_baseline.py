"""Timed CPU baseline: LAPACK zhegv (itype=1, jobz='V', uplo='L', scipy's
bundled OpenBLAS) over the host cores, one single-threaded worker process
per core (OPENBLAS_NUM_THREADS=1), batch split statically. This is the
solver the reference's own tests time on the host
(tests/static/test_full_batched_n54.cpp, LAPACKE_zhegv).

Workers are started with the `spawn` method so that they never inherit a
CUDA context.
"""
from __future__ import annotations

import multiprocessing as mp
import os
import time

_H = _S = None


def _init(n, count, seed, kappa):
    os.environ["OPENBLAS_NUM_THREADS"] = "1"
    import sys
    from pathlib import Path
    sys.path.insert(0, str(Path(__file__).resolve().parents[1]))
    from sunny_gen_eigensolver_b200.generators import baseline_problems
    global _H, _S
    _H, _S = baseline_problems(n, count, seed=seed + os.getpid() % 100000, kappa=kappa)


def _solve_all(_):
    from scipy.linalg import lapack
    t0 = time.perf_counter()
    for b in range(_H.shape[0]):
        lapack.zhegv(_H[b], _S[b], itype=1, jobz="V", uplo="L")
    return _H.shape[0], time.perf_counter() - t0


def usable_cores() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


class ZhegvPool:
    """`workers` spawned processes, each holding `per_worker` seeded problems.
    One `step()` has every worker solve its problems once."""

    def __init__(self, n: int = 54, per_worker: int = 32, workers: int | None = None,
                 seed: int = 20261205, kappa: float = 100.0):
        self.n, self.per_worker = n, per_worker
        self.workers = workers or usable_cores()
        before = os.environ.get("OPENBLAS_NUM_THREADS")
        os.environ["OPENBLAS_NUM_THREADS"] = "1"
        try:
            self.pool = mp.get_context("spawn").Pool(self.workers, initializer=_init,
                                                     initargs=(n, per_worker, seed, kappa))
        finally:
            if before is None:
                os.environ.pop("OPENBLAS_NUM_THREADS", None)
            else:
                os.environ["OPENBLAS_NUM_THREADS"] = before

    def step(self):
        """Returns (solves, wall seconds) of one pass over every worker's sample."""
        t0 = time.perf_counter()
        res = self.pool.map(_solve_all, range(self.workers), chunksize=1)
        return sum(r[0] for r in res), time.perf_counter() - t0

    def close(self):
        self.pool.close()
        self.pool.join()


def time_zhegv(n: int = 54, per_worker: int = 32, workers: int | None = None, seconds: float = 8.0,
               seed: int = 20261205, kappa: float = 100.0) -> dict:
    """Solves/s of zhegv over the host cores, re-solving each worker's
    sample until at least `seconds` of wall time have passed."""
    p = ZhegvPool(n, per_worker, workers, seed, kappa)
    try:
        p.step()  # warm-up (imports, page-in)
        total, wall = 0, 0.0
        while wall < seconds:
            s, t = p.step()
            total += s
            wall += t
    finally:
        p.close()
    return {
        "value": total / wall,
        "unit": "solves/s",
        "cores": p.workers,
        "kind": "port",
        "sample": (f"LAPACK zhegv (scipy OpenBLAS, 1 thread per worker) on {p.workers} worker processes, "
                   f"each re-solving its own {per_worker} seeded N={n} problems; {total} solves in {wall:.1f} s"),
    }
