"""Autotuner for the solver's launch-shape parameters, measured on the caller's own systems.

The kernels' tile shapes are fixed by the data layout (a subdomain is a bank of 32 block rows, one
warp; a subdomain matrix is 32 x block_dim rows), so what is tuned are the runtime choices that
depend on the system sizes and the GPU:

* ``poll_period`` - PCG iterations per replayed CUDA graph (and per host poll of the convergence
  flag): short graphs stop sooner after convergence, long ones cost fewer launches and polls.
  Small systems are launch-bound and prefer long graphs; large ones barely care.
* ``threads`` of ``solve_batch`` / ``solve_batch_device`` - host threads (one CUDA stream each)
  driving a batch of independent systems: too few leave the GPU idle between small solves, too
  many contend on the host.

Each candidate is timed with the real call (synchronous, host clock) after one untimed call, the
median of ``repeats`` runs is kept, and the fastest candidate wins. Results can be cached in a JSON
file keyed by the systems' sizes, so a tuned process skips the search on the next run.
"""

from __future__ import annotations

import json
import os
import statistics
import time


def _median_ms(fn, repeats: int) -> float:
    fn()  # untimed: graph capture, first-touch allocations
    times = []
    for _ in range(repeats):
        t0 = time.perf_counter()
        fn()
        times.append((time.perf_counter() - t0) * 1000.0)
    return statistics.median(times)


def _load_cache(path):
    if path and os.path.exists(path):
        with open(path) as fh:
            return json.load(fh)
    return {}


def _store_cache(path, cache) -> None:
    if path:
        with open(path, "w") as fh:
            json.dump(cache, fh, indent=1, sort_keys=True)


def signature(ns) -> str:
    """Cache key: the sorted system sizes."""
    return "n=" + ",".join(str(n) for n in sorted(ns))


def tune_poll_period(solvers, run, candidates=(5, 10, 20, 40), repeats: int = 3) -> dict:
    """Sets ``poll_period`` on every solver to each candidate, times ``run()`` (which solves with
    them), keeps the fastest and returns ``{"best": value, "ms": {candidate: median ms}}``."""
    table = {}
    for c in candidates:
        for s in solvers:
            s.set_parameters({"MAS": {"poll_period": int(c)}})
        table[int(c)] = _median_ms(run, repeats)
    best = min(table, key=table.get)
    for s in solvers:
        s.set_parameters({"MAS": {"poll_period": best}})
    return {"best": best, "ms": table}


def tune_batch_threads(run_with_threads, candidates=(4, 8, 16, 32, 64), repeats: int = 3) -> dict:
    """Times ``run_with_threads(t)`` for each thread count; returns the fastest and the table."""
    table = {int(t): _median_ms(lambda t=t: run_with_threads(int(t)), repeats) for t in candidates}
    best = min(table, key=table.get)
    return {"best": best, "ms": table}


def tune_batch(solvers, b_ptrs, x_ptrs, ns, *, cache_path: str | None = None, repeats: int = 3,
               poll_candidates=(5, 10, 20, 40), thread_candidates=(4, 8, 16, 32, 64)) -> dict:
    """Tunes ``poll_period`` (all solvers) and the host thread count of ``solve_batch_device`` for
    these systems; returns ``{"poll_period": p, "threads": t, "tables": {...}, "cached": bool}``
    and leaves ``poll_period`` set on the solvers. With ``cache_path`` a previous result for the
    same sizes is reused."""
    from .solver import solve_batch_device

    key = signature(ns)
    cache = _load_cache(cache_path)
    if key in cache:
        res = dict(cache[key], cached=True)
        for s in solvers:
            s.set_parameters({"MAS": {"poll_period": int(res["poll_period"])}})
        return res
    threads0 = min(32, max(1, len(solvers)))
    poll = tune_poll_period(solvers, lambda: solve_batch_device(solvers, b_ptrs, x_ptrs, ns, threads=threads0),
                            poll_candidates, repeats)
    thr = tune_batch_threads(lambda t: solve_batch_device(solvers, b_ptrs, x_ptrs, ns, threads=t),
                             [t for t in thread_candidates if t <= max(1, len(solvers))] or [1], repeats)
    res = {"poll_period": poll["best"], "threads": thr["best"],
           "tables": {"poll_period_ms": poll["ms"], "threads_ms": thr["ms"]}}
    cache[key] = res
    _store_cache(cache_path, cache)
    return dict(res, cached=False)


__all__ = ["tune_poll_period", "tune_batch_threads", "tune_batch", "signature"]
