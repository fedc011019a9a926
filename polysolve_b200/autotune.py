"""Autotuner for the solver's launch-shape parameters, measured on the caller's own systems.

The kernels' tile shapes are fixed by the data layout (a subdomain is a bank of 32 block rows, one
warp; a subdomain matrix is 32 x block_dim rows), so what is tuned are the launch shapes and
runtime choices that depend on the system sizes and the GPU:

* ``spmv_unroll`` - slots of the block SpMV per loop trip (1, 2 or 4; three compiled variants):
  more slots keep more loads in flight per warp but cost registers (56, 80, 128) and so CTAs per
  SM; small systems with few banks and large ones need different points.
* ``poll_period`` - PCG iterations per replayed CUDA graph (and per host poll of the convergence
  flag): short graphs stop sooner after convergence, long ones cost fewer launches and polls.
  Small systems are launch-bound and prefer long graphs; large ones barely care.
* ``apply_items_per_warp`` - the fewest inverses each warp of the MAS apply multiplies (1, 2, 4,
  8): 1 gives a lone solve the most CTAs; in a batch of small systems more items per warp let the
  apply's copy pipeline run past its start-up latency and leave SMs to the other systems.
* ``batch_launch`` of ``solve_batch`` / ``solve_batch_device`` - one launch per PCG phase for each
  group of systems ("fused") or one CUDA stream per system ("streams"); with "fused",
  ``batch_groups`` - how many such groups (each on its own stream) the batch is cut into by size.
* ``threads`` of ``solve_batch`` / ``solve_batch_device`` - host threads driving a batch of
  independent systems (with "streams" one CUDA stream each: too few leave the GPU idle between
  small solves, too many contend on the host; with "fused" they run the per-system input and
  result steps).

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


def tune_param(solvers, run, key: str, candidates, repeats: int = 3) -> dict:
    """Sets the integer parameter ``key`` on every solver to each candidate, times ``run()`` (which
    solves with them), keeps the fastest and returns ``{"best": value, "ms": {candidate: median
    ms}}`` with the best value left set."""
    table = {}
    for c in candidates:
        for s in solvers:
            s.set_parameters({"MAS": {key: int(c)}})
        table[int(c)] = _median_ms(run, repeats)
    best = min(table, key=table.get)
    for s in solvers:
        s.set_parameters({"MAS": {key: best}})
    return {"best": best, "ms": table}


def tune_poll_period(solvers, run, candidates=(5, 10, 20, 40), repeats: int = 3) -> dict:
    """``tune_param`` for ``poll_period`` (iterations per replayed CUDA graph)."""
    return tune_param(solvers, run, "poll_period", candidates, repeats)


def tune_spmv_unroll(solvers, run, candidates=(1, 2, 4), repeats: int = 3) -> dict:
    """``tune_param`` for ``spmv_unroll`` (slots of the block SpMV per loop trip)."""
    return tune_param(solvers, run, "spmv_unroll", candidates, repeats)


def tune_batch_threads(run_with_threads, candidates=(4, 8, 16, 32, 64), repeats: int = 3) -> dict:
    """Times ``run_with_threads(t)`` for each thread count; returns the fastest and the table."""
    table = {int(t): _median_ms(lambda t=t: run_with_threads(int(t)), repeats) for t in candidates}
    best = min(table, key=table.get)
    return {"best": best, "ms": table}


def tune_batch_launch(solvers, run, candidates=("fused", "streams"), repeats: int = 3) -> dict:
    """Times ``run()`` with each ``batch_launch`` mode set on every solver; keeps the fastest."""
    table = {}
    for c in candidates:
        for s in solvers:
            s.set_parameters({"MAS": {"batch_launch": c}})
        table[c] = _median_ms(run, repeats)
    best = min(table, key=table.get)
    for s in solvers:
        s.set_parameters({"MAS": {"batch_launch": best}})
    return {"best": best, "ms": table}


def tune_batch(solvers, b_ptrs, x_ptrs, ns, *, cache_path: str | None = None, repeats: int = 3,
               poll_candidates=(5, 10, 20, 40), unroll_candidates=(1, 2, 4),
               thread_candidates=(4, 8, 16, 32, 64), launch_candidates=("fused", "streams"),
               group_candidates=(1, 2, 4, 8), ipw_candidates=(1, 2, 4, 8)) -> dict:
    """Tunes ``apply_items_per_warp``, ``batch_launch`` (with ``batch_groups`` when fused),
    ``poll_period`` and ``spmv_unroll`` (all solvers) and the host thread count of
    ``solve_batch_device`` for these systems, one after another; returns ``{"apply_items_per_warp":
    k, "batch_launch": m, "batch_groups": g, "poll_period": p, "spmv_unroll": u, "threads": t,
    "tables": {...}, "cached": bool}`` and leaves the parameters set on the solvers. With
    ``cache_path`` a previous result for the same sizes is reused."""
    from .solver import solve_batch_device

    key = signature(ns)
    cache = _load_cache(cache_path)
    if key in cache:
        res = dict(cache[key], cached=True)
        for s in solvers:
            s.set_parameters({"MAS": {"poll_period": int(res["poll_period"]),
                                      "spmv_unroll": int(res.get("spmv_unroll", 2)),
                                      "batch_launch": str(res.get("batch_launch", "streams")),
                                      "batch_groups": int(res.get("batch_groups", 0)),
                                      "apply_items_per_warp": int(res.get("apply_items_per_warp", 1))}})
        return res
    threads0 = min(32, max(1, len(solvers)))
    run0 = lambda: solve_batch_device(solvers, b_ptrs, x_ptrs, ns, threads=threads0)  # noqa: E731
    ipw = tune_param(solvers, run0, "apply_items_per_warp", ipw_candidates, repeats)
    groups = {"best": 0, "ms": {}}
    if "fused" in launch_candidates:
        for s in solvers:
            s.set_parameters({"MAS": {"batch_launch": "fused"}})
        cands = [g for g in group_candidates if g <= max(1, len(solvers))] or [1]
        groups = tune_param(solvers, run0, "batch_groups", cands, repeats)
    launch = tune_batch_launch(solvers, run0, launch_candidates, repeats)
    poll = tune_poll_period(solvers, run0, poll_candidates, repeats)
    unroll = tune_spmv_unroll(solvers, run0, unroll_candidates, repeats)
    thr = tune_batch_threads(lambda t: solve_batch_device(solvers, b_ptrs, x_ptrs, ns, threads=t),
                             [t for t in thread_candidates if t <= max(1, len(solvers))] or [1], repeats)
    res = {"apply_items_per_warp": ipw["best"], "batch_launch": launch["best"], "batch_groups": groups["best"],
           "poll_period": poll["best"], "spmv_unroll": unroll["best"], "threads": thr["best"],
           "tables": {"apply_items_per_warp_ms": ipw["ms"], "batch_groups_ms": groups["ms"],
                      "batch_launch_ms": launch["ms"], "poll_period_ms": poll["ms"], "spmv_unroll_ms": unroll["ms"],
                      "threads_ms": thr["ms"]}}
    cache[key] = res
    _store_cache(cache_path, cache)
    return dict(res, cached=False)


__all__ = ["tune_param", "tune_poll_period", "tune_spmv_unroll", "tune_batch_launch", "tune_batch_threads", "tune_batch",
           "signature"]
