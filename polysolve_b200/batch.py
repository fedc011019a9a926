"""Batches of independent systems across GPUs (the 64-system workload).

Independent systems shard with no collective on the data path: each rank (one process per GPU)
factorizes and solves its share with ``solve_batch`` (concurrent streams on its GPU), and only the
per-system results (iterations, status, residuals, times) are gathered at the end. The share is
fixed by a cost model, longest-processing-time first, so ranks get balanced work.
"""

from __future__ import annotations

from typing import Any, Sequence


def system_cost(nnzb: int, dof: int) -> float:
    """Estimated solve cost: block nonzeros (bytes per iteration) times the expected iteration
    count, which for these elasticity meshes grows like the grid edge, i.e. dof^(1/3)."""
    return float(nnzb) * max(1.0, float(dof)) ** (1.0 / 3.0)


def assign_lpt(costs: Sequence[float], ranks: int) -> list[list[int]]:
    """Longest-processing-time-first assignment of items to `ranks` bins: items in decreasing
    cost (ties by index) each go to the least loaded rank (ties by rank). Deterministic, so every
    rank computes the same plan without communication. Each rank's list is sorted."""
    if ranks < 1:
        raise ValueError("ranks must be >= 1")
    load = [0.0] * ranks
    plan: list[list[int]] = [[] for _ in range(ranks)]
    for i in sorted(range(len(costs)), key=lambda k: (-float(costs[k]), k)):
        r = min(range(ranks), key=lambda q: (load[q], q))
        plan[r].append(i)
        load[r] += float(costs[i])
    return [sorted(p) for p in plan]


def imbalance(costs: Sequence[float], plan: list[list[int]]) -> float:
    """max rank load / mean rank load (1.0 = perfect)."""
    loads = [sum(float(costs[i]) for i in p) for p in plan]
    mean = sum(loads) / max(len(loads), 1)
    return max(loads) / mean if mean > 0 else 1.0


def gather_results(local: dict[int, Any], group=None) -> dict[int, Any]:
    """Merge every rank's {system index: result} on all ranks (torch.distributed object
    all-gather; a single process returns its own dict)."""
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()):
        return dict(local)
    parts: list[Any] = [None] * dist.get_world_size(group)
    dist.all_gather_object(parts, local, group=group)
    out: dict[int, Any] = {}
    for p in parts:
        out.update(p)
    return out


def edges_cost(edges: Sequence[int]) -> list[float]:
    """Cost of each N^3 grid system of the batch workload from its edge N (V = (N + 1)^3 blocks,
    about 15 blocks per row)."""
    out = []
    for N in edges:
        V = (N + 1) ** 3
        out.append(system_cost(15 * V, 3 * V))
    return out


__all__ = ["system_cost", "assign_lpt", "imbalance", "gather_results", "edges_cost"]
