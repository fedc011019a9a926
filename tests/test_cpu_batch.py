"""Host-side logic of batched solves across ranks: the cost-model plan and the result gather.

The multi-rank path runs as two `gloo` processes on the CPU: each rank solves the systems the
plan gives it (with the CPU oracle standing in for the GPU solver) and the results are merged on
every rank; each system must be solved exactly once, with the same results as a single rank.
"""

from __future__ import annotations

import os
import socket

import numpy as np
import pytest

from polysolve_b200 import batch, synthetic


def test_lpt_plan_covers_every_system_once_and_balances():
    edges = synthetic.batch_edges(64, seed=0)
    costs = batch.edges_cost(edges)
    for ranks in (1, 2, 3, 4, 8):
        plan = batch.assign_lpt(costs, ranks)
        flat = sorted(i for p in plan for i in p)
        assert flat == list(range(64))
        assert batch.imbalance(costs, plan) < 1.05
        assert plan == batch.assign_lpt(costs, ranks)  # deterministic: every rank computes it alone


def test_lpt_plan_edge_cases():
    assert batch.assign_lpt([], 3) == [[], [], []]
    assert batch.assign_lpt([5.0], 2) == [[0], []]
    with pytest.raises(ValueError):
        batch.assign_lpt([1.0], 0)
    # equal costs: round-robin by index
    assert batch.assign_lpt([1.0] * 4, 2) == [[0, 2], [1, 3]]


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, world: int, port: int, edges: list[int], out_path: str) -> None:
    import torch.distributed as dist

    from oracle import oracle as O

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        plan = batch.assign_lpt(batch.edges_cost(edges), world)
        local = {}
        for i in plan[rank]:
            s = synthetic.elasticity(edges[i], young_sigma=0.5, seed=i)
            b = synthetic.rhs(s.n, seed=i)
            x, it, rel = O.jacobi_pcg(s.outer, s.inner, s.vals, s.n, b, 1e-8)
            local[i] = {"rank": rank, "iters": int(it), "rel": float(rel), "xsum": float(np.sum(x))}
        merged = batch.gather_results(local)
        if rank == 0:
            import json

            with open(out_path, "w") as f:
                json.dump({str(k): v for k, v in merged.items()}, f)
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_solve_each_system_once(tmp_path):
    import torch.multiprocessing as mp

    edges = [4, 6, 5, 7, 3, 6, 4, 5]
    out = tmp_path / "merged.json"
    mp.start_processes(_rank_main, args=(2, _free_port(), edges, str(out)), nprocs=2, join=True,
                       start_method="spawn")
    import json

    merged = {int(k): v for k, v in json.load(open(out)).items()}
    assert sorted(merged) == list(range(len(edges)))
    plan = batch.assign_lpt(batch.edges_cost(edges), 2)
    for r, items in enumerate(plan):
        for i in items:
            assert merged[i]["rank"] == r
            assert merged[i]["rel"] <= 1e-8
    # the same systems solved by one process give the same results
    from oracle import oracle as O

    for i in (0, 3):
        s = synthetic.elasticity(edges[i], young_sigma=0.5, seed=i)
        b = synthetic.rhs(s.n, seed=i)
        x, it, _ = O.jacobi_pcg(s.outer, s.inner, s.vals, s.n, b, 1e-8)
        assert merged[i]["iters"] == it
        assert merged[i]["xsum"] == pytest.approx(float(np.sum(x)), rel=1e-12)
