"""Batched solves of independent systems (`mas_solve_batch`) against one-at-a-time solves."""

from __future__ import annotations

import numpy as np
import pytest

from polysolve_b200 import MasError, Solver, solve_batch, synthetic

pytestmark = pytest.mark.gpu

PARAMS = {"block_dim": 3, "relative_tolerance": 1e-8, "absolute_tolerance": 0.0, "precision": "fp16",
          "true_residual_period": 50, "check_period": 1}


def _solver(system, params=PARAMS):
    s = Solver.create("MAS", "")
    s.set_parameters({"MAS": params})
    s.set_positions(system.positions)
    A = system.scipy()
    s.analyze_pattern(A, A.shape[0])
    s.factorize(A)
    return s


@pytest.fixture(scope="module")
def systems():
    edges = [3, 9, 5, 14, 7, 4, 11, 6]
    return [synthetic.elasticity(N, young_sigma=0.5, jitter=0.2, seed=10 + k) for k, N in enumerate(edges)]


def test_batch_matches_individual_solves(systems):
    solvers = [_solver(s) for s in systems]
    bs = [synthetic.rhs(s.n, seed=20 + k) for k, s in enumerate(systems)]
    ref = []
    for s, b in zip(solvers, bs):
        x = np.zeros_like(b)
        s.solve(b, x)
        ref.append((x, s.get_info({})["solver_iter"]))
    for threads in (0, 1, 3):
        xs = solve_batch(solvers, bs, threads=threads)
        for (xr, it), x, s, sysm, b in zip(ref, xs, solvers, systems, bs):
            # same kernels, same deterministic reductions: bit-identical to the single solve
            np.testing.assert_array_equal(x, xr)
            assert s.get_info({})["solver_iter"] == it
            A = sysm.scipy()
            assert np.linalg.norm(A @ x - b) <= 5e-8 * np.linalg.norm(b)


def test_batch_reports_each_failure(systems):
    good = _solver(systems[0])
    unfactorized = Solver.create("MAS", "")
    unfactorized.set_parameters({"MAS": PARAMS})
    b0 = synthetic.rhs(systems[0].n, seed=1)
    with pytest.raises(MasError):
        solve_batch([good, unfactorized], [b0, b0])
    # the good one still solved
    assert good.get_info({})["solver_status"] == "Reach relative tolerance"
    with pytest.raises(MasError):
        solve_batch([good, good], [b0, b0])  # the same handle twice
    assert solve_batch([], []) == []
