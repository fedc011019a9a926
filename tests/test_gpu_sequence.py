"""A Newton-like sequence: same pattern, new values every step, warm starts from previous
solutions (values-only refactorization)."""

import numpy as np
import pytest

from polysolve_b200 import Solver, synthetic
from polysolve_b200.sequence import solve_sequence

pytestmark = pytest.mark.gpu


def test_warm_starts_save_iterations_on_a_sequence():
    N, steps = 10, 6
    systems, rhs = [], []
    for k in range(steps):
        sk, bk = synthetic.workload_sequence60(k, seed=3, N=N)
        systems.append(sk.scipy())
        rhs.append(bk)
    pos = synthetic.workload_sequence60(0, seed=3, N=N)[0].positions
    totals = {}
    for mode in ("zero", "previous", "extrapolate"):
        s = Solver.create("MAS", "")
        s.set_parameters({"MAS": {"block_dim": 3, "relative_tolerance": 1e-8, "absolute_tolerance": 0.0,
                                  "precision": "fp16", "true_residual_period": 50, "check_period": 1,
                                  "initial_guess": "input"}})
        s.set_positions(pos)
        s.analyze_pattern(systems[0], systems[0].shape[0])
        res = solve_sequence(s, systems, rhs, mode)
        assert all(r["status"] == "Reach relative tolerance" for r in res)
        assert all(r["rel"] <= 5e-8 for r in res)
        totals[mode] = sum(r["iterations"] for r in res)
    assert totals["previous"] < totals["zero"]
    assert totals["extrapolate"] <= totals["previous"]


def test_values_only_refactorize_matches_fresh_solver():
    """Refactorizing the same pattern with new values (same positions, not lazy) keeps the
    ordering and coarse space and refreshes only the inverses: the solution is bit-identical to
    a fresh solver's on the new values."""
    s0, b = synthetic.workload_sequence60(0, seed=5, N=9)
    s1, _ = synthetic.workload_sequence60(7, seed=5, N=9)
    params = {"MAS": {"block_dim": 3, "relative_tolerance": 1e-9, "absolute_tolerance": 0.0,
                      "precision": "fp16"}}

    def fresh(system):
        s = Solver.create("MAS", "")
        s.set_parameters(params)
        s.set_positions(s0.positions)
        s.analyze_pattern(system.scipy(), system.n)
        s.factorize(system.scipy())
        return s

    reused = fresh(s0)
    x0 = np.zeros(s0.n)
    reused.solve(b, x0)
    reused.factorize(s1.scipy())
    x1 = np.zeros(s0.n)
    reused.solve(b, x1)
    x2 = np.zeros(s0.n)
    fresh(s1).solve(b, x2)
    assert not np.array_equal(x0, x1)
    assert np.array_equal(x1, x2)


def test_preconditioner_refresh_period():
    """preconditioner_refresh 3: two of three values-only refactorizations keep the previous
    inverses (PCG still uses the new matrix), every solve meets the tolerance, and the iteration
    count stays close to rebuilding every time."""
    steps = [synthetic.workload_sequence60(k, seed=9, N=9) for k in range(7)]
    totals, flags = {}, []
    for period in (1, 3):
        s = Solver.create("MAS", "")
        s.set_parameters({"MAS": {"block_dim": 3, "relative_tolerance": 1e-8, "absolute_tolerance": 0.0,
                                  "precision": "fp16", "preconditioner_refresh": period}})
        s.set_positions(steps[0][0].positions)
        s.analyze_pattern(steps[0][0].scipy(), steps[0][0].n)
        it = 0
        for sk, bk in steps:
            A = sk.scipy()
            s.factorize(A)
            x = np.zeros(sk.n)
            s.solve(bk, x)
            info = s.get_info({})
            assert info["solver_status"] == "Reach relative tolerance"
            assert np.linalg.norm(A @ x - bk) <= 2e-8 * np.linalg.norm(bk)
            it += info["solver_iter"]
            if period == 3:
                flags.append(info["preconditioner_current"])
        totals[period] = it
    assert flags == [True, False, False, True, False, False, True]
    assert totals[3] <= 1.3 * totals[1], totals
    with pytest.raises(Exception):
        s.set_parameters({"MAS": {"preconditioner_refresh": 0}})


def test_pipelined_value_upload_on_a_large_system():
    """nnz x 8 bytes above two 16 MB staging chunks: the CSC values go through the pinned double
    buffer (full and values-only factorizations); both solves meet the tolerance against the
    matrices on the host."""
    s0, b0 = synthetic.workload_sequence60(0, seed=12, N=40)
    s1, b1 = synthetic.workload_sequence60(1, seed=12, N=40)
    assert s0.vals.size * 8 > 2 * (16 << 20)
    s = Solver.create("MAS", "")
    s.set_parameters({"MAS": {"block_dim": 3, "relative_tolerance": 1e-8, "absolute_tolerance": 0.0,
                              "precision": "fp16"}})
    s.set_positions(s0.positions)
    s.analyze_pattern(s0.scipy(), s0.n)
    for sk, bk in ((s0, b0), (s1, b1)):
        A = sk.scipy()
        s.factorize(A)
        x = np.zeros(sk.n)
        s.solve(bk, x)
        assert np.linalg.norm(A @ x - bk) <= 2e-8 * np.linalg.norm(bk)
    assert "mas_inverses" in s.get_info({})["factorize_phases_ms"]  # the second one was values-only


def test_declared_values_only_refactorization():
    """mas_factorize_values (values in the last matrix's CSC order, no row indices, no pattern
    check) gives exactly the solve of factorize on the same matrix; it is refused before any
    factorization, with a different nnz, and after the positions changed."""
    from polysolve_b200 import MasError

    s0, b0 = synthetic.workload_sequence60(0, seed=4, N=9)
    s1, b1 = synthetic.workload_sequence60(1, seed=4, N=9)
    A0, A1 = s0.scipy().tocsc(), s1.scipy().tocsc()
    params = {"block_dim": 3, "relative_tolerance": 1e-8, "absolute_tolerance": 0.0, "precision": "fp16",
              "true_residual_period": 50, "check_period": 1}

    def solver():
        s = Solver.create("MAS", "")
        s.set_parameters({"MAS": params})
        s.set_positions(s0.positions)
        return s

    ref, dec = solver(), solver()
    with pytest.raises(MasError):
        dec.factorize_values(A1)
    ref.factorize(A0)
    ref.factorize(A1)
    dec.factorize(A0)
    dec.factorize_values(A1)
    assert "upload" in dec.get_info({})["factorize_phases_ms"]
    x_ref, x = np.zeros(A1.shape[0]), np.zeros(A1.shape[0])
    ref.solve(b1, x_ref)
    dec.solve(b1, x)
    np.testing.assert_array_equal(x, x_ref)
    with pytest.raises(MasError):
        dec.factorize_values(A1.data[:-1])
    dec.set_positions(s0.positions + 1e-3)
    with pytest.raises(MasError):
        dec.factorize_values(A1)
