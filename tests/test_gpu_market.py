"""A system read from Matrix Market files (as polysolve's tests load theirs) is the in-memory one
bit for bit and solves to the same solution."""

import numpy as np
import pytest
import scipy.io

from polysolve_b200 import Solver, market, synthetic

pytestmark = pytest.mark.gpu


def test_solve_from_matrix_market_files(tmp_path):
    system = synthetic.elasticity(9, young_sigma=1.0, jitter=0.2, seed=8)
    A = system.scipy()
    b = synthetic.rhs(system.n, seed=8)
    # general: every stored value round-trips exactly (a symmetric file keeps one triangle, and
    # the assembled matrix is symmetric only to rounding)
    scipy.io.mmwrite(tmp_path / "A.mtx", A, symmetry="general", precision=17)
    market.save_vector(tmp_path / "b.mtx", b)
    A2 = market.load_matrix(tmp_path / "A.mtx")
    b2 = market.load_vector(tmp_path / "b.mtx")
    A.sort_indices()
    assert np.array_equal(A2.indptr, A.indptr) and np.array_equal(A2.indices, A.indices)
    assert np.array_equal(A2.data, A.data) and np.array_equal(b2, b)
    xs = []
    for M, rhs in ((A, b), (A2, b2)):
        s = Solver.create("MAS", "")
        s.set_parameters({"MAS": {"block_dim": 3, "relative_tolerance": 1e-8, "absolute_tolerance": 0.0}})
        s.set_positions(system.positions)
        s.analyze_pattern(M, M.shape[0])
        s.factorize(M)
        x = np.zeros(M.shape[0])
        s.solve(rhs, x)
        xs.append(x)
        assert np.linalg.norm(M @ x - rhs) <= 1e-8 * np.linalg.norm(rhs)
    assert np.array_equal(xs[0], xs[1])  # factorize and solve are deterministic
