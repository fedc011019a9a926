"""Several right-hand sides at once (`mas_solve_multi`): groups of four or sixteen independent PCG
solves that share every read of the matrix and of the binary16 MAS inverses, against one-at-a-time
solves and the CPU oracle. The group width is the ``rhs_group`` parameter (automatic: sixteen for
more than four right-hand sides with block_dim 3)."""

from __future__ import annotations

import numpy as np
import pytest

from polysolve_b200 import Solver, synthetic

from .helpers import oracle_for

pytestmark = pytest.mark.gpu

CHOSEN = {"block_dim": 3, "relative_tolerance": 1e-8, "absolute_tolerance": 0.0, "precision": "fp16",
          "true_residual_period": 50, "check_period": 1}


def _solver(system, params):
    s = Solver.create("MAS", "")
    s.set_parameters({"MAS": params})
    s.set_positions(system.positions)
    A = system.scipy()
    s.analyze_pattern(A, A.shape[0])
    s.factorize(A)
    return s


@pytest.fixture(scope="module")
def contact_system():
    return synthetic.elasticity(9, young_sigma=1.0, jitter=0.2, seed=5, contact_pairs=80, contact_k=1e4,
                                contact_sigma=1.5)


@pytest.mark.parametrize("group,nrhs", [(4, 1), (4, 4), (4, 6), (16, 1), (16, 6), (16, 16), (0, 17)])
def test_multi_matches_single_solves_and_oracle(contact_system, group, nrhs):
    system = contact_system
    s = _solver(system, dict(CHOSEN, rhs_group=group))
    A = system.scipy()
    B = np.stack([synthetic.rhs(system.n, seed=40 + c) for c in range(nrhs)])
    X = s.solve_multi(B)
    info = s.get_info({})
    assert info["rhs_iterations"] and len(info["rhs_iterations"]) == nrhs
    assert all(st == "Reach relative tolerance" for st in info["rhs_status"])
    orc, _ = oracle_for(system, s, 3)
    for c in range(nrhs):
        b = B[c]
        assert np.linalg.norm(A @ X[c] - b) <= 5e-8 * np.linalg.norm(b)
        x1 = np.zeros(system.n)
        s.solve(b, x1)
        it1 = s.get_info({})["solver_iter"]
        # the same algorithm per right-hand side; the apply rounds x to binary16 hi + lo per column
        # and sums in another order, so counts may differ by a couple of iterations
        assert abs(info["rhs_iterations"][c] - it1) <= 2
        assert np.linalg.norm(X[c] - x1) <= 1e-5 * np.linalg.norm(x1)
        xo, oinfo = orc.pcg(b, rel_tol=1e-8, abs_tol=0.0, true_residual_period=50, check_period=1, mas_fp32=16)
        assert abs(info["rhs_iterations"][c] - oinfo["solver_iter"]) <= 2
        assert np.linalg.norm(X[c] - xo) <= 1e-5 * np.linalg.norm(xo)


@pytest.mark.parametrize("group", [4, 16])
def test_multi_repeatable_and_graph_free_equal(contact_system, group):
    """Deterministic: the same block of right-hand sides twice gives identical results, with and
    without graph replay of the iterations."""
    system = contact_system
    B = np.stack([synthetic.rhs(system.n, seed=70 + c) for c in range(5)])
    s = _solver(system, dict(CHOSEN, rhs_group=group))
    X1 = s.solve_multi(B)
    X2 = s.solve_multi(B)
    np.testing.assert_array_equal(X1, X2)
    s2 = _solver(system, dict(CHOSEN, cuda_graphs=False, rhs_group=group))
    X3 = s2.solve_multi(B)
    np.testing.assert_array_equal(X1, X3)


def test_multi_falls_back_to_single_solves_without_fp16(contact_system):
    system = contact_system
    params = dict(CHOSEN, precision="fp32")
    s = _solver(system, params)
    B = np.stack([synthetic.rhs(system.n, seed=90 + c) for c in range(3)])
    X = s.solve_multi(B)
    for c in range(3):
        x1 = np.zeros(system.n)
        s.solve(B[c], x1)
        np.testing.assert_array_equal(X[c], x1)


@pytest.mark.parametrize("group", [4, 16])
def test_multi_max_iterations(contact_system, group):
    system = contact_system
    s = _solver(system, dict(CHOSEN, max_iter=7, rhs_group=group))
    B = np.stack([synthetic.rhs(system.n, seed=3 + c) for c in range(4)])
    s.solve_multi(B)
    info = s.get_info({})
    assert info["rhs_iterations"] == [7, 7, 7, 7]
    assert all(st == "Reach max iterations" for st in info["rhs_status"])


def test_wide_and_narrow_groups_agree(contact_system):
    """Groups of sixteen and of four are the same algorithm per right-hand side (the sums run in
    another order): every column within 1e-6 and iteration counts within two."""
    system = contact_system
    B = np.stack([synthetic.rhs(system.n, seed=120 + c) for c in range(12)])
    s4 = _solver(system, dict(CHOSEN, rhs_group=4))
    s16 = _solver(system, dict(CHOSEN, rhs_group=16))
    X4, X16 = s4.solve_multi(B), s16.solve_multi(B)
    i4, i16 = s4.get_info()["rhs_iterations"], s16.get_info()["rhs_iterations"]
    for c in range(12):
        assert np.linalg.norm(X16[c] - X4[c]) <= 1e-6 * np.linalg.norm(X4[c])
        assert abs(i4[c] - i16[c]) <= 2


@pytest.mark.parametrize("nrhs", [1, 6, 16])
def test_tcgen05_wide_apply_matches_mma_sync(contact_system, nrhs):
    """The sixteen-wide apply on the fifth-generation tensor cores (full binary16 inverses in the
    tcgen05 operand layout, FP32 accumulation in tensor memory) is the same algorithm as the
    mma.sync one: every column meets the tolerance, within 1e-6 of it, iteration counts within two;
    repeated solves (graph replay) and solves after a refactorization give the same bits."""
    system = contact_system
    A = system.scipy()
    B = np.stack([synthetic.rhs(system.n, seed=200 + c) for c in range(nrhs)])
    sm = _solver(system, dict(CHOSEN, rhs_group=16))
    st = _solver(system, dict(CHOSEN, rhs_group=16, wide_apply="tcgen05"))
    Xm, Xt = sm.solve_multi(B), st.solve_multi(B)
    im, it = sm.get_info()["rhs_iterations"], st.get_info()["rhs_iterations"]
    assert all(v == "Reach relative tolerance" for v in st.get_info()["rhs_status"])
    for c in range(nrhs):
        assert np.linalg.norm(A @ Xt[c] - B[c]) <= 5e-8 * np.linalg.norm(B[c])
        assert np.linalg.norm(Xt[c] - Xm[c]) <= 1e-6 * np.linalg.norm(Xm[c])
        assert abs(im[c] - it[c]) <= 2
    np.testing.assert_array_equal(st.solve_multi(B), Xt)
    st.factorize(A)
    np.testing.assert_array_equal(st.solve_multi(B), Xt)


def test_wide_apply_is_validated():
    from polysolve_b200 import MasError

    s = Solver.create("MAS", "")
    with pytest.raises(MasError):
        s.set_parameters({"MAS": {"wide_apply": "wgmma"}})


def test_rhs_group_is_validated():
    from polysolve_b200 import MasError

    s = Solver.create("MAS", "")
    with pytest.raises(MasError):
        s.set_parameters({"MAS": {"rhs_group": 8}})
