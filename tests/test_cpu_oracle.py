"""The CPU oracle: pinned against an independent dense construction of the MAS operator, against
the committed golden fixtures, and checked for the reference's PCG semantics."""

from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

from oracle import oracle as O
from polysolve_b200 import synthetic

GOLDEN = Path(__file__).resolve().parent / "golden"


def _oracle(N, bd=3, **kw):
    s = synthetic.elasticity(N, **kw)
    V = -(-s.n // bd)
    if bd == 3:
        iso = O.isolated_blocks(s.outer, s.inner, s.n, 3)
        perm, off = O.morton_order(s.positions, iso)
    else:
        perm = np.arange(V, dtype=np.int32)
        off = np.append(np.arange(0, V, 32), V).astype(np.int32)
    return s, O.MasOracle(s.outer, s.inner, s.vals, s.n, bd, perm, off)


@pytest.mark.parametrize("N,bd,kw", [
    (3, 3, {}),
    (4, 3, dict(young_sigma=1.0, jitter=0.2)),
    (5, 3, dict(young_sigma=1.0, jitter=0.2, contact_pairs=40)),
    (4, 1, dict(young_sigma=1.0)),
    (4, 2, dict(young_sigma=1.0)),
])
def test_apply_equals_dense_definition(N, bd, kw):
    """z = sum_l P_l (P_l^T A P_l | banks)^-1 P_l^T r, built densely in numpy."""
    s, orc = _oracle(N, bd, **kw)
    Minv = O.dense_mas_operator(orc)
    r = np.random.default_rng(1).standard_normal(orc.s.V * bd)
    z = orc.apply(r)
    assert np.linalg.norm(z - Minv @ r) <= 1e-10 * np.linalg.norm(Minv @ r)
    assert np.abs(Minv - Minv.T).max() <= 1e-10 * np.abs(Minv).max()


def test_inverses_are_inverses():
    s, orc = _oracle(4, 3, young_sigma=1.0, jitter=0.2)
    assert orc.inverse_ok
    rows, cols, vals = orc.bsr()
    inv = orc.inverses()
    N = 96
    # Level-0 matrix of bank 0: the partition's diagonal block of A.
    r2p, _ = orc.maps()
    nodes = [v for v in range(orc.s.V) if r2p[v] // 32 == 0]
    A0 = np.zeros((N, N))
    for v in nodes:
        for k in range(rows[v], rows[v + 1]):
            w = cols[k]
            if r2p[w] // 32 == 0:
                A0[(r2p[v] % 32) * 3:(r2p[v] % 32) * 3 + 3, (r2p[w] % 32) * 3:(r2p[w] % 32) * 3 + 3] = vals[k]
    for i in range(N):
        if A0[i, i] == 0:
            A0[i, i] = 1
    M = np.zeros((N, N))
    M[np.triu_indices(N)] = inv[0]
    M = M + M.T - np.diag(np.diag(M))
    assert np.linalg.norm(M @ A0 - np.eye(N)) <= 1e-9 * N


def test_reference_pcg_semantics():
    s, orc = _oracle(6, 3, young_sigma=1.0, jitter=0.2)
    b = synthetic.rhs(s.n, 3)
    x, info = orc.pcg(b, rel_tol=1e-8, abs_tol=0.0)
    A = s.scipy()
    assert info["solver_status"] == "Reach relative tolerance"
    assert info["solver_iter"] % 10 == 0  # convergence only tested every 10 iterations
    assert np.linalg.norm(A @ x - b) <= 1e-8 * np.linalg.norm(b)
    # solver_error is the absolute ||r|| (MASSolver.cu:551)
    assert info["solver_error"] <= 1e-8 * np.sqrt(info["rr0"])
    # absolute tolerance status
    x2, info2 = orc.pcg(b, rel_tol=0.0, abs_tol=1e-6)
    assert info2["solver_status"] == "Reach absolute tolerance"
    # max iterations
    x3, info3 = orc.pcg(b, rel_tol=1e-14, abs_tol=0.0, max_iter=7)
    assert info3["solver_status"] == "Reach max iterations" and info3["solver_iter"] == 7
    # NaN -> invalid initial residual
    bn = b.copy()
    bn[0] = np.nan
    _, info4 = orc.pcg(bn)
    assert info4["solver_status"] == "Invalid initial residual"


def test_preconditioned_norm_and_modes():
    s, orc = _oracle(6, 3, young_sigma=1.0, jitter=0.2)
    b = synthetic.rhs(s.n, 4)
    A = s.scipy()
    for kw in [dict(use_preconditioned_residual_norm=True), dict(true_residual_period=50, check_period=1),
               dict(true_residual_period=50, check_period=1, mas_fp32=True, polak_ribiere=True)]:
        x, info = orc.pcg(b, rel_tol=1e-9, abs_tol=0.0, **kw)
        assert info["solver_status"] == "Reach relative tolerance", kw
        assert np.linalg.norm(A @ x - b) <= 1e-7 * np.linalg.norm(b), kw


def test_half_round_is_ieee_nearest_even():
    """The oracle's binary16 rounding equals IEEE conversion (numpy float32 -> float16), including
    ties, subnormals and the smallest subnormal's half-way region."""
    rng = np.random.default_rng(0)
    v = np.concatenate([
        rng.standard_normal(20000).astype(np.float32) * np.float32(2.0) ** rng.integers(-30, 16, 20000),
        np.float32([2.0 ** -24, 2.0 ** -25, 1.5 * 2.0 ** -25, 0.75 * 2.0 ** -24, 2.0 ** -26, 1.0 + 2.0 ** -11,
                    1.0 + 3 * 2.0 ** -11, 2048.0 + 1.0, 2048.0 + 3.0, 6.0e-5, -6.0e-8, 32767.0, 65504.0]),
    ]).astype(np.float32)
    got = O.half_round(v)
    with np.errstate(over="ignore"):
        want = v.astype(np.float16).astype(np.float32)
    np.testing.assert_array_equal(got, want)


def test_fp16_storage_apply_close_to_fp64():
    """Scaled binary16 inverses change the MAS apply by about the format's precision (2^-11)."""
    s, orc = _oracle(6, 3, young_sigma=1.0, jitter=0.2)
    # r = A x: every row (stiff rows and unit Dirichlet rows alike) contributes O(|x|) to z.
    r = orc.spmv(np.random.default_rng(3).standard_normal(orc.s.V * 3))
    z64 = orc.apply(r)
    z16 = orc.apply(r, storage=16)
    z32 = orc.apply(r, storage=1)
    e16 = np.linalg.norm(z16 - z64) / np.linalg.norm(z64)
    e32 = np.linalg.norm(z32 - z64) / np.linalg.norm(z64)
    assert 0 < e32 < 1e-6
    assert 1e-6 < e16 < 2e-3
    b = synthetic.rhs(s.n, 4)
    x, info = orc.pcg(b, rel_tol=1e-9, abs_tol=0.0, true_residual_period=50, check_period=1, mas_fp32=16)
    assert info["solver_status"] == "Reach relative tolerance"
    assert np.linalg.norm(s.scipy() @ x - b) <= 1e-7 * np.linalg.norm(b)


def test_initial_guess_is_used_when_asked():
    s, orc = _oracle(6, 3, young_sigma=1.0)
    b = synthetic.rhs(s.n, 5)
    x, info = orc.pcg(b, rel_tol=1e-9, abs_tol=0.0, check_period=1)
    x2, info2 = orc.pcg(b, x0=x, rel_tol=1e-9, abs_tol=0.0, check_period=1, use_initial_guess=True)
    assert info2["solver_iter"] < info["solver_iter"]
    # reference behaviour: the caller's x is ignored (MASSolver.cu:395-398)
    x3, info3 = orc.pcg(b, x0=x, rel_tol=1e-9, abs_tol=0.0, check_period=1)
    assert info3["solver_iter"] == info["solver_iter"]


def test_absolute_alpha_guard_stalls_like_reference():
    """alpha = 0 once |p.Ap| < 1e-20 (MASSolver.cu:53): on this small, stiff system the iteration
    stops improving near 5e-10 relative residual and runs to max_iter."""
    s, orc = _oracle(6, 3, young_sigma=1.0)
    b = synthetic.rhs(s.n, 5)
    x, info = orc.pcg(b, rel_tol=1e-11, abs_tol=0.0, check_period=1, max_iter=200)
    assert info["solver_status"] == "Reach max iterations"
    rel = np.linalg.norm(s.scipy() @ x - b) / np.linalg.norm(b)
    assert 1e-11 < rel < 1e-9


def test_jacobi_cg_baseline():
    s = synthetic.workload_cpu20()
    b = synthetic.rhs(s.n, 0)
    x, it, rel = O.jacobi_pcg(s.outer, s.inner, s.vals, s.n, b, 1e-8)
    assert rel < 1e-8
    assert np.linalg.norm(s.scipy() @ x - b) <= 1.01e-8 * np.linalg.norm(b)


def test_scipy_cross_check_small():
    """Direct FP64 solve (scipy splu) as the CHOLMOD stand-in: solution error <= 1e-6."""
    import scipy.sparse.linalg as spla

    s, orc = _oracle(5, 3, young_sigma=1.0, jitter=0.2)
    b = synthetic.rhs(s.n, 6)
    x, info = orc.pcg(b, rel_tol=1e-10, abs_tol=0.0)
    xd = spla.splu(s.scipy().tocsc()).solve(b)
    assert np.linalg.norm(x - xd) <= 1e-6 * np.linalg.norm(xd)


@pytest.mark.parametrize("name", ["grid3", "grid4_jitter", "grid5_contact"])
def test_golden_fixtures(name):
    d = np.load(GOLDEN / f"{name}.npz")
    n = int(d["n"])
    iso = O.isolated_blocks(d["outer"], d["inner"], n, 3)
    padded = O.morton_padded(d["positions"], iso)
    np.testing.assert_array_equal(padded, d["padded"])
    perm, offsets = O.partition_from_padded(padded)
    np.testing.assert_array_equal(perm, d["perm"])
    orc = O.MasOracle(d["outer"], d["inner"], d["vals"], n, 3, perm, offsets)
    r2p, cmap = orc.maps()
    np.testing.assert_array_equal(r2p, d["r2p"])
    np.testing.assert_array_equal(cmap[:, : orc.s.level_num], d["cmap"][:, : orc.s.level_num])
    np.testing.assert_array_equal(orc.s.cco_nums, d["cco_nums"])
    z = orc.apply(d["r"])
    assert np.linalg.norm(z - d["z"]) <= 1e-12 * np.linalg.norm(d["z"])
    x, info = orc.pcg(d["b"], rel_tol=1e-8, abs_tol=0.0)
    assert info["solver_iter"] == int(d["iters"])
    assert np.linalg.norm(x - d["x"]) <= 1e-9 * np.linalg.norm(d["x"])


def test_golden_generator_inputs_stable():
    """The synthetic generator still produces the fixtures' matrices (seeded, thread-independent)."""
    d = np.load(GOLDEN / "grid4_jitter.npz")
    s = synthetic.elasticity(4, young_sigma=1.0, jitter=0.2, seed=2)
    np.testing.assert_array_equal(s.outer, d["outer"])
    np.testing.assert_array_equal(s.inner, d["inner"])
    np.testing.assert_array_equal(s.vals, d["vals"])


def test_cpu20_oracle_matches_sparse_lu():
    """The CPU-runnable configuration (20^3, 27,783 DOF, E 1e5, Dirichlet x = 0, b ~ N(0,1)): the
    oracle's reference-mode PCG and the Jacobi-PCG baseline both reach 1e-8 and agree with an FP64
    sparse LU (the CHOLMOD stand-in) to 1e-6."""
    import scipy.sparse.linalg as sla

    s = synthetic.workload_cpu20()
    b = synthetic.rhs(s.n, seed=0)
    A = s.scipy().tocsc()
    x_lu = sla.splu(A).solve(b)
    iso = O.isolated_blocks(s.outer, s.inner, s.n, 3)
    perm, off = O.morton_order(s.positions, iso)
    orc = O.MasOracle(s.outer, s.inner, s.vals, s.n, 3, perm, off)
    x, info = orc.pcg(b, rel_tol=1e-8, abs_tol=0.0)
    assert info["solver_status"] == "Reach relative tolerance"
    assert info["solver_iter"] % 10 == 0
    assert np.linalg.norm(A @ x - b) <= 1e-8 * np.linalg.norm(b)
    assert np.linalg.norm(x - x_lu) <= 1e-6 * np.linalg.norm(x_lu)
    xj, itj, rel = O.jacobi_pcg(s.outer, s.inner, s.vals, s.n, b, 1e-8)
    assert rel <= 1e-8 and itj > info["solver_iter"]
    assert np.linalg.norm(xj - x_lu) <= 1e-6 * np.linalg.norm(x_lu)
