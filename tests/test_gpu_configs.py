"""Parity at the benchmark configurations' own sizes (not only on toy grids).

* 20^3 elasticity, 27,783 DOF (the CPU-runnable configuration): the reference's algorithm (x0 = 0,
  FP64 MAS, true residual every 4, test every 10) gives the oracle's iteration count and a solution
  within 1e-6 of the oracle's and of an FP64 sparse LU (scipy ``splu``, the CHOLMOD stand-in); the
  chosen configuration (binary16 inverses, true residual every 50, test every iteration) is within
  2 iterations of the oracle run the same way and within 1e-6 of the LU solution.
* 20^3 jittered mesh with lognormal stiffness plus 20,000 contact couplings and 16 right-hand sides
  through ``solve_multi``: every column within 1e-6 of the LU solution.
* 80^3 jittered mesh with lognormal stiffness, 1,594,323 DOF (the headline system): reference mode
  gives the oracle's iteration count and a solution within 1e-6 of the oracle's.
* The committed golden fixtures (oracle outputs on fixed inputs, ``tests/golden``): ordering and
  coarse maps bit-exact, the MAS apply within 1e-10, reference-mode PCG with the same iteration
  count and a solution within 1e-6.

Reference semantics: MASSolver.cu:469-595 (PCG), tests/test_linear_solver.cpp:103-164 (residual
style).
"""

from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

from oracle import oracle as O
from polysolve_b200 import Solver, synthetic

from .helpers import oracle_for, oracle_to_padded, padded_to_oracle, real_to_padded_nodes

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden"

REFERENCE_MODE = {}
CHOSEN_MODE = {"precision": "fp16", "true_residual_period": 50, "check_period": 1}


def _solver(system, params):
    s = Solver.create("MAS", "")
    p = {"block_dim": 3, "relative_tolerance": 1e-8, "absolute_tolerance": 0.0}
    p.update(params)
    s.set_parameters({"MAS": p})
    s.set_positions(system.positions)
    A = system.scipy()
    s.analyze_pattern(A, A.shape[0])
    s.factorize(A)
    return s


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.fixture(scope="module")
def cpu20():
    import scipy.sparse.linalg as sla

    system = synthetic.workload_cpu20()
    b = synthetic.rhs(system.n, seed=0)
    lu = sla.splu(system.scipy().tocsc())
    return system, b, lu.solve(b)


def test_cpu20_reference_mode_matches_oracle_and_lu(cpu20):
    system, b, x_lu = cpu20
    s = _solver(system, REFERENCE_MODE)
    x = np.zeros(system.n)
    s.solve(b, x)
    info = s.get_info()
    orc, _ = oracle_for(system, s)
    xo, oinfo = orc.pcg(b, rel_tol=1e-8, abs_tol=0.0)
    assert info["solver_status"] == oinfo["solver_status"] == "Reach relative tolerance"
    assert info["solver_iter"] == oinfo["solver_iter"]
    assert _rel(x, xo) <= 1e-6
    assert _rel(x, x_lu) <= 1e-6
    assert np.linalg.norm(system.scipy() @ x - b) <= 1e-8 * np.linalg.norm(b)


def test_cpu20_chosen_mode_matches_oracle_and_lu(cpu20):
    system, b, x_lu = cpu20
    s = _solver(system, CHOSEN_MODE)
    x = np.zeros(system.n)
    s.solve(b, x)
    info = s.get_info()
    orc, _ = oracle_for(system, s)
    xo, oinfo = orc.pcg(b, rel_tol=1e-8, abs_tol=0.0, true_residual_period=50, check_period=1, mas_fp32=16)
    assert info["solver_status"] == "Reach relative tolerance"
    assert abs(info["solver_iter"] - oinfo["solver_iter"]) <= 2
    assert _rel(x, x_lu) <= 1e-6
    assert _rel(x, xo) <= 1e-6


def test_contact20_sixteen_right_hand_sides_match_lu():
    import scipy.sparse.linalg as sla

    system = synthetic.workload_contact80(seed=0, N=20, pairs=20000)
    A = system.scipy().tocsc()
    B = synthetic.rhs(system.n, seed=5, count=16)
    lu = sla.splu(A)
    s = _solver(system, CHOSEN_MODE)
    X = s.solve_multi(B)
    info = s.get_info()
    assert all(st == "Reach relative tolerance" for st in info["rhs_status"]), info["rhs_status"]
    for k in range(16):
        x_lu = lu.solve(B[k])
        assert np.linalg.norm(A @ X[k] - B[k]) <= 2e-8 * np.linalg.norm(B[k]), k
        assert _rel(X[k], x_lu) <= 1e-6, k


def test_grid80_reference_mode_matches_oracle():
    """The 1.6 M-DOF headline system: the CPU oracle takes a few seconds on the host's cores."""
    system = synthetic.workload_grid80()
    b = synthetic.rhs(system.n, seed=0)
    s = _solver(system, REFERENCE_MODE)
    x = np.zeros(system.n)
    s.solve(b, x)
    info = s.get_info()
    orc, _ = oracle_for(system, s)
    xo, oinfo = orc.pcg(b, rel_tol=1e-8, abs_tol=0.0)
    assert info["solver_status"] == oinfo["solver_status"] == "Reach relative tolerance"
    assert info["solver_iter"] == oinfo["solver_iter"]
    assert _rel(x, xo) <= 1e-6


@pytest.mark.parametrize("name", ["grid3", "grid4_jitter", "grid5_contact"])
def test_golden_fixtures_on_gpu(name):
    d = np.load(GOLDEN / f"{name}.npz")
    n = int(d["n"])
    system = synthetic.System(n=n, outer=d["outer"], inner=d["inner"], vals=d["vals"], positions=d["positions"])
    s = _solver(system, REFERENCE_MODE)
    padded = s.ordering()
    np.testing.assert_array_equal(padded, d["padded"])
    sz = s.sizes()
    assert sz["level_num"] == int(d["level_num"])
    assert sz["cco_nums"] == [int(v) for v in d["cco_nums"]]
    r2p = real_to_padded_nodes(padded, d["perm"])
    cmap = s.coarse_map()[r2p][:, : int(d["level_num"])]
    np.testing.assert_array_equal(cmap, d["cmap"][:, : int(d["level_num"])])
    z = padded_to_oracle(s.debug_apply(oracle_to_padded(d["r"], r2p, 3, sz["nodes"])), r2p, 3)
    assert _rel(z, d["z"]) <= 1e-10
    x = np.zeros(n)
    s.solve(d["b"], x)
    assert s.get_info()["solver_iter"] == int(d["iters"])
    assert _rel(x, d["x"]) <= 1e-6
