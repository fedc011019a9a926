"""Failure detection without a GPU fault: the reference reports an allocation failure as
mas::CudaOutOfMemoryError with the requested and free MB (mas_utils/CudaUtils.cuh:41-124) and has no
device-side waits. Here both failure paths are made on purpose, in forms that fault nothing:

* an allocation failure injected on the host (``debug_fail_allocation``: the N-th next device
  allocation reports out-of-memory without calling cudaMalloc);
* a bounded device-side wait that runs out: ``device_wait_limit 0`` makes every mbarrier wait of
  the MAS apply give up at once; the kernel records MAS_ERR_TIMEOUT, drains its own bulk copies
  (with the default limit) and returns, and the solve stops with that status.

After each failure the same handle must work again and give the result of a fresh solver.
"""

from __future__ import annotations

import numpy as np
import pytest

from polysolve_b200 import CudaOutOfMemoryError, MasError, Solver, synthetic
from polysolve_b200.solver import MAS_ERR_TIMEOUT, debug_fail_allocation

pytestmark = pytest.mark.gpu


def _solver(system, params=None):
    s = Solver.create("MAS", "")
    p = {"block_dim": 3, "relative_tolerance": 1e-8, "absolute_tolerance": 0.0}
    p.update(params or {})
    s.set_parameters({"MAS": p})
    s.set_positions(system.positions)
    return s


@pytest.fixture(autouse=True)
def _hook_off():
    debug_fail_allocation(-1)
    yield
    debug_fail_allocation(-1)


@pytest.mark.parametrize("after", [0, 3, 12])
def test_injected_allocation_failure_raises_oom_and_handle_recovers(after):
    system = synthetic.elasticity(7, young_sigma=1.0, jitter=0.2, seed=50)
    b = synthetic.rhs(system.n, seed=50)
    ref = _solver(system)
    ref.factorize(system.scipy())
    x_ref = np.zeros(system.n)
    ref.solve(b, x_ref)

    s = _solver(system)
    debug_fail_allocation(after)
    with pytest.raises(CudaOutOfMemoryError) as e:
        s.factorize(system.scipy())
    msg = str(e.value)
    assert msg.startswith("[MAS] Failed to allocate") and "MB" in msg and "free" in msg, msg
    # The hook fired once and is off again: the same handle factorizes and solves as a fresh one.
    s.factorize(system.scipy())
    x = np.zeros(system.n)
    s.solve(b, x)
    np.testing.assert_array_equal(x, x_ref)


def test_injected_allocation_failure_during_solve_buffers():
    """A failure while the warm-start scratch is allocated (inside solve) leaves the handle usable."""
    seq = [synthetic.workload_sequence60(k, seed=3, N=6) for k in range(3)]
    s = _solver(seq[0][0], {"precision": "fp16", "initial_guess": "learned"})
    s.set_warm_start_model()
    xs = []
    for k, (sk, bk) in enumerate(seq):
        s.factorize(sk.scipy())
        x = np.zeros(sk.n)
        if k == 2:
            debug_fail_allocation(0)
            with pytest.raises(CudaOutOfMemoryError):
                s.solve(bk, x)
            debug_fail_allocation(-1)
        s.solve(bk, x)
        assert s.get_info()["solver_status"] == "Reach relative tolerance"
        A = sk.scipy()
        assert np.linalg.norm(A @ x - bk) <= 2e-8 * np.linalg.norm(bk)
        xs.append(x)


@pytest.mark.parametrize("precision", ["fp64", "fp16"])
@pytest.mark.parametrize("graphs", [True, False])
def test_device_wait_timeout_is_reported_and_handle_recovers(precision, graphs):
    system = synthetic.elasticity(9, young_sigma=1.0, jitter=0.2, seed=51)
    b = synthetic.rhs(system.n, seed=51)
    params = {"precision": precision, "cuda_graphs": graphs, "check_period": 1, "true_residual_period": 50}
    ref = _solver(system, params)
    ref.factorize(system.scipy())
    x_ref = np.zeros(system.n)
    ref.solve(b, x_ref)

    s = _solver(system, params)
    s.factorize(system.scipy())
    s.set_parameters({"MAS": {"device_wait_limit": 0}})
    x = np.zeros(system.n)
    with pytest.raises(MasError) as e:
        s.solve(b, x)
    assert e.value.code == MAS_ERR_TIMEOUT and "timed out" in str(e.value)
    # Back to the default limit: the handle solves exactly as a fresh one.
    s.set_parameters({"MAS": {"device_wait_limit": 1 << 20}})
    s.solve(b, x)
    assert s.get_info()["solver_status"] == "Reach relative tolerance"
    np.testing.assert_array_equal(x, x_ref)


@pytest.mark.parametrize("group,wide_apply", [(4, "mma_sync"), (16, "mma_sync"), (16, "tcgen05")])
def test_device_wait_timeout_several_right_hand_sides(group, wide_apply):
    system = synthetic.elasticity(8, young_sigma=1.0, jitter=0.2, seed=52)
    B = synthetic.rhs(system.n, seed=52, count=4)
    params = {"precision": "fp16", "check_period": 1, "true_residual_period": 50, "rhs_group": group,
              "wide_apply": wide_apply}
    s = _solver(system, params)
    s.factorize(system.scipy())
    X_ref = s.solve_multi(B)
    s.set_parameters({"MAS": {"device_wait_limit": 0}})
    with pytest.raises(MasError) as e:
        s.solve_multi(B)
    assert e.value.code == MAS_ERR_TIMEOUT
    s.set_parameters({"MAS": {"device_wait_limit": 1 << 20}})
    np.testing.assert_array_equal(s.solve_multi(B), X_ref)


def test_device_wait_limit_is_validated():
    s = Solver.create("MAS", "")
    with pytest.raises(MasError):
        s.set_parameters({"MAS": {"device_wait_limit": -1}})
