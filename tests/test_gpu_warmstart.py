"""Learned warm start on the GPU: the features, the network and the Galerkin combination
against the NumPy oracle, and sequences solved through the public API."""

import numpy as np
import pytest
import scipy.sparse.linalg as sla

from oracle import warmstart_oracle as WO
from polysolve_b200 import Solver, synthetic
from polysolve_b200 import warmstart as W
from polysolve_b200.sequence import solve_sequence

pytestmark = pytest.mark.gpu

PARAMS = {"block_dim": 3, "relative_tolerance": 1e-8, "absolute_tolerance": 0.0, "precision": "fp16",
          "true_residual_period": 50, "check_period": 1}


def _exact_sequence(N, steps, seed):
    systems, rhs, xs = [], [], []
    for k in range(steps):
        s, b = synthetic.workload_sequence60(k, seed=seed, N=N)
        A = s.scipy().tocsc()
        systems.append(s)
        rhs.append(b)
        xs.append(sla.splu(A).solve(b))
    return systems, rhs, xs


def _solver(system, initial_guess="learned"):
    s = Solver.create("MAS", "")
    s.set_parameters({"MAS": dict(PARAMS, initial_guess=initial_guess)})
    s.set_positions(system.positions)
    s.analyze_pattern(system.scipy(), system.n)
    return s


def _random_params(seed):
    return (0.3 * np.random.default_rng(seed).standard_normal(W.PARAMS)).astype(np.float32)


@pytest.mark.parametrize("params", ["random", "shipped"])
def test_prediction_matches_oracle(params):
    systems, rhs, xs = _exact_sequence(7, 5, seed=11)
    A = systems[4].scipy().tocsr()
    b, x1, x2, x3, x4 = rhs[4], xs[3], xs[2], xs[1], xs[0]
    s = _solver(systems[4])
    s.factorize(systems[4].scipy())
    prm = _random_params(5) if params == "random" else W.default_weights()
    s.set_warm_start_model(prm)
    d = s.debug_warm_start(b, x1, x2, x3, x4)

    src, dst, w, D = WO.graph(A)
    # the first pass (history only) against the oracle's Galerkin rule, then the features from
    # the device's x_g
    basis = WO.galerkin_basis((x1, x2, x3, x4), np.zeros_like(b))
    yh, _, _, _, _ = WO.galerkin(A, b, x1, x2, np.zeros_like(b), x3, x4)
    xg_orc = sum(yi * vi for yi, vi in zip(yh, basis))
    xg = sum(yi * vi for yi, vi in zip(d["coef_history"], basis))
    assert np.linalg.norm(xg - xg_orc) <= 1e-7 * np.linalg.norm(xg_orc)
    raw, sums = WO.features(A, b, x1, x2, D, xg)
    scale = np.maximum(np.abs(raw).max(axis=0), 1e-300)
    assert np.all(np.abs(d["features"] - raw) <= 1e-6 * scale + 1e-6 * np.abs(raw))
    assert np.allclose(d["sums"], sums, rtol=1e-10)
    # bf16 hidden states: the tolerance covers rounding-boundary flips from the summation order
    c_orc = WO.forward_device(prm, raw.astype(np.float32), sums, src, dst, w).reshape(-1)
    assert np.linalg.norm(d["c"] - c_orc) <= 2e-2 * np.linalg.norm(c_orc)
    y, e, e1, fb, rank = WO.galerkin(A, b, x1, x2, d["c"], x3, x4)
    assert d["fallback"] == fb and d["rank"] == rank
    # the 5 x 5 system can be ill-conditioned (the differences shrink with the step): compare the
    # starting guesses and their energies rather than the coefficients
    x0 = sum(yi * vi for yi, vi in zip(y, WO.galerkin_basis((x1, x2, x3, x4), d["c"])))
    assert np.linalg.norm(d["x0"] - x0) <= 1e-7 * np.linalg.norm(x0)
    assert abs(d["energy"] - e) <= 1e-7 * abs(e)
    assert d["energy"] <= d["energy_previous"]
    # fewer kept solutions: the missing differences are dropped
    d2 = s.debug_warm_start(b, x1, x2)
    y2, e2, _, _, rank2 = WO.galerkin(A, b, x1, x2, d2["c"])
    assert d2["rank"] == rank2 <= 3 and abs(d2["energy"] - e2) <= 1e-7 * abs(e2)
    assert d["energy"] <= d2["energy"] + 1e-12 * abs(d2["energy"])


def test_learned_sequence_converges_and_beats_extrapolation():
    N, steps, seed = 12, 8, 3
    systems = [synthetic.workload_sequence60(k, seed=seed, N=N) for k in range(steps)]
    mats, rhs = [s.scipy() for s, _ in systems], [b for _, b in systems]
    totals = {}
    for mode in ("extrapolate", "learned"):
        s = _solver(systems[0][0], "learned" if mode == "learned" else "input")
        if mode == "learned":
            s.set_warm_start_model()
        res = solve_sequence(s, mats, rhs, mode)
        assert all(r["status"] == "Reach relative tolerance" for r in res)
        assert all(r["rel"] <= 5e-8 for r in res)
        if mode == "learned":
            assert [r["x0_source"] for r in res[:3]] == ["zero", "previous", "learned"]
            assert all(r["x0_source"].startswith(("learned", "previous")) for r in res[2:])
            info = s.get_info({})
            assert info["warm_start"]["predicted"] and info["warm_start"]["energy"] <= \
                info["warm_start"]["energy_previous"]
        totals[mode] = sum(r["iterations"] for r in res[2:])
    assert totals["learned"] <= totals["extrapolate"], totals


def test_fallbacks_and_history():
    systems = [synthetic.workload_sequence60(k, seed=4, N=6) for k in range(4)]
    s = _solver(systems[0][0])
    x = np.zeros(systems[0][0].n)
    sources = []
    for sk, bk in systems[:3]:  # no model: zero, then the previous solution
        s.factorize(sk.scipy())
        s.solve(bk, x)
        sources.append(s.get_info({})["x0_source"])
    assert sources == ["zero", "previous", "previous"]
    s.set_warm_start_model(_random_params(1))
    s.factorize(systems[3][0].scipy())
    s.solve(systems[3][1], x)
    assert s.get_info({})["x0_source"].startswith(("learned", "previous"))
    # several right-hand sides start from zero and leave the history alone
    B = np.stack([systems[3][1], 2.0 * systems[3][1]])
    X = s.solve_multi(B)
    assert np.allclose(X[1], 2.0 * X[0], rtol=1e-6, atol=1e-12 * np.abs(X[0]).max())
    s.solve(systems[3][1], x)
    assert s.get_info({})["x0_source"].startswith(("learned", "previous"))
    s.reset_warm_start()
    s.solve(systems[3][1], x)
    assert s.get_info({})["x0_source"] == "zero"
    # a different pattern forgets the kept solutions
    other, b2 = synthetic.workload_sequence60(0, seed=4, N=5)
    s.set_positions(other.positions)
    s.factorize(other.scipy())
    x2 = np.zeros(other.n)
    s.solve(b2, x2)
    assert s.get_info({})["x0_source"] == "zero"


def test_bad_model_rejected():
    sk, _ = synthetic.workload_sequence60(0, seed=1, N=4)
    s = _solver(sk)
    with pytest.raises(Exception):
        s.set_warm_start_model(np.zeros(10, dtype=np.float32))
    bad = _random_params(2)
    bad[7] = np.nan
    with pytest.raises(Exception):
        s.set_warm_start_model(bad)


def test_learned_mode_other_block_sizes_fall_back_to_previous():
    """The network is defined for three displacement components per vertex: with block_dim 1
    the learned mode starts from the previous solution and still meets the tolerance."""
    systems = [synthetic.workload_sequence60(k, seed=6, N=5) for k in range(3)]
    s = Solver.create("MAS", "")
    s.set_parameters({"MAS": dict(PARAMS, block_dim=1, initial_guess="learned")})
    s.analyze_pattern(systems[0][0].scipy(), systems[0][0].n)
    s.set_warm_start_model()
    res = solve_sequence(s, [sk.scipy() for sk, _ in systems], [bk for _, bk in systems], "learned")
    assert [r["x0_source"] for r in res] == ["zero", "previous", "previous"]
    assert all(r["rel"] <= 5e-8 for r in res)
