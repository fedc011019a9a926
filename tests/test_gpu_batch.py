"""Batched solves of independent systems (`mas_solve_batch`) against one-at-a-time solves."""

from __future__ import annotations

import numpy as np
import pytest

from polysolve_b200 import MasError, Solver, solve_batch, synthetic

pytestmark = pytest.mark.gpu

PARAMS = {"block_dim": 3, "relative_tolerance": 1e-8, "absolute_tolerance": 0.0, "precision": "fp16",
          "true_residual_period": 50, "check_period": 1}
FUSED = dict(PARAMS, batch_launch="fused")


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


def _single(s, b, x0=None):
    x = np.zeros_like(b) if x0 is None else x0.copy()
    s.solve(b, x)
    info = s.get_info({})
    return x, info["solver_iter"], info["solver_status"], info["solver_error"]


def _mixed_params():
    """Per-system settings a fused batch may mix (the true-residual period, graph length, SpMV
    unroll, precision and block_dim are shared)."""
    return [dict(FUSED), dict(FUSED, max_iter=7), dict(FUSED, relative_tolerance=1e-4),
            dict(FUSED, beta="polak_ribiere"), dict(FUSED, check_period=3, use_preconditioned_residual_norm=True),
            dict(FUSED, initial_guess="input"), dict(FUSED, absolute_tolerance=1e-3), dict(FUSED)]


def test_fused_batch_bit_identical_to_single_solves_mixed_settings(systems):
    """One launch per PCG phase for all systems (batch_launch fused): each system's
    iterates are those of its own solve bit for bit, with per-system tolerances, iteration caps,
    beta formula, residual norm and initial guess."""
    params = _mixed_params()
    solvers = [_solver(s, p) for s, p in zip(systems, params)]
    bs = [synthetic.rhs(s.n, seed=40 + k) for k, s in enumerate(systems)]
    x0s = [np.random.default_rng(k).standard_normal(s.n) * 0.1 for k, s in enumerate(systems)]
    ref = [_single(s, b, x0) for s, b, x0 in zip(solvers, bs, x0s)]
    for threads, groups in ((0, 0), (1, 1), (3, 3), (0, 8)):
        for s in solvers:
            s.set_parameters({"MAS": {"batch_groups": groups}})
        xs = solve_batch(solvers, bs, [x0.copy() for x0 in x0s], threads=threads)
        for (xr, it, stat, err), x, s in zip(ref, xs, solvers):
            np.testing.assert_array_equal(x, xr)
            info = s.get_info({})
            assert (info["solver_iter"], info["solver_status"], info["solver_error"]) == (it, stat, err)
    assert solvers[1].get_info({})["solver_status"] == "Reach max iterations"
    assert solvers[1].get_info({})["solver_iter"] == 7


def test_fused_and_stream_batches_agree_and_mixed_modes_fall_back(systems):
    solvers = [_solver(s, FUSED) for s in systems]
    bs = [synthetic.rhs(s.n, seed=60 + k) for k, s in enumerate(systems)]
    fused = [x.copy() for x in solve_batch(solvers, bs)]
    launches0 = sum(s.get_info({})["kernel_launches_total"] for s in solvers)
    solve_batch(solvers, bs)
    fused_launches = sum(s.get_info({})["kernel_launches_total"] for s in solvers) - launches0
    for s in solvers:
        s.set_parameters({"MAS": {"batch_launch": "streams"}})
    launches0 = sum(s.get_info({})["kernel_launches_total"] for s in solvers)
    streams = solve_batch(solvers, bs)
    stream_launches = sum(s.get_info({})["kernel_launches_total"] for s in solvers) - launches0
    for a, c in zip(fused, streams):
        np.testing.assert_array_equal(a, c)
    # one launch per phase for the whole batch instead of one per system
    assert 0 < fused_launches < stream_launches / 2
    # one handle asking for streams: the whole batch takes the stream path, same bits
    for s in solvers:
        s.set_parameters({"MAS": {"batch_launch": "fused"}})
    solvers[2].set_parameters({"MAS": {"batch_launch": "streams"}})
    for a, c in zip(fused, solve_batch(solvers, bs)):
        np.testing.assert_array_equal(a, c)
    with pytest.raises(MasError):
        solvers[0].set_parameters({"MAS": {"batch_launch": "persistent"}})


def test_fused_batch_reuses_its_tables_across_calls_and_refactorizations(systems):
    solvers = [_solver(s, FUSED) for s in systems[:5]]
    bs = [synthetic.rhs(s.n, seed=80 + k) for k, s in enumerate(systems[:5])]
    first = [x.copy() for x in solve_batch(solvers, bs)]
    for a, c in zip(first, solve_batch(solvers, bs)):
        np.testing.assert_array_equal(a, c)
    # new values, same pattern and buffers: the kept launch tables serve the new inverses
    for s, sysm in zip(solvers, systems[:5]):
        s.factorize(sysm.scipy() * 2.0)
    ref = [_single(s, b)[0] for s, b in zip(solvers, bs)]
    for a, c, x1 in zip(ref, solve_batch(solvers, bs), first):
        np.testing.assert_array_equal(a, c)
        assert np.linalg.norm(c - 0.5 * x1) <= 1e-6 * np.linalg.norm(x1)
    # a different subset and order: its own launch tables
    sub = [solvers[3], solvers[0], solvers[4]]
    bsub = [bs[3], bs[0], bs[4]]
    for a, c in zip([ref[3], ref[0], ref[4]], solve_batch(sub, bsub)):
        np.testing.assert_array_equal(a, c)


def test_fused_batch_reports_a_bad_system_and_solves_the_others(systems):
    solvers = [_solver(s, FUSED) for s in systems[:4]]
    bs = [synthetic.rhs(s.n, seed=90 + k) for k, s in enumerate(systems[:4])]
    ref = [_single(s, b)[0] for s, b in zip(solvers, bs)]
    bad = bs[1].copy()
    bad[3] = np.nan
    xs = [np.zeros_like(b) for b in bs]
    with pytest.raises(MasError) as e:
        solve_batch(solvers, [bs[0], bad, bs[2], bs[3]], xs)
    assert "Invalid initial residual" in str(e.value)
    for k in (0, 2, 3):
        np.testing.assert_array_equal(xs[k], ref[k])
    # a system with the wrong length leaves the batch before any launch
    xs = [np.zeros_like(b) for b in bs]
    with pytest.raises(MasError):
        solve_batch(solvers, [bs[0], bs[1][:-3], bs[2], bs[3]], [xs[0], xs[1][:-3], xs[2], xs[3]])
    for k in (0, 2, 3):
        np.testing.assert_array_equal(xs[k], ref[k])


def test_fused_batch_timeout_is_reported_and_handles_recover(systems):
    from polysolve_b200.solver import MAS_ERR_TIMEOUT

    solvers = [_solver(s, FUSED) for s in systems[:3]]
    bs = [synthetic.rhs(s.n, seed=95 + k) for k, s in enumerate(systems[:3])]
    ref = [_single(s, b)[0] for s, b in zip(solvers, bs)]
    for s in solvers:
        s.set_parameters({"MAS": {"device_wait_limit": 0}})
    with pytest.raises(MasError) as e:
        solve_batch(solvers, bs)
    assert e.value.code == MAS_ERR_TIMEOUT
    for s in solvers:
        s.set_parameters({"MAS": {"device_wait_limit": 1 << 20}})
    for a, c in zip(ref, solve_batch(solvers, bs)):
        np.testing.assert_array_equal(a, c)


def test_fused_batch_device_pointers_match_host_arrays(systems):
    import torch

    from polysolve_b200 import solve_batch_device

    solvers = [_solver(s, FUSED) for s in systems]
    bs = [synthetic.rhs(s.n, seed=70 + k) for k, s in enumerate(systems)]
    host = [x.copy() for x in solve_batch(solvers, bs)]
    db = [torch.from_numpy(b).cuda() for b in bs]
    dx = [torch.zeros_like(t) for t in db]
    solve_batch_device(solvers, [t.data_ptr() for t in db], [t.data_ptr() for t in dx], [t.numel() for t in db])
    torch.cuda.synchronize()
    for a, t in zip(host, dx):
        np.testing.assert_array_equal(a, t.cpu().numpy())


def test_apply_items_per_warp_batches_match_single_solves(systems):
    """apply_items_per_warp (a launch shape: fewer, longer-lived apply CTAs) changes the apply's
    grid and so the grouping of its dot products; single solves, fused and stream batches with the
    same setting agree bit for bit, and every setting meets the tolerance."""
    bs = [synthetic.rhs(s.n, seed=110 + k) for k, s in enumerate(systems)]
    base = [_single(_solver(s), b)[0] for s, b in zip(systems, bs)]
    for ipw in (2, 4, 8):
        solvers = [_solver(s, dict(FUSED, apply_items_per_warp=ipw)) for s in systems]
        ref = [_single(s, b) for s, b in zip(solvers, bs)]
        fused = [x.copy() for x in solve_batch(solvers, bs)]
        for s in solvers:
            s.set_parameters({"MAS": {"batch_launch": "streams"}})
        streams = solve_batch(solvers, bs)
        for (xr, it, _, _), xf, xs, x1, sysm, b in zip(ref, fused, streams, base, systems, bs):
            np.testing.assert_array_equal(xf, xr)
            np.testing.assert_array_equal(xs, xr)
            A = sysm.scipy()
            assert np.linalg.norm(A @ xr - b) <= 5e-8 * np.linalg.norm(b)
            assert np.linalg.norm(xr - x1) <= 1e-6 * np.linalg.norm(x1)
    with pytest.raises(MasError):
        solvers[0].set_parameters({"MAS": {"apply_items_per_warp": 0}})
