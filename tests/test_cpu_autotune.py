"""The autotuner's search and cache logic with stand-in solvers and timed callables (no GPU)."""

import time

from polysolve_b200 import autotune


class FakeSolver:
    def __init__(self):
        self.params = {}

    def set_parameters(self, p):
        self.params.update(p["MAS"])


def test_poll_period_picks_the_fastest_and_leaves_it_set():
    solvers = [FakeSolver(), FakeSolver()]
    cost = {5: 0.03, 10: 0.005, 20: 0.02}

    def run():
        time.sleep(cost[solvers[0].params["poll_period"]])

    res = autotune.tune_poll_period(solvers, run, candidates=(5, 10, 20), repeats=2)
    assert res["best"] == 10 and set(res["ms"]) == {5, 10, 20}
    assert all(s.params["poll_period"] == 10 for s in solvers)


def test_threads_pick_the_fastest():
    res = autotune.tune_batch_threads(lambda t: time.sleep(0.004 * abs(t - 8) + 0.002), candidates=(2, 8, 32),
                                      repeats=2)
    assert res["best"] == 8


def test_cache_round_trip(tmp_path):
    path = tmp_path / "tune.json"
    cache = {autotune.signature([30, 10]): {"poll_period": 20, "threads": 16, "tables": {}}}
    autotune._store_cache(str(path), cache)
    assert autotune._load_cache(str(path)) == cache
    assert autotune.signature([10, 30]) == autotune.signature([30, 10])


def test_spmv_unroll_picks_the_fastest_and_leaves_it_set():
    solvers = [FakeSolver(), FakeSolver()]
    cost = {1: 0.02, 2: 0.012, 4: 0.004}

    def run():
        time.sleep(cost[solvers[0].params["spmv_unroll"]])

    res = autotune.tune_spmv_unroll(solvers, run, repeats=2)
    assert res["best"] == 4 and set(res["ms"]) == {1, 2, 4}
    assert all(s.params["spmv_unroll"] == 4 for s in solvers)


def test_cached_result_sets_both_parameters(tmp_path, monkeypatch):
    path = tmp_path / "tune.json"
    ns = [100, 200]
    autotune._store_cache(str(path), {autotune.signature(ns): {"poll_period": 40, "spmv_unroll": 1, "threads": 8,
                                                                "tables": {}}})
    solvers = [FakeSolver(), FakeSolver()]
    res = autotune.tune_batch(solvers, [0, 0], [0, 0], ns, cache_path=str(path))
    assert res["cached"] and res["threads"] == 8
    # an entry without batch_launch (older cache) restores the defaults
    assert all(s.params == {"poll_period": 40, "spmv_unroll": 1, "batch_launch": "streams", "batch_groups": 0,
                            "apply_items_per_warp": 1} for s in solvers)


def test_batch_launch_picks_the_fastest_and_leaves_it_set():
    solvers = [FakeSolver(), FakeSolver()]
    cost = {"fused": 0.004, "streams": 0.02}

    def run():
        time.sleep(cost[solvers[0].params["batch_launch"]])

    res = autotune.tune_batch_launch(solvers, run, repeats=2)
    assert res["best"] == "fused" and set(res["ms"]) == {"fused", "streams"}
    assert all(s.params["batch_launch"] == "fused" for s in solvers)


def test_tune_batch_searches_every_shape_and_caches(tmp_path, monkeypatch):
    """The whole batch search with stand-in solvers: each parameter is searched with the earlier
    choices in place, the fastest values are left set, and the result is cached by sizes."""
    from polysolve_b200 import solver as solver_mod

    solvers = [FakeSolver(), FakeSolver()]
    best = {"apply_items_per_warp": 4, "batch_groups": 2, "batch_launch": "fused", "poll_period": 20,
            "spmv_unroll": 1}
    calls = []

    def fake_batch(svs, bp, xp, ns, threads=0):
        p = svs[0].params
        calls.append(dict(p, threads=threads))
        miss = sum(1 for k, v in best.items() if k in p and p[k] != v)
        time.sleep(0.001 + 0.002 * miss + 0.001 * abs(threads - 8) / 8)

    monkeypatch.setattr(solver_mod, "solve_batch_device", fake_batch)
    path = tmp_path / "tune.json"
    res = autotune.tune_batch(solvers, [0, 0], [0, 0], [10, 20], cache_path=str(path), repeats=2,
                              thread_candidates=(1, 2, 8))
    assert not res["cached"]
    for k, v in best.items():
        assert res[k] == v
        assert all(s.params[k] == v for s in solvers)
    # thread counts above the number of systems are not tried
    assert res["threads"] == 2 and set(res["tables"]["threads_ms"]) == {1, 2}
    assert set(res["tables"]) == {"apply_items_per_warp_ms", "batch_groups_ms", "batch_launch_ms", "poll_period_ms",
                                  "spmv_unroll_ms", "threads_ms"}
    # group counts above the number of systems are not tried, and they are timed in the fused form
    assert set(res["tables"]["batch_groups_ms"]) == {1, 2}
    assert any(c.get("batch_launch") == "fused" and c.get("batch_groups") == 2 for c in calls)
    fresh = [FakeSolver(), FakeSolver()]
    again = autotune.tune_batch(fresh, [0, 0], [0, 0], [20, 10], cache_path=str(path))
    assert again["cached"] and all(s.params["batch_launch"] == "fused" and s.params["batch_groups"] == 2 for s in fresh)
