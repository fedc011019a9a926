"""Host-side logic without a GPU: the C ABI library loads and exports every declared symbol, the
ordering matches its restatement, the synthetic workloads have the stated shapes, and creating a
solver without a device fails the way the reference does."""

from __future__ import annotations

import ctypes
import re
from pathlib import Path

import numpy as np
import pytest

from oracle import oracle as O
from polysolve_b200 import MasError, Solver, synthetic
from polysolve_b200.solver import EXPORTED_SYMBOLS, library, order_blocks

ROOT = Path(__file__).resolve().parents[1]


def declared_symbols() -> list[str]:
    text = (ROOT / "include" / "polysolve_mas.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(mas_[a-z_0-9]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = library()
    declared = declared_symbols()
    assert declared, "no declarations found"
    for name in declared:
        assert hasattr(lib, name), name
    assert sorted(EXPORTED_SYMBOLS) == declared


def test_name_without_device():
    assert library().mas_name().decode() == "MAS"


def test_create_without_gpu_fails_like_reference():
    try:
        import torch

        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    with pytest.raises(MasError) as e:
        Solver.create("MAS", "")
    assert e.value.code == 8
    assert "No Nvidia GPU!!" in str(e.value)


def test_create_json_rejects_bad_params_before_device():
    with pytest.raises(MasError) as e:
        Solver.create({"solver": "MAS", "MAS": {"block_dim": 5}})
    assert "block_dim" in str(e.value)
    with pytest.raises(MasError):
        Solver.create({"solver": "MAS", "MAS": {"max_iter": "many"}})
    with pytest.raises(MasError):
        Solver.create({"solver": "MAS", "MAS": {"unknown_key": 1}})
    with pytest.raises(MasError):
        Solver.create({"solver": "AMGCL"})


@pytest.mark.parametrize("key,bad", [("batch_launch", "persistent"), ("batch_groups", -1), ("batch_groups", 65),
                                     ("apply_items_per_warp", 0), ("apply_items_per_warp", 65),
                                     ("spmv_unroll", 3)])
def test_launch_shape_parameters_are_validated_before_device(key, bad):
    with pytest.raises(MasError) as e:
        Solver.create({"solver": "MAS", "MAS": {key: bad}})
    assert key in str(e.value)


@pytest.mark.parametrize("N,kw", [(5, {}), (12, dict(young_sigma=1.0, jitter=0.2)),
                                  (16, dict(jitter=0.2, contact_pairs=200))])
def test_morton_ordering_matches_restatement(N, kw):
    s = synthetic.elasticity(N, **kw)
    iso = O.isolated_blocks(s.outer, s.inner, s.n, 3)
    ref = O.morton_padded(s.positions, iso)
    got, banks = order_blocks(s, 3, "morton", s.positions)
    np.testing.assert_array_equal(got, ref)
    assert banks == int(ref.max()) // 32 + 1


@pytest.mark.parametrize("mode", ["graph", "natural"])
def test_orderings_are_valid(mode):
    s = synthetic.elasticity(9, young_sigma=1.0, jitter=0.2)
    V = s.n // 3
    padded, banks = order_blocks(s, 3, mode)
    assert padded.size == V
    assert len(np.unique(padded)) == V
    assert padded.min() >= 0 and padded.max() < banks * 32
    perm, offsets = O.partition_from_padded(padded)
    assert np.all(np.diff(offsets) <= 32) and np.all(np.diff(offsets) >= 1)


class _Csc:
    def __init__(self, n, outer, inner, vals):
        self.n, self.outer, self.inner, self.vals = n, outer, inner, vals


def test_invalid_patterns_are_rejected_on_the_host():
    """The pattern pass (shared with factorize) rejects row indices outside [0, n) and
    decreasing column pointers before anything reads through them; row order inside a column
    does not change the ordering."""
    s = synthetic.elasticity(6, young_sigma=1.0)
    ref, ref_banks = order_blocks(s, 3, "graph")
    inner_rev = s.inner.copy()
    for j in range(s.n):
        inner_rev[s.outer[j]:s.outer[j + 1]] = s.inner[s.outer[j]:s.outer[j + 1]][::-1]
    got, banks = order_blocks(_Csc(s.n, s.outer, inner_rev, s.vals), 3, "graph")
    np.testing.assert_array_equal(got, ref)
    assert banks == ref_banks
    for bad_row in (s.n, -1, 2 ** 31 - 1):
        inner = s.inner.copy()
        inner[len(inner) // 2] = bad_row
        with pytest.raises(MasError):
            order_blocks(_Csc(s.n, s.outer, inner, s.vals), 3, "graph")
    outer = s.outer.copy()
    j = s.n // 2
    outer[j] = outer[j + 1] + 1  # column j - 1 runs past column j's start
    with pytest.raises(MasError):
        order_blocks(_Csc(s.n, outer, s.inner, s.vals), 3, "natural")


def test_graph_ordering_is_local():
    """Graph bisection banks are mostly connected (few level-0 components per bank)."""
    s = synthetic.elasticity(12, young_sigma=1.0)
    padded, banks = order_blocks(s, 3, "graph")
    perm, offsets = O.partition_from_padded(padded)
    orc = O.MasOracle(s.outer, s.inner, s.vals, s.n, 3, perm, offsets)
    iso = O.isolated_blocks(s.outer, s.inner, s.n, 3)
    coupled_banks = orc.s.P - -(-int(iso.sum()) // 32)
    assert orc.s.cco_nums[0] - int(iso.sum()) <= 1.5 * coupled_banks


def test_synthetic_shapes():
    s = synthetic.workload_cpu20()
    assert s.n == 27783 and s.nverts == 9261
    A = s.scipy()
    assert abs(A - A.T).max() == 0.0
    s4 = synthetic.elasticity(4, young_sigma=1.0, jitter=0.2, contact_pairs=20)
    A4 = s4.scipy().toarray()
    assert np.allclose(A4, A4.T, rtol=0, atol=0)
    assert np.linalg.eigvalsh(A4).min() > 0
    assert len(synthetic.batch_edges()) == 64
    assert all(8 <= e <= 48 for e in synthetic.batch_edges())


def test_synthetic_thread_independent(monkeypatch):
    s1 = synthetic.elasticity(6, young_sigma=1.0, jitter=0.2, seed=9)
    s2 = synthetic.elasticity(6, young_sigma=1.0, jitter=0.2, seed=9)
    np.testing.assert_array_equal(s1.vals, s2.vals)
    np.testing.assert_array_equal(s1.positions, s2.positions)
