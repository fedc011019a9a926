"""The C++ drop-in header (include/polysolve/linear/MASSolver.hpp) driven by a C++ program that
mirrors polysolve's TEST_CASE("all") and TEST_CASE("pre_factor")."""

from __future__ import annotations

import subprocess

import numpy as np
import pytest

from polysolve_b200 import _build, synthetic

pytestmark = pytest.mark.gpu


def write_market(path, A) -> None:
    A = A.tocoo()
    with open(path, "w") as f:
        f.write("%%MatrixMarket matrix coordinate real general\n")
        f.write(f"{A.shape[0]} {A.shape[1]} {A.nnz}\n")
        for i, j, v in zip(A.row, A.col, A.data):
            f.write(f"{i + 1} {j + 1} {v:.17g}\n")


def test_cpp_api_all_and_pre_factor(tmp_path):
    exe = _build.build_cpp_test()
    # scaled so the reference's absolute alpha guard (|p.Ap| < 1e-20) does not stall at abs 1e-8
    A = (synthetic.elasticity(5, young_sigma=0.5, seed=13).scipy() * 1e-3).tocsc()
    path = tmp_path / "A.mtx"
    write_market(path, A)
    res = subprocess.run([str(exe), str(path)], stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True,
                         timeout=600)
    print(res.stdout)
    assert res.returncode == 0, res.stdout
    assert res.stdout.strip().endswith("OK")
