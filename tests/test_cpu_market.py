"""Matrix Market I/O (the format of the reference's test fixtures, read there with Eigen's
loadMarket / loadMarketVector) against scipy.io's independent reader and writer."""

import numpy as np
import pytest
import scipy.io
import scipy.sparse as sp

from polysolve_b200 import market, synthetic
from polysolve_b200.solver import MasError


@pytest.fixture(scope="module")
def system():
    return synthetic.elasticity(4, young_sigma=1.0, jitter=0.2, seed=3)


def test_read_scipy_written_general_and_symmetric(tmp_path, system):
    A = system.scipy()
    scipy.io.mmwrite(tmp_path / "g.mtx", A, symmetry="general")
    scipy.io.mmwrite(tmp_path / "s.mtx", A, symmetry="symmetric")
    for name in ("g.mtx", "s.mtx"):
        B = market.load_matrix(tmp_path / name)
        assert B.has_sorted_indices
        assert (abs(B - A) > 0).nnz == 0
        assert np.array_equal(B.indptr, A.indptr) and np.array_equal(B.indices, A.indices)


def test_round_trip_is_exact(tmp_path, system):
    A = system.scipy()
    market.save_matrix(tmp_path / "a.mtx", A)
    market.save_matrix(tmp_path / "a_sym.mtx", A, symmetric=True)
    for name in ("a.mtx", "a_sym.mtx"):
        B = market.load_matrix(tmp_path / name)
        assert np.array_equal(B.indptr, A.indptr) and np.array_equal(B.indices, A.indices)
        assert np.array_equal(B.data, A.data)
        # scipy reads what we write
        C = sp.csc_matrix(scipy.io.mmread(tmp_path / name))
        assert (abs(C - A) > 0).nnz == 0
    b = np.random.default_rng(0).standard_normal(A.shape[0])
    market.save_vector(tmp_path / "b.mtx", b)
    assert np.array_equal(market.load_vector(tmp_path / "b.mtx"), b)
    assert np.array_equal(np.asarray(scipy.io.mmread(tmp_path / "b.mtx")).reshape(-1), b)


def test_duplicates_pattern_integer_comments(tmp_path):
    (tmp_path / "d.mtx").write_text(
        "%%MatrixMarket matrix coordinate real general\n% a comment\n%\n3 3 5\n"
        "1 1 1.5\n3 1 -2\n1 1 0.5\n2 2 4e0\n3 3 +7\n")
    A = market.load_matrix(tmp_path / "d.mtx").toarray()
    assert np.array_equal(A, [[2.0, 0, 0], [0, 4, 0], [-2, 0, 7]])
    (tmp_path / "p.mtx").write_text("%%MatrixMarket matrix coordinate pattern symmetric\n3 3 2\n2 1\n3 3\n")
    P = market.load_matrix(tmp_path / "p.mtx").toarray()
    assert np.array_equal(P, [[0, 1, 0], [1, 0, 0], [0, 0, 1]])
    (tmp_path / "i.mtx").write_text("%%MatrixMarket matrix array integer general\n2 2\n1\n2\n3\n4\n")
    assert np.array_equal(market.load_matrix(tmp_path / "i.mtx").toarray(), [[1, 3], [2, 4]])
    (tmp_path / "v.mtx").write_text("%%MatrixMarket matrix coordinate real general\n4 1 2\n2 1 5\n4 1 -1\n")
    assert np.array_equal(market.load_vector(tmp_path / "v.mtx"), [0, 5, 0, -1])


@pytest.mark.parametrize("text", [
    "%%MatrixMarket matrix coordinate complex general\n1 1 1\n1 1 1 0\n",
    "%%MatrixMarket vector coordinate real general\n1 1 1\n1 1 1\n",
    "not a header\n1 1 1\n1 1 1\n",
    "%%MatrixMarket matrix coordinate real general\n2 2 1\n3 1 1\n",
    "%%MatrixMarket matrix coordinate real general\n2 2 2\n1 1 1\n",
    "%%MatrixMarket matrix coordinate real symmetric\n2 3 0\n",
])
def test_malformed_files_are_rejected(tmp_path, text):
    (tmp_path / "bad.mtx").write_text(text)
    with pytest.raises(MasError) as e:
        market.load_matrix(tmp_path / "bad.mtx")
    assert "[MAS]" in str(e.value)


def test_missing_file(tmp_path):
    with pytest.raises(MasError):
        market.load_matrix(tmp_path / "nope.mtx")
    with pytest.raises(MasError):
        market.load_vector(tmp_path / "nope.mtx")
