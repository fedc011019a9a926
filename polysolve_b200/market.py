"""Matrix Market files for A and b (``mas_market_*`` in the C ABI).

The reference's tests read their systems with Eigen's loadMarket / loadMarketVector
(tests/test_linear_solver.cpp:25-50, :211-213); these functions read the same files, so a system
exported from polyfem can be solved here in place of the synthetic ones:

    A = market.load_matrix("A.mat")      # scipy CSC (symmetric files expanded, duplicates summed)
    b = market.load_vector("b.mat")      # numpy float64 (array or single-column coordinate file)
    solver.factorize(A); solver.solve(b, x)
"""

from __future__ import annotations

import ctypes
import os

import numpy as np

from .solver import MAS_OK, MasError, library

_READY = False


def _lib():
    global _READY
    L = library()
    if not _READY:
        vp, i = ctypes.c_void_p, ctypes.c_int
        L.mas_market_load.argtypes = [ctypes.c_char_p, ctypes.POINTER(vp)]
        L.mas_market_dims.argtypes = [vp, ctypes.POINTER(i), ctypes.POINTER(i), ctypes.POINTER(ctypes.c_longlong),
                                      ctypes.POINTER(i)]
        L.mas_market_copy_csc.argtypes = [vp, vp, vp, vp]
        L.mas_market_copy_dense.argtypes = [vp, vp, ctypes.c_longlong]
        L.mas_market_free.argtypes = [vp]
        L.mas_market_free.restype = None
        L.mas_market_last_error.restype = ctypes.c_char_p
        L.mas_market_write_csc.argtypes = [ctypes.c_char_p, i, vp, vp, vp, i]
        L.mas_market_write_vector.argtypes = [ctypes.c_char_p, vp, ctypes.c_longlong]
        _READY = True
    return L


def _check(rc: int) -> None:
    if rc != MAS_OK:
        raise MasError(int(rc), _lib().mas_market_last_error().decode(errors="replace"))


def _load(path):
    L = _lib()
    h = ctypes.c_void_p()
    _check(L.mas_market_load(os.fsencode(path), ctypes.byref(h)))
    rows, cols, dense = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    nnz = ctypes.c_longlong()
    L.mas_market_dims(h, ctypes.byref(rows), ctypes.byref(cols), ctypes.byref(nnz), ctypes.byref(dense))
    return h, rows.value, cols.value, nnz.value, bool(dense.value)


def load_matrix(path):
    """A sparse matrix file as scipy CSC (sorted indices, float64, int32 indices)."""
    import scipy.sparse as sp

    L = _lib()
    h, rows, cols, nnz, dense = _load(path)
    try:
        if dense:
            out = np.empty(rows * cols)
            _check(L.mas_market_copy_dense(h, out.ctypes.data, out.size))
            return sp.csc_matrix(out.reshape(cols, rows).T)
        outer = np.empty(cols + 1, dtype=np.int32)
        inner = np.empty(max(nnz, 1), dtype=np.int32)
        vals = np.empty(max(nnz, 1))
        _check(L.mas_market_copy_csc(h, outer.ctypes.data, inner.ctypes.data, vals.ctypes.data))
        return sp.csc_matrix((vals[:nnz], inner[:nnz], outer), shape=(rows, cols))
    finally:
        L.mas_market_free(h)


def load_vector(path) -> np.ndarray:
    """A vector file (n x 1 array, or a single-column coordinate file) as float64."""
    L = _lib()
    h, rows, cols, nnz, dense = _load(path)
    try:
        if cols != 1:
            raise MasError(1, f"[MAS] {path}: a vector file has one column, not {cols}")
        if dense:
            out = np.empty(rows)
            _check(L.mas_market_copy_dense(h, out.ctypes.data, rows))
            return out
        outer = np.empty(2, dtype=np.int32)
        inner = np.empty(max(nnz, 1), dtype=np.int32)
        vals = np.empty(max(nnz, 1))
        _check(L.mas_market_copy_csc(h, outer.ctypes.data, inner.ctypes.data, vals.ctypes.data))
        out = np.zeros(rows)
        out[inner[:nnz]] = vals[:nnz]
        return out
    finally:
        L.mas_market_free(h)


def save_matrix(path, A, symmetric: bool = False) -> None:
    """A square sparse matrix as coordinate real general (or its lower triangle, symmetric)."""
    import scipy.sparse as sp

    A = sp.csc_matrix(A)
    A.sort_indices()
    n = A.shape[0]
    if A.shape[1] != n:
        raise ValueError("save_matrix writes square matrices")
    outer = np.ascontiguousarray(A.indptr, dtype=np.int32)
    inner = np.ascontiguousarray(A.indices, dtype=np.int32)
    vals = np.ascontiguousarray(A.data, dtype=np.float64)
    _check(_lib().mas_market_write_csc(os.fsencode(path), n, outer.ctypes.data, inner.ctypes.data,
                                       vals.ctypes.data, int(bool(symmetric))))


def save_vector(path, x) -> None:
    x = np.ascontiguousarray(x, dtype=np.float64).reshape(-1)
    _check(_lib().mas_market_write_vector(os.fsencode(path), x.ctypes.data, x.size))


__all__ = ["load_matrix", "load_vector", "save_matrix", "save_vector"]
