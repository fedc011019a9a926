"""Python mirror of polysolve's linear ``Solver`` interface for the "MAS" solver.

Same names, argument meaning and error behaviour as polysolve::linear::Solver / MASSolver
(src/polysolve/linear/Solver.hpp:31-132, src/polysolve/linear/MASSolver.hpp:35-72):

    solver = Solver.create("MAS", "")             # impl defaults (MASSolver.cu:137-143)
    solver = Solver.create(params_dict, logger)   # spec defaults (linear-solver-spec.json:456-509)
    solver.set_parameters({"MAS": {...}})
    solver.analyze_pattern(A, A.shape[0])
    solver.factorize(A)                           # A: scipy CSC (or anything with .tocsc())
    solver.solve(b, x)                            # x is written in place
    solver.get_info(info)                         # solver_iter, solver_error, solver_status, ...
    solver.name() == "MAS"

Everything runs through the C ABI of ``libpolysolve_mas.so`` (include/polysolve_mas.h). There is
no CPU fallback: without the library or a GPU the calls raise.
"""

from __future__ import annotations

import ctypes
import json
from typing import Any

import numpy as np

from . import _build

MAS_OK = 0
MAS_ERR_INVALID = 1
MAS_ERR_OOM = 2
MAS_ERR_NOT_FACTORIZED = 3
MAS_ERR_CUDA = 4
MAS_ERR_NONFINITE = 5
MAS_ERR_INVERSE = 6
MAS_ERR_TIMEOUT = 7
MAS_ERR_NO_DEVICE = 8

EXPORTED_SYMBOLS = [
    "mas_create", "mas_create_json", "mas_destroy", "mas_set_parameters", "mas_get_info", "mas_name",
    "mas_analyze_pattern", "mas_set_positions", "mas_factorize_csc", "mas_factorize_values", "mas_solve", "mas_solve_multi",
    "mas_solve_device", "mas_solve_batch", "mas_set_stream", "mas_spmv_dot_noalloc", "mas_last_error", "mas_get_sizes", "mas_get_ordering", "mas_order_blocks",
    "mas_get_coarse_map", "mas_get_inverses", "mas_debug_spmv", "mas_debug_apply", "mas_debug_apply_multi",
    "mas_debug_spmv_multi", "mas_set_warm_start_model", "mas_reset_warm_start", "mas_debug_warm_start",
    "mas_market_load", "mas_market_dims", "mas_market_copy_csc", "mas_market_copy_dense", "mas_market_free",
    "mas_market_last_error", "mas_market_write_csc", "mas_market_write_vector", "mas_debug_fail_allocation",
    "mas_ws_trainer_create", "mas_ws_trainer_destroy", "mas_ws_trainer_add_sample", "mas_ws_trainer_sample_count",
    "mas_ws_trainer_train", "mas_ws_trainer_evaluate", "mas_ws_trainer_gradient", "mas_ws_trainer_get_params",
    "mas_ws_trainer_last_error",
]


class CudaOutOfMemoryError(RuntimeError):
    """Device allocation failure (reference: mas::CudaOutOfMemoryError, CudaUtils.cuh:33-37)."""


class MasError(RuntimeError):
    """Any other non-zero status of the C ABI (reference: std::runtime_error)."""

    def __init__(self, code: int, message: str):
        super().__init__(message)
        self.code = code


_LIB = None


def library() -> ctypes.CDLL:
    """Load libpolysolve_mas.so (built in-tree). Raises if it is missing: no fallback."""
    global _LIB
    if _LIB is None:
        path = _build.MAS_LIB
        if not path.exists():
            raise RuntimeError(f"[MAS] native library not built: {path} (run __graft_entry__.build())")
        L = ctypes.CDLL(str(path))
        vp, ip, i = ctypes.c_void_p, ctypes.POINTER(ctypes.c_int), ctypes.c_int
        hp = ctypes.POINTER(ctypes.c_void_p)
        L.mas_create.argtypes = [ctypes.c_char_p, ctypes.c_char_p, hp]
        L.mas_create_json.argtypes = [ctypes.c_char_p, i, hp]
        L.mas_destroy.argtypes = [vp]
        L.mas_destroy.restype = None
        L.mas_set_parameters.argtypes = [vp, ctypes.c_char_p]
        L.mas_get_info.argtypes = [vp, ctypes.c_char_p, ctypes.c_size_t, ctypes.POINTER(ctypes.c_size_t)]
        L.mas_name.restype = ctypes.c_char_p
        L.mas_analyze_pattern.argtypes = [vp, i, vp, vp, i, i]
        L.mas_set_positions.argtypes = [vp, vp, i]
        L.mas_factorize_csc.argtypes = [vp, i, vp, vp, vp, i]
        L.mas_factorize_values.argtypes = [vp, vp, i]
        L.mas_solve.argtypes = [vp, vp, vp, i]
        L.mas_solve_multi.argtypes = [vp, vp, vp, i, i]
        L.mas_solve_device.argtypes = [vp, ctypes.c_void_p, ctypes.c_void_p, i]
        L.mas_solve_batch.argtypes = [hp, i, hp, hp, ip, i, i, ip]
        L.mas_set_stream.argtypes = [vp, vp]
        L.mas_spmv_dot_noalloc.argtypes = [vp, vp, vp, vp, i, vp]
        L.mas_last_error.argtypes = [vp]
        L.mas_last_error.restype = ctypes.c_char_p
        L.mas_get_sizes.argtypes = [vp, ip]
        L.mas_get_ordering.argtypes = [vp, ip, i]
        L.mas_get_coarse_map.argtypes = [vp, ip, i]
        L.mas_get_inverses.argtypes = [vp, vp, ctypes.c_size_t]
        L.mas_debug_spmv.argtypes = [vp, vp, vp, i]
        L.mas_debug_apply.argtypes = [vp, vp, vp, i]
        L.mas_debug_apply_multi.argtypes = [vp, vp, vp, i]
        L.mas_debug_spmv_multi.argtypes = [vp, vp, vp, i]
        L.mas_set_warm_start_model.argtypes = [vp, vp, ctypes.c_longlong]
        L.mas_reset_warm_start.argtypes = [vp]
        L.mas_debug_warm_start.argtypes = [vp, vp, vp, i, vp, vp, vp, vp]
        L.mas_order_blocks.argtypes = [i, vp, vp, i, vp, ctypes.c_char_p, ip, ip]
        L.mas_debug_fail_allocation.argtypes = [ctypes.c_longlong]
        L.mas_ws_trainer_create.argtypes = [vp, ctypes.c_longlong, hp]
        L.mas_ws_trainer_destroy.argtypes = [vp]
        L.mas_ws_trainer_destroy.restype = None
        L.mas_ws_trainer_add_sample.argtypes = [vp, vp, vp, vp, i, vp, i]
        L.mas_ws_trainer_sample_count.argtypes = [vp]
        L.mas_ws_trainer_train.argtypes = [vp, vp, vp, i, vp]
        L.mas_ws_trainer_evaluate.argtypes = [vp, vp, i, vp]
        L.mas_ws_trainer_gradient.argtypes = [vp, i, vp, ctypes.c_longlong, vp]
        L.mas_ws_trainer_get_params.argtypes = [vp, vp, ctypes.c_longlong]
        L.mas_ws_trainer_last_error.argtypes = [vp]
        L.mas_ws_trainer_last_error.restype = ctypes.c_char_p
        _LIB = L
    return _LIB


def solve_batch(solvers: list, bs: list, xs: list | None = None, *, threads: int = 0) -> list:
    """New: solve independent factorized systems concurrently (``mas_solve_batch``): solver i
    solves A_i x_i = b_i, on its own CUDA stream (``"batch_launch": "streams"``, the default) or
    in fused launches, one per PCG phase for all systems of a size group (``"fused"``, results
    bit-identical to single solves), with a pool of host threads for the per-system steps.
    bs / xs hold float64 numpy arrays (written in place; allocated when xs is None). Returns xs.
    Raises the first failing solver's error; every solver's status stays readable through its
    ``get_info``."""
    count = len(solvers)
    if len(bs) != count or (xs is not None and len(xs) != count):
        raise ValueError("solvers, bs and xs must have the same length")
    bs = [np.ascontiguousarray(b, dtype=np.float64) for b in bs]
    if xs is None:
        xs = [np.zeros_like(b) for b in bs]
    for x, b in zip(xs, bs):
        if not (isinstance(x, np.ndarray) and x.dtype == np.float64 and x.flags.c_contiguous) or x.size != b.size:
            raise TypeError("each x must be a contiguous float64 numpy array of its b's size")
    VP = ctypes.c_void_p
    handles = (VP * max(count, 1))(*[s._h for s in solvers])
    bp = (VP * max(count, 1))(*[b.ctypes.data for b in bs])
    xp = (VP * max(count, 1))(*[x.ctypes.data for x in xs])
    ns = np.array([b.size for b in bs] or [0], dtype=np.int32)
    st = np.zeros(max(count, 1), dtype=np.int32)
    rc = library().mas_solve_batch(handles, count, bp, xp, ns.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), 0,
                                   int(threads), st.ctypes.data_as(ctypes.POINTER(ctypes.c_int)))
    if rc != MAS_OK:
        bad = next((k for k in range(count) if st[k] != MAS_OK), None)
        _check(int(rc), solvers[bad]._h if bad is not None else (solvers[0]._h if count else None))
    return xs


def solve_batch_device(solvers: list, b_ptrs: list, x_ptrs: list, ns: list, *, threads: int = 0) -> None:
    """New: like ``solve_batch`` with device pointers (e.g. torch ``data_ptr()``) in each system's
    caller order."""
    count = len(solvers)
    if not (len(b_ptrs) == len(x_ptrs) == len(ns) == count):
        raise ValueError("solvers, b_ptrs, x_ptrs and ns must have the same length")
    VP = ctypes.c_void_p
    handles = (VP * max(count, 1))(*[s._h for s in solvers])
    bp = (VP * max(count, 1))(*[int(p) for p in b_ptrs])
    xp = (VP * max(count, 1))(*[int(p) for p in x_ptrs])
    nn = np.array(list(ns) or [0], dtype=np.int32)
    st = np.zeros(max(count, 1), dtype=np.int32)
    rc = library().mas_solve_batch(handles, count, bp, xp, nn.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), 1,
                                   int(threads), st.ctypes.data_as(ctypes.POINTER(ctypes.c_int)))
    if rc != MAS_OK:
        bad = next((k for k in range(count) if st[k] != MAS_OK), None)
        _check(int(rc), solvers[bad]._h if bad is not None else (solvers[0]._h if count else None))


def debug_fail_allocation(after: int) -> None:
    """Test hook (process-wide): after ``after`` more successful device allocations the next one
    fails as if the device were out of memory, once (the solver raises CudaOutOfMemoryError with
    the requested and free MB, as mas_utils/CudaUtils.cuh:68-79). Negative: off."""
    library().mas_debug_fail_allocation(int(after))


def order_blocks(A, block_dim: int, mode: str, positions: np.ndarray | None = None) -> tuple[np.ndarray, int]:
    """Host-only: the padded subdomain ordering factorize computes (padded id per block row, banks)."""
    n, outer, inner, _ = _csc_arrays(A)
    V = -(-n // block_dim)
    padded = np.empty(V, dtype=np.int32)
    banks = ctypes.c_int()
    xyz = None
    if positions is not None:
        xyz = np.ascontiguousarray(positions, dtype=np.float64).reshape(-1, 3)
    rc = library().mas_order_blocks(n, outer.ctypes.data, inner.ctypes.data, block_dim,
                                    None if xyz is None else xyz.ctypes.data, mode.encode(),
                                    padded.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), ctypes.byref(banks))
    if rc != MAS_OK:
        raise MasError(rc, f"[MAS] order_blocks failed ({mode})")
    return padded, banks.value


def _check(rc: int, h=None) -> None:
    if rc == MAS_OK:
        return
    msg = library().mas_last_error(h).decode()
    if rc == MAS_ERR_OOM:
        raise CudaOutOfMemoryError(msg)
    raise MasError(rc, msg or f"[MAS] error {rc}")


def _csc_arrays(A) -> tuple[int, np.ndarray, np.ndarray, np.ndarray]:
    """(n, outer, inner, vals) of a square CSC matrix, int32/float64 contiguous."""
    if hasattr(A, "outer") and hasattr(A, "inner") and hasattr(A, "vals"):
        n = int(A.n)
        outer, inner, vals = A.outer, A.inner, A.vals
    else:
        if not hasattr(A, "tocsc"):
            raise TypeError("A must be a scipy sparse matrix or provide outer/inner/vals")
        Ac = A.tocsc()
        if Ac.shape[0] != Ac.shape[1]:
            raise ValueError("[MAS] A must be square")
        # Row order inside a column is free, and the library checks the row range and the
        # column pointers itself in its pattern pass (scipy's sortedness scan of a new matrix
        # costs more than a values-only refactorization).
        n = int(Ac.shape[0])
        outer, inner, vals = Ac.indptr, Ac.indices, Ac.data
    if np.asarray(outer)[-1] >= 2 ** 31:
        raise ValueError("[MAS] A is too large. Non-zero number exceeding int32 max.")
    return (n, np.ascontiguousarray(outer, dtype=np.int32), np.ascontiguousarray(inner, dtype=np.int32),
            np.ascontiguousarray(vals, dtype=np.float64))


class Solver:
    """polysolve::linear::Solver for the "MAS" solver (the only one this library provides)."""

    def __init__(self, handle: int):
        self._h = ctypes.c_void_p(handle)
        self._n = 0

    # -- constructors (Solver.cpp:145-167, 310-499) ------------------------------------------
    @staticmethod
    def create(params: Any, precond_or_logger: Any = "", strict_validation: bool = True) -> "Solver":
        L = library()
        h = ctypes.c_void_p()
        if isinstance(params, str):
            rc = L.mas_create(params.encode(), str(precond_or_logger or "").encode(), ctypes.byref(h))
        else:
            rc = L.mas_create_json(json.dumps(params).encode(), 1 if strict_validation else 0, ctypes.byref(h))
        if rc != MAS_OK:
            msg = L.mas_last_error(None).decode()
            if rc == MAS_ERR_OOM:
                raise CudaOutOfMemoryError(msg)
            raise MasError(rc, msg)
        return Solver(h.value)

    @staticmethod
    def available_solvers() -> list[str]:
        return ["MAS"]

    @staticmethod
    def default_solver() -> str:
        return "MAS"

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                library().mas_destroy(h)
            except Exception:
                pass
            self._h = ctypes.c_void_p()

    # -- interface --------------------------------------------------------------------------
    def set_parameters(self, params: dict) -> None:
        _check(library().mas_set_parameters(self._h, json.dumps(params).encode()), self._h)

    def get_info(self, params: dict | None = None) -> dict:
        L = library()
        need = ctypes.c_size_t()
        _check(L.mas_get_info(self._h, None, 0, ctypes.byref(need)), self._h)
        buf = ctypes.create_string_buffer(need.value)
        _check(L.mas_get_info(self._h, buf, need.value, ctypes.byref(need)), self._h)
        info = json.loads(buf.value.decode())
        if params is not None:
            params.update(info)
        return info

    def analyze_pattern(self, A, precond_num: int = 0) -> None:
        n, outer, inner, vals = _csc_arrays(A)
        _check(library().mas_analyze_pattern(self._h, n, outer.ctypes.data, inner.ctypes.data, int(inner.size),
                                             int(precond_num)), self._h)

    def set_positions(self, xyz: np.ndarray) -> None:
        """New: vertex positions (one xyz per block row) for the Morton subdomain ordering."""
        xyz = np.ascontiguousarray(xyz, dtype=np.float64).reshape(-1, 3)
        self._pos = xyz
        _check(library().mas_set_positions(self._h, xyz.ctypes.data, int(xyz.shape[0])), self._h)

    def factorize(self, A) -> None:
        n, outer, inner, vals = _csc_arrays(A)
        _check(library().mas_factorize_csc(self._h, n, outer.ctypes.data, inner.ctypes.data, vals.ctypes.data,
                                           int(inner.size)), self._h)
        self._n = n

    def factorize_values(self, A) -> None:
        """New: values-only refactorization declared by the caller. A is a matrix with the pattern
        of the last factorized one (only its values are used) or the values array itself, in that
        matrix's CSC order; the pattern check is skipped."""
        if hasattr(A, "tocsc"):
            vals = A.tocsc().data
        elif hasattr(A, "vals"):
            vals = A.vals
        else:
            vals = A
        vals = np.ascontiguousarray(vals, dtype=np.float64)
        _check(library().mas_factorize_values(self._h, vals.ctypes.data, int(vals.size)), self._h)

    def solve(self, b: np.ndarray, x: np.ndarray) -> None:
        """Solve A x = b; x (float64, contiguous) is written in place."""
        b = np.ascontiguousarray(b, dtype=np.float64)
        if not (isinstance(x, np.ndarray) and x.dtype == np.float64 and x.flags.c_contiguous):
            raise TypeError("x must be a contiguous float64 numpy array (written in place)")
        if b.size != x.size:
            raise MasError(MAS_ERR_NOT_FACTORIZED, "[MAS] Size mismatch. Did you forget to call factorize?")
        _check(library().mas_solve(self._h, b.ctypes.data, x.ctypes.data, int(b.size)), self._h)

    def solve_multi(self, B: np.ndarray) -> np.ndarray:
        """New: nrhs right-hand sides as rows of B (nrhs, n); returns X (nrhs, n)."""
        B = np.ascontiguousarray(B, dtype=np.float64)
        X = np.zeros_like(B)
        nrhs, n = B.shape
        _check(library().mas_solve_multi(self._h, B.ctypes.data, X.ctypes.data, n, nrhs), self._h)
        return X

    def solve_device(self, d_b: int, d_x: int, n: int) -> None:
        """New: device pointers (e.g. torch.Tensor.data_ptr()) in the caller's order."""
        _check(library().mas_solve_device(self._h, ctypes.c_void_p(d_b), ctypes.c_void_p(d_x), int(n)), self._h)

    def set_stream(self, stream_handle: int | None) -> None:
        """New: run on the caller's CUDA stream (e.g. torch.cuda.current_stream().cuda_stream)."""
        _check(library().mas_set_stream(self._h, ctypes.c_void_p(stream_handle or 0)), self._h)

    def spmv_dot_noalloc(self, d_x: int, d_y: int, d_dot: int, length: int, stream: int | None = None) -> None:
        """New: y = A x and *d_dot = x . y on device pointers in padded block order, with no
        device allocation (static scratch; for callers that cannot allocate at call time)."""
        _check(library().mas_spmv_dot_noalloc(self._h, ctypes.c_void_p(d_x), ctypes.c_void_p(d_y),
                                               ctypes.c_void_p(d_dot), int(length), ctypes.c_void_p(stream or 0)),
               self._h)

    def name(self) -> str:
        return library().mas_name().decode()

    # -- inspection (new) -------------------------------------------------------------------
    def sizes(self) -> dict:
        s = (ctypes.c_int * 12)()
        _check(library().mas_get_sizes(self._h, s), self._h)
        keys = ["n", "block_dim", "V", "banks", "nodes", "nnzb", "level_num", "total_mats"]
        d = {k: int(s[i]) for i, k in enumerate(keys)}
        d["cco_nums"] = [int(s[8 + i]) for i in range(4)]
        return d

    def ordering(self) -> np.ndarray:
        V = self.sizes()["V"]
        out = np.empty(V, dtype=np.int32)
        _check(library().mas_get_ordering(self._h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), V), self._h)
        return out

    def coarse_map(self) -> np.ndarray:
        nodes = self.sizes()["nodes"]
        out = np.empty(nodes * 4, dtype=np.int32)
        _check(library().mas_get_coarse_map(self._h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), nodes),
               self._h)
        return out.reshape(nodes, 4)

    def inverses(self) -> np.ndarray:
        s = self.sizes()
        N = 32 * s["block_dim"]
        S = N * (N + 1) // 2
        out = np.empty(s["total_mats"] * S, dtype=np.float64)
        _check(library().mas_get_inverses(self._h, out.ctypes.data, out.size), self._h)
        return out.reshape(s["total_mats"], S)

    def debug_spmv(self, x_padded: np.ndarray) -> np.ndarray:
        x = np.ascontiguousarray(x_padded, dtype=np.float64)
        y = np.empty_like(x)
        _check(library().mas_debug_spmv(self._h, x.ctypes.data, y.ctypes.data, int(x.size)), self._h)
        return y

    def debug_apply(self, r_padded: np.ndarray) -> np.ndarray:
        r = np.ascontiguousarray(r_padded, dtype=np.float64)
        z = np.empty_like(r)
        _check(library().mas_debug_apply(self._h, r.ctypes.data, z.ctypes.data, int(r.size)), self._h)
        return z

    def debug_apply_multi(self, R_padded: np.ndarray) -> np.ndarray:
        """R_padded: (padded length, 4) columns; returns M^-1 applied to each (several-RHS kernels)."""
        r = np.ascontiguousarray(R_padded, dtype=np.float64)
        z = np.empty_like(r)
        _check(library().mas_debug_apply_multi(self._h, r.ctypes.data, z.ctypes.data, int(r.size)), self._h)
        return z

    def set_warm_start_model(self, params=None) -> None:
        """New: the network of ``initial_guess: "learned"``: a float32 parameter vector, a path to
        a ``.psws`` file, or None for the shipped weights (``polysolve_b200.warmstart``)."""
        from . import warmstart

        if params is None:
            params = warmstart.default_weights()
        elif not isinstance(params, np.ndarray):
            params = warmstart.load(params)
        prm = np.ascontiguousarray(params, dtype=np.float32)
        _check(library().mas_set_warm_start_model(self._h, prm.ctypes.data, int(prm.size)), self._h)

    def reset_warm_start(self) -> None:
        """New: forget the kept solutions (the next learned-mode solve starts from zero)."""
        _check(library().mas_reset_warm_start(self._h), self._h)

    def debug_warm_start(self, b: np.ndarray, *history: np.ndarray) -> dict:
        """Test hook: the learned starting guess for b given 2 to 4 kept solutions (x_{k-1} first,
        caller order), without a solve: c, x0, raw features (nverts, 16) and the reduction record
        (Galerkin matrix / right-hand side of the basis {x1, x1 - x2, x2 - x3, x3 - x4, c}; the
        coefficients of x_g, the first pass without c, in ``coef_history``)."""
        from . import warmstart

        b = np.ascontiguousarray(b, dtype=np.float64)
        hist = np.ascontiguousarray(np.stack([np.asarray(h, dtype=np.float64) for h in history]))
        n = b.size
        c = np.empty(n)
        x0 = np.empty(n)
        feat = np.empty(((n + 2) // 3, warmstart.FEATURES), dtype=np.float32)
        nb = warmstart.BASIS
        ng = nb * (nb + 1) // 2 + nb
        state = np.empty(5 + ng + nb + 4 + nb)
        _check(library().mas_debug_warm_start(self._h, b.ctypes.data, hist.ctypes.data, int(hist.shape[0]),
                                              c.ctypes.data, x0.ctypes.data, feat.ctypes.data, state.ctypes.data),
               self._h)
        e = 5 + ng
        return {"c": c, "x0": x0, "features": feat, "sums": state[0:5], "gram": state[5:e], "coef": state[e:e + nb],
                "energy": state[e + nb], "energy_previous": state[e + nb + 1], "fallback": bool(state[e + nb + 2]),
                "rank": int(state[e + nb + 3]), "coef_history": state[e + nb + 4:e + 2 * nb + 4]}

    def debug_spmv_multi(self, X_padded: np.ndarray) -> np.ndarray:
        x = np.ascontiguousarray(X_padded, dtype=np.float64)
        y = np.empty_like(x)
        _check(library().mas_debug_spmv_multi(self._h, x.ctypes.data, y.ctypes.data, int(x.size)), self._h)
        return y


MASSolver = Solver


class WarmStartTrainer:
    """New: GPU training of the learned warm start's network (``mas_ws_trainer_*``): the library's own
    forward / reverse-pass kernels and Adam, samples resident in device memory."""

    def __init__(self, params: np.ndarray):
        p = np.ascontiguousarray(params, dtype=np.float32)
        h = ctypes.c_void_p()
        rc = library().mas_ws_trainer_create(p.ctypes.data, p.size, ctypes.byref(h))
        if rc != MAS_OK:
            msg = library().mas_ws_trainer_last_error(None).decode()
            if rc == MAS_ERR_OOM:
                raise CudaOutOfMemoryError(msg)
            raise MasError(rc, msg or f"[MAS] error {rc}")
        self._t = h

    def __del__(self):
        t = getattr(self, "_t", None)
        if t is not None and t.value:
            try:
                library().mas_ws_trainer_destroy(t)
            except Exception:
                pass
            self._t = None

    def _check(self, rc: int) -> None:
        if rc == MAS_OK:
            return
        msg = library().mas_ws_trainer_last_error(self._t).decode()
        if rc == MAS_ERR_OOM:
            raise CudaOutOfMemoryError(msg)
        raise MasError(rc, msg or f"[MAS] error {rc}")

    def add_sample(self, solver: "Solver", b: np.ndarray, history, x_exact: np.ndarray) -> int:
        """Sample from ``solver`` (factorized with this step's matrix): b, the kept solutions (newest
        first, 2 to 4) and the exact solution, caller order. Returns the sample index."""
        b = np.ascontiguousarray(b, dtype=np.float64)
        hist = np.ascontiguousarray(np.stack([np.asarray(h, dtype=np.float64) for h in history]))
        x = np.ascontiguousarray(x_exact, dtype=np.float64)
        self._check(library().mas_ws_trainer_add_sample(self._t, solver._h, b.ctypes.data, hist.ctypes.data,
                                                         hist.shape[0], x.ctypes.data, b.size))
        return self.sample_count - 1

    @property
    def sample_count(self) -> int:
        return int(library().mas_ws_trainer_sample_count(self._t))

    def train(self, samples, lrs) -> np.ndarray:
        """One Adam step per listed sample (in order) with the given learning rates; the losses."""
        idx = np.ascontiguousarray(samples, dtype=np.int32)
        lr = np.ascontiguousarray(np.broadcast_to(np.asarray(lrs, dtype=np.float32), idx.shape))
        out = np.zeros(idx.size)
        self._check(library().mas_ws_trainer_train(self._t, idx.ctypes.data, lr.ctypes.data, idx.size,
                                                    out.ctypes.data))
        return out

    def evaluate(self, samples) -> np.ndarray:
        """rho of each listed sample under the current parameters."""
        idx = np.ascontiguousarray(samples, dtype=np.int32)
        out = np.zeros(idx.size)
        self._check(library().mas_ws_trainer_evaluate(self._t, idx.ctypes.data, idx.size, out.ctypes.data))
        return out

    def gradient(self, sample: int) -> tuple[float, np.ndarray]:
        """(loss, gradient) of one sample; no update."""
        g = np.zeros(_ws_params(), dtype=np.float32)
        loss = ctypes.c_double()
        self._check(library().mas_ws_trainer_gradient(self._t, int(sample), g.ctypes.data, g.size,
                                                       ctypes.byref(loss)))
        return loss.value, g

    def params(self) -> np.ndarray:
        p = np.zeros(_ws_params(), dtype=np.float32)
        self._check(library().mas_ws_trainer_get_params(self._t, p.ctypes.data, p.size))
        return p


def _ws_params() -> int:
    from . import warmstart

    return warmstart.PARAMS
