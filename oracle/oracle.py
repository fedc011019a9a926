"""ORACLE — test infrastructure only (the checker, never the product path).

Python side of the CPU restatement of polysolve's MAS-PCG (``mas_oracle.cpp``), plus:

* ``morton_order``: the Morton (Z-order) vertex ordering that the solver's factorize uses when
  vertex positions are given, restated in numpy so the product's permutation can be checked bit
  for bit. (The reference partitions with KaMinPar, mas_utils/GraphPartition.cpp:176-289, which is
  not in this image; given a partition, everything downstream restates the reference.)
* ``dense_mas_operator``: an independent dense numpy construction of
  M^-1 = sum_l P_l A_l^-1 P_l^T from the coarse maps, used to cross-check the C++ restatement on
  small systems.

Parity status: parity unpinned — the reference's MAS path cannot be built here and its tests
carry no golden vectors for MAS (only residual thresholds on unshipped data).

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline legs import this.
"""

from __future__ import annotations

import ctypes
import subprocess
from dataclasses import dataclass
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "libmas_oracle.so"
BANK = 32
MAX_COARSE = 4
LEVELS = MAX_COARSE + 1


def build(force: bool = False) -> Path:
    """Compile the C++ restatement (g++ -O2 -fopenmp)."""
    src = HERE / "mas_oracle.cpp"
    if force or not LIB_PATH.exists() or LIB_PATH.stat().st_mtime < src.stat().st_mtime:
        cmd = ["g++", "-O2", "-std=c++17", "-fopenmp", "-fPIC", "-shared", "-o", str(LIB_PATH), str(src)]
        res = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
        if res.returncode != 0:
            raise RuntimeError("oracle build failed:\n" + res.stdout)
    return LIB_PATH


class PcgParams(ctypes.Structure):
    _fields_ = [
        ("max_iter", ctypes.c_int),
        ("rel_tol", ctypes.c_double),
        ("abs_tol", ctypes.c_double),
        ("use_preconditioned_residual_norm", ctypes.c_int),
        ("true_residual_period", ctypes.c_int),
        ("check_period", ctypes.c_int),
        ("use_initial_guess", ctypes.c_int),
        ("mas_fp32", ctypes.c_int),
        ("polak_ribiere", ctypes.c_int),
    ]


class PcgResult(ctypes.Structure):
    _fields_ = [
        ("iterations", ctypes.c_int),
        ("status", ctypes.c_int),
        ("residual_norm", ctypes.c_double),
        ("rz0", ctypes.c_double),
        ("rr0", ctypes.c_double),
    ]


STATUS_NAMES = {0: "Running", 1: "Reach relative tolerance", 2: "Reach absolute tolerance",
                3: "Reach max iterations", -1: "Invalid initial residual"}

_LIB = None


def lib():
    global _LIB
    if _LIB is None:
        build()
        L = ctypes.CDLL(str(LIB_PATH))
        vp = ctypes.c_void_p
        L.orc_create.restype = vp
        L.orc_create.argtypes = [ctypes.c_int, vp, vp, vp, ctypes.c_int, vp, ctypes.c_int, vp]
        L.orc_free.argtypes = [vp]
        L.orc_inverse_ok.argtypes = [vp]
        L.orc_sizes.argtypes = [vp, vp]
        L.orc_levels.argtypes = [vp, vp, vp, vp, vp]
        L.orc_export_bsr.argtypes = [vp, vp, vp, vp]
        L.orc_export_maps.argtypes = [vp, vp, vp]
        L.orc_export_inverses.argtypes = [vp, vp]
        L.orc_apply.argtypes = [vp, vp, vp]
        L.orc_apply_storage.argtypes = [vp, vp, vp, ctypes.c_int]
        L.orc_half_round.argtypes = [vp, vp, ctypes.c_longlong]
        L.orc_spmv.argtypes = [vp, vp, vp]
        L.orc_pcg.argtypes = [vp, vp, vp, ctypes.POINTER(PcgParams), ctypes.POINTER(PcgResult)]
        L.orc_jacobi_pcg.argtypes = [ctypes.c_int, vp, vp, vp, vp, vp, ctypes.c_double, ctypes.c_int,
                                     ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_double)]
        _LIB = L
    return _LIB


def _p(a: np.ndarray):
    return a.ctypes.data


# ---------------------------------------------------------------------------------------------
# Orderings
# ---------------------------------------------------------------------------------------------

def _spread3(v: np.ndarray) -> np.ndarray:
    """Spread the low 21 bits of v so bit i lands at bit 3i."""
    v = v.astype(np.uint64) & np.uint64(0x1FFFFF)
    v = (v | (v << np.uint64(32))) & np.uint64(0x1F00000000FFFF)
    v = (v | (v << np.uint64(16))) & np.uint64(0x1F0000FF0000FF)
    v = (v | (v << np.uint64(8))) & np.uint64(0x100F00F00F00F00F)
    v = (v | (v << np.uint64(4))) & np.uint64(0x10C30C30C30C30C3)
    v = (v | (v << np.uint64(2))) & np.uint64(0x1249249249249249)
    return v


def morton_codes(positions: np.ndarray) -> np.ndarray:
    """63-bit Morton codes, coordinates quantised in units of the mean point spacing
    h = (bounding-box volume / count)^(1/dims), rounded to nearest, clamped to 21 bits."""
    pos = np.asarray(positions, dtype=np.float64).reshape(-1, 3)
    V = pos.shape[0]
    lo = pos.min(axis=0)
    ext = pos.max(axis=0) - lo
    dims = [d for d in range(3) if ext[d] > 0.0]
    if dims:
        vol = 1.0
        for d in dims:
            vol = vol * float(ext[d])
        h = float(np.power(vol / V, 1.0 / len(dims)))
        scale = min(1.0 / h, 2097151.0 / float(np.max(ext)))
        q = np.floor((pos - lo) * scale + 0.5)
    else:
        q = np.zeros_like(pos)
    q = np.clip(q, 0, 2097151).astype(np.uint64)
    return _spread3(q[:, 0]) | (_spread3(q[:, 1]) << np.uint64(1)) | (_spread3(q[:, 2]) << np.uint64(2))


def isolated_blocks(outer, inner, n: int, block_dim: int) -> np.ndarray:
    """Block rows with no off-diagonal block (identity / Dirichlet rows)."""
    V = -(-n // block_dim)
    outer = np.asarray(outer, dtype=np.int64)
    inner = np.asarray(inner, dtype=np.int64)
    colblk = np.repeat(np.arange(n) // block_dim, np.diff(outer))
    rowblk = inner // block_dim
    off = rowblk != colblk
    iso = np.ones(V, dtype=bool)
    iso[rowblk[off]] = False
    iso[colblk[off]] = False
    return iso


def morton_padded(positions: np.ndarray, isolated: np.ndarray) -> np.ndarray:
    """Padded id (bank * 32 + lane) per block: coupled blocks in Morton order, chunked by 32,
    then the isolated blocks in Morton order from the next bank on."""
    codes = morton_codes(positions)
    V = codes.size
    iso = np.asarray(isolated, dtype=bool)
    order = np.lexsort((np.arange(V), codes, iso.astype(np.uint8)))
    nreal = int((~iso).sum())
    padded = np.empty(V, dtype=np.int64)
    padded[order[:nreal]] = np.arange(nreal)
    base = -(-nreal // BANK) * BANK
    padded[order[nreal:]] = base + np.arange(V - nreal)
    return padded


def morton_order(positions: np.ndarray, isolated: np.ndarray | None = None) -> tuple[np.ndarray, np.ndarray]:
    """Reference-style (perm, part_offsets) of the Morton partition."""
    pos = np.asarray(positions).reshape(-1, 3)
    iso = np.zeros(pos.shape[0], dtype=bool) if isolated is None else isolated
    return partition_from_padded(morton_padded(pos, iso))


def partition_from_padded(padded_ids: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    """From a padded numbering (old block -> bank*32 + lane) to the reference's representation:
    perm[old] = gap-free rank, part_offsets[P+1]."""
    padded_ids = np.asarray(padded_ids, dtype=np.int64)
    V = padded_ids.size
    order = np.argsort(padded_ids, kind="stable")
    perm = np.empty(V, dtype=np.int32)
    perm[order] = np.arange(V, dtype=np.int32)
    banks = padded_ids[order] // BANK
    P = int(banks.max()) + 1 if V else 0
    counts = np.bincount(banks, minlength=P)
    offsets = np.zeros(P + 1, dtype=np.int32)
    np.cumsum(counts, out=offsets[1:])
    return perm, offsets


# ---------------------------------------------------------------------------------------------
# The restated solver
# ---------------------------------------------------------------------------------------------

@dataclass
class Structure:
    V: int
    nnzb: int
    P: int
    padded: int
    level_num: int
    total_mats: int
    mat_dim: int
    total_level_nodes: int
    cco_nums: np.ndarray
    mat_counts: np.ndarray
    mat_offsets: np.ndarray
    level_offsets: np.ndarray


class MasOracle:
    """CPU MAS-PCG restating MASSolverImpl + MASPreconditioner for a given partition."""

    def __init__(self, outer, inner, vals, n: int, block_dim: int, perm, part_offsets):
        L = lib()
        self.n = int(n)
        self.bd = int(block_dim)
        self._keep = [np.ascontiguousarray(outer, dtype=np.int32), np.ascontiguousarray(inner, dtype=np.int32),
                      np.ascontiguousarray(vals, dtype=np.float64)]
        self.perm = np.ascontiguousarray(perm, dtype=np.int32)
        self.part_offsets = np.ascontiguousarray(part_offsets, dtype=np.int32)
        o, i, v = self._keep
        self.h = L.orc_create(self.n, _p(o), _p(i), _p(v), self.bd, _p(self.perm),
                              int(self.part_offsets.size - 1), _p(self.part_offsets))
        if not self.h:
            raise ValueError("oracle: invalid matrix, permutation or partition")
        s = np.zeros(8, dtype=np.int32)
        L.orc_sizes(self.h, _p(s))
        cco = np.zeros(4, dtype=np.int32)
        mc = np.zeros(5, dtype=np.int32)
        mo = np.zeros(5, dtype=np.int32)
        lo = np.zeros(5, dtype=np.int32)
        L.orc_levels(self.h, _p(cco), _p(mc), _p(mo), _p(lo))
        self.s = Structure(int(s[0]), int(s[1]), int(s[2]), int(s[3]), int(s[4]), int(s[5]), int(s[6]),
                           int(s[7]), cco, mc, mo, lo)

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_free(self.h)
            self.h = None

    @property
    def inverse_ok(self) -> bool:
        return bool(lib().orc_inverse_ok(self.h))

    def bsr(self):
        s = self.s
        rows = np.empty(s.V + 1, dtype=np.int32)
        cols = np.empty(s.nnzb, dtype=np.int32)
        vals = np.empty(s.nnzb * self.bd * self.bd, dtype=np.float64)
        lib().orc_export_bsr(self.h, _p(rows), _p(cols), _p(vals))
        return rows, cols, vals.reshape(s.nnzb, self.bd, self.bd)

    def maps(self):
        r2p = np.empty(self.s.V, dtype=np.int32)
        cmap = np.empty(self.s.V * MAX_COARSE, dtype=np.int32)
        lib().orc_export_maps(self.h, _p(r2p), _p(cmap))
        return r2p, cmap.reshape(self.s.V, MAX_COARSE)

    def inverses(self) -> np.ndarray:
        storage = self.s.mat_dim * (self.s.mat_dim + 1) // 2
        out = np.empty(self.s.total_mats * storage, dtype=np.float64)
        lib().orc_export_inverses(self.h, _p(out))
        return out.reshape(self.s.total_mats, storage)

    # vectors below are in permuted block order (length V * bd)
    def apply(self, r: np.ndarray, storage: int = 0) -> np.ndarray:
        """z = M^-1 r; storage 1 / 16 emulates FP32 / scaled binary16 inverses (FP64 arithmetic)."""
        r = np.ascontiguousarray(r, dtype=np.float64)
        z = np.empty_like(r)
        if storage:
            lib().orc_apply_storage(self.h, _p(r), _p(z), int(storage))
        else:
            lib().orc_apply(self.h, _p(r), _p(z))
        return z

    def spmv(self, x: np.ndarray) -> np.ndarray:
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.empty_like(x)
        lib().orc_spmv(self.h, _p(x), _p(y))
        return y

    def to_block_order(self, v: np.ndarray) -> np.ndarray:
        """Original order (length n) -> permuted block order (length V*bd, zero padded)."""
        V, bd = self.s.V, self.bd
        out = np.zeros(V * bd)
        full = np.zeros(V * bd)
        full[: self.n] = v
        out.reshape(V, bd)[self.perm] = full.reshape(V, bd)
        return out

    def from_block_order(self, v: np.ndarray) -> np.ndarray:
        V, bd = self.s.V, self.bd
        return v.reshape(V, bd)[self.perm].reshape(-1)[: self.n]

    def pcg(self, b: np.ndarray, x0: np.ndarray | None = None, *, max_iter=5000, rel_tol=1e-5, abs_tol=1e-8,
            use_preconditioned_residual_norm=False, true_residual_period=4, check_period=10,
            use_initial_guess=False, mas_fp32=False, polak_ribiere=False):
        """MAS-PCG with the reference's defaults (MASSolver.cu:137-143, 498-583)."""
        prm = PcgParams(max_iter, rel_tol, abs_tol, int(use_preconditioned_residual_norm), true_residual_period,
                        check_period, int(use_initial_guess), int(mas_fp32), int(polak_ribiere))
        res = PcgResult()
        b = np.ascontiguousarray(b, dtype=np.float64)
        x = np.zeros(self.n) if x0 is None else np.array(x0, dtype=np.float64)
        rc = lib().orc_pcg(self.h, _p(b), _p(x), ctypes.byref(prm), ctypes.byref(res))
        info = dict(solver_iter=res.iterations, solver_error=res.residual_norm,
                    solver_status=STATUS_NAMES.get(res.status, "Unknown"), status_code=res.status, rz0=res.rz0,
                    rr0=res.rr0, rc=rc)
        return x, info


def half_round(v: np.ndarray) -> np.ndarray:
    """The oracle's float -> nearest binary16 rounding (as float32), for checking it."""
    v = np.ascontiguousarray(v, dtype=np.float32)
    out = np.empty_like(v)
    lib().orc_half_round(_p(v), _p(out), v.size)
    return out


def jacobi_pcg(outer, inner, vals, n: int, b: np.ndarray, tol: float = 1e-8, max_iter: int | None = None,
               x0: np.ndarray | None = None):
    """Jacobi-preconditioned CG restating Eigen::ConjugateGradient's algorithm (CPU baseline)."""
    o = np.ascontiguousarray(outer, dtype=np.int32)
    i = np.ascontiguousarray(inner, dtype=np.int32)
    v = np.ascontiguousarray(vals, dtype=np.float64)
    b = np.ascontiguousarray(b, dtype=np.float64)
    x = np.zeros(n) if x0 is None else np.array(x0, dtype=np.float64)
    it = ctypes.c_int()
    rr = ctypes.c_double()
    lib().orc_jacobi_pcg(n, _p(o), _p(i), _p(v), _p(b), _p(x), float(tol), int(max_iter or 2 * n), ctypes.byref(it),
                         ctypes.byref(rr))
    return x, it.value, rr.value


# ---------------------------------------------------------------------------------------------
# Independent dense check (small systems only)
# ---------------------------------------------------------------------------------------------

def dense_mas_operator(orc: MasOracle) -> np.ndarray:
    """M^-1 = sum_l P_l (P_l^T A P_l restricted to banks)^-1 P_l^T, built densely in numpy from
    the oracle's maps and BSR (permuted block order). Virtual slots get identity rows."""
    s = orc.s
    bd = orc.bd
    rows, cols, vals = orc.bsr()
    V = s.V
    A = np.zeros((V * bd, V * bd))
    for r in range(V):
        for k in range(rows[r], rows[r + 1]):
            A[r * bd:(r + 1) * bd, cols[k] * bd:(cols[k] + 1) * bd] = vals[k]
    r2p, cmap = orc.maps()
    Minv = np.zeros_like(A)
    groupings = [r2p] + [cmap[:, lv] for lv in range(s.level_num)]
    for g in groupings:
        nodes_of_slot = {}
        for v_, slot in enumerate(g):
            nodes_of_slot.setdefault(int(slot), []).append(v_)
        nslots = max(nodes_of_slot) + 1
        nbank = (nslots + BANK - 1) // BANK
        for bank in range(nbank):
            N = BANK * bd
            # P: (V*bd) x N, columns = slot*bd + comp
            Pm = np.zeros((V * bd, N))
            used = np.zeros(N, dtype=bool)
            for lane in range(BANK):
                slot = bank * BANK + lane
                for v_ in nodes_of_slot.get(slot, []):
                    for c in range(bd):
                        Pm[v_ * bd + c, lane * bd + c] = 1.0
                        used[lane * bd + c] = True
            Ac = Pm.T @ A @ Pm
            for i in range(N):
                if Ac[i, i] == 0.0:
                    Ac[i, i] = 1.0
            Minv += Pm @ np.linalg.inv(Ac) @ Pm.T
    return Minv
