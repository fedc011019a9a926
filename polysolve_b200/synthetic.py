"""Seeded synthetic tetrahedral-elasticity systems (the solver's benchmark workloads).

The heavy lifting is in ``csrc/synthetic.cpp`` (OpenMP C++). This module wraps it and defines
the named workloads:

* ``elasticity(N, ...)``   - one system on an N^3 grid (Kuhn 6-tet split, K + M/dt^2, Dirichlet
  on x = 0 as identity rows/cols).
* ``workload_cpu20()``     - 20^3, E = 1e5, no jitter (27,783 DOF).
* ``workload_grid80()``    - 80^3 jittered +-0.2h, E lognormal(ln 1e5, 1.0) (1,594,323 DOF).
* ``workload_contact80()`` - the 80^3 mesh plus 20,000 contact pairs (lognormal(ln 1e4, 1.5)).
* ``workload_batch64()``   - 64 systems with grid edge log-uniform in [8, 48], E sigma 0.5.
* ``workload_sequence60()`` - a 60^3 sequence with E_k = E_0 (1 + 0.3 sin(2 pi k / 50 + phase_e)).

Right-hand sides are N(0, 1) from numpy's PCG64 seeded generator.
"""

from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass, field

import numpy as np

from . import _build


class _SynParams(ctypes.Structure):
    _fields_ = [
        ("N", ctypes.c_int),
        ("young", ctypes.c_double),
        ("young_sigma", ctypes.c_double),
        ("poisson", ctypes.c_double),
        ("density", ctypes.c_double),
        ("dt", ctypes.c_double),
        ("jitter", ctypes.c_double),
        ("dirichlet_x0", ctypes.c_int),
        ("seed", ctypes.c_ulonglong),
        ("contact_pairs", ctypes.c_int),
        ("contact_k", ctypes.c_double),
        ("contact_sigma", ctypes.c_double),
        ("young_override", ctypes.POINTER(ctypes.c_double)),
    ]


_LIB = None


def _lib():
    global _LIB
    if _LIB is None:
        path = _build.SYN_LIB
        if not path.exists():
            _build.build_syn()
        lib = ctypes.CDLL(str(path))
        lib.syn_build.restype = ctypes.c_void_p
        lib.syn_build.argtypes = [ctypes.POINTER(_SynParams)]
        lib.syn_sizes.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int),
                                  ctypes.POINTER(ctypes.c_longlong), ctypes.POINTER(ctypes.c_int)]
        lib.syn_copy.argtypes = [ctypes.c_void_p] + [ctypes.c_void_p] * 4
        lib.syn_free.argtypes = [ctypes.c_void_p]
        lib.syn_young.argtypes = [ctypes.POINTER(_SynParams), ctypes.c_void_p]
        _LIB = lib
    return _LIB


@dataclass
class System:
    """A CSC system matrix (polysolve StiffnessMatrix layout) with vertex positions."""

    n: int
    outer: np.ndarray  # int32[n+1]
    inner: np.ndarray  # int32[nnz]
    vals: np.ndarray  # float64[nnz]
    positions: np.ndarray  # float64[nverts, 3]
    grid: int = 0
    meta: dict = field(default_factory=dict)

    @property
    def nnz(self) -> int:
        return int(self.inner.size)

    @property
    def nverts(self) -> int:
        return int(self.positions.shape[0])

    def scipy(self):
        import scipy.sparse as sp

        return sp.csc_matrix((self.vals, self.inner, self.outer), shape=(self.n, self.n))

    def matvec(self, x: np.ndarray) -> np.ndarray:
        return self.scipy() @ x


def _params(N, young, young_sigma, poisson, density, dt, jitter, dirichlet, seed, contact_pairs,
            contact_k, contact_sigma, young_override=None):
    p = _SynParams()
    p.N = int(N)
    p.young = float(young)
    p.young_sigma = float(young_sigma)
    p.poisson = float(poisson)
    p.density = float(density)
    p.dt = float(dt)
    p.jitter = float(jitter)
    p.dirichlet_x0 = 1 if dirichlet else 0
    p.seed = int(seed) & 0xFFFFFFFFFFFFFFFF
    p.contact_pairs = int(contact_pairs)
    p.contact_k = float(contact_k)
    p.contact_sigma = float(contact_sigma)
    if young_override is not None:
        p.young_override = young_override.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    else:
        p.young_override = ctypes.POINTER(ctypes.c_double)()
    return p


def elasticity(N: int, *, young: float = 1e5, young_sigma: float = 0.0, poisson: float = 0.3,
               density: float = 1000.0, dt: float = 1e-2, jitter: float = 0.0, dirichlet: bool = True,
               seed: int = 0, contact_pairs: int = 0, contact_k: float = 1e4, contact_sigma: float = 1.5,
               young_override: np.ndarray | None = None) -> System:
    """Assemble one tetrahedral elasticity system on an N^3 grid of the unit cube."""
    lib = _lib()
    yo = None
    if young_override is not None:
        yo = np.ascontiguousarray(young_override, dtype=np.float64)
        if yo.size != 6 * N ** 3:
            raise ValueError("young_override needs 6*N^3 values")
    p = _params(N, young, young_sigma, poisson, density, dt, jitter, dirichlet, seed, contact_pairs,
                contact_k, contact_sigma, yo)
    h = lib.syn_build(ctypes.byref(p))
    if not h:
        raise ValueError("invalid synthetic system parameters")
    try:
        n = ctypes.c_int()
        nnz = ctypes.c_longlong()
        nv = ctypes.c_int()
        lib.syn_sizes(h, ctypes.byref(n), ctypes.byref(nnz), ctypes.byref(nv))
        if nnz.value >= 2 ** 31:
            raise ValueError("system too large for int32 CSC")
        outer = np.empty(n.value + 1, dtype=np.int32)
        inner = np.empty(nnz.value, dtype=np.int32)
        vals = np.empty(nnz.value, dtype=np.float64)
        pos = np.empty((nv.value, 3), dtype=np.float64)
        lib.syn_copy(h, outer.ctypes.data, inner.ctypes.data, vals.ctypes.data, pos.ctypes.data)
    finally:
        lib.syn_free(h)
    meta = dict(N=N, young=young, young_sigma=young_sigma, poisson=poisson, density=density, dt=dt,
                jitter=jitter, dirichlet=dirichlet, seed=seed, contact_pairs=contact_pairs)
    return System(n=n.value, outer=outer, inner=inner, vals=vals, positions=pos, grid=N, meta=meta)


def element_young(N: int, *, young: float = 1e5, young_sigma: float = 0.0, seed: int = 0) -> np.ndarray:
    """The per-element Young's moduli ``elasticity`` draws for these parameters."""
    lib = _lib()
    p = _params(N, young, young_sigma, 0.3, 1000.0, 1e-2, 0.0, True, seed, 0, 0.0, 0.0)
    out = np.empty(6 * N ** 3, dtype=np.float64)
    lib.syn_young(ctypes.byref(p), out.ctypes.data)
    return out


def rhs(n: int, seed: int = 0, count: int | None = None) -> np.ndarray:
    """N(0, 1) right-hand side(s) from numpy's PCG64 generator."""
    rng = np.random.Generator(np.random.PCG64(seed))
    if count is None:
        return rng.standard_normal(n)
    return rng.standard_normal((count, n))


# ---------------------------------------------------------------------------------------------
# Named workloads
# ---------------------------------------------------------------------------------------------

def workload_cpu20(seed: int = 0) -> System:
    """20^3 grid, E = 1e5, nu = 0.3, rho = 1000, dt = 1e-2, Dirichlet x = 0 (27,783 DOF)."""
    return elasticity(20, seed=seed)


def workload_grid80(seed: int = 0, N: int = 80) -> System:
    """80^3 grid jittered +-0.2h, E lognormal(ln 1e5, 1.0) per element (1,594,323 DOF)."""
    return elasticity(N, young_sigma=1.0, jitter=0.2, seed=seed)


def workload_contact80(seed: int = 0, N: int = 80, pairs: int = 20000) -> System:
    """The jittered 80^3 mesh plus ``pairs`` contact couplings k n n^T, k ~ lognormal(ln 1e4, 1.5)."""
    return elasticity(N, young_sigma=1.0, jitter=0.2, seed=seed, contact_pairs=pairs,
                      contact_k=1e4, contact_sigma=1.5)


def batch_edges(count: int = 64, seed: int = 0, lo: int = 8, hi: int = 48) -> list[int]:
    """Grid edges drawn log-uniform in [lo, hi]."""
    rng = np.random.Generator(np.random.PCG64(seed + 7919))
    u = rng.uniform(math.log(lo), math.log(hi), size=count)
    return [int(round(math.exp(v))) for v in u]


def workload_batch64(seed: int = 0, count: int = 64, lo: int = 8, hi: int = 48) -> list[System]:
    """Independent systems built like the 20^3 one, edges log-uniform in [lo, hi], E sigma 0.5."""
    return [elasticity(N, young_sigma=0.5, seed=seed * 1000 + s) for s, N in
            enumerate(batch_edges(count, seed, lo, hi))]


def sequence_young(N: int, k: int, seed: int = 0, sigma: float = 0.8, period: int = 50) -> np.ndarray:
    """E_k = E_0 (1 + 0.3 sin(2 pi k / period + phase_e)), E_0 lognormal(ln 1e5, sigma) per element."""
    e0 = element_young(N, young=1e5, young_sigma=sigma, seed=seed)
    rng = np.random.Generator(np.random.PCG64(seed + 104729))
    phase = rng.uniform(0.0, 2.0 * math.pi, size=e0.size)
    return e0 * (1.0 + 0.3 * np.sin(2.0 * math.pi * k / period + phase))


def sequence_rhs(positions: np.ndarray, k: int, seed: int = 0, bumps: int = 8, steps: int = 200) -> np.ndarray:
    """b_k: a sum of ``bumps`` seeded Gaussian bumps whose centres drift linearly in k."""
    rng = np.random.Generator(np.random.PCG64(seed + 15485863))
    c0 = rng.uniform(0.2, 0.8, size=(bumps, 3))
    c1 = rng.uniform(0.2, 0.8, size=(bumps, 3))
    amp = rng.standard_normal((bumps, 3))
    width = rng.uniform(0.05, 0.15, size=bumps)
    t = k / max(steps - 1, 1)
    centres = (1.0 - t) * c0 + t * c1
    b = np.zeros_like(positions)
    for q in range(bumps):
        d2 = np.sum((positions - centres[q]) ** 2, axis=1)
        b += np.exp(-d2 / (2.0 * width[q] ** 2))[:, None] * amp[q][None, :]
    return b.reshape(-1)


def workload_sequence60(k: int, seed: int = 0, N: int = 60):
    """Step k of the 60^3 sequence: (system, b_k)."""
    sys_k = elasticity(N, jitter=0.2, seed=seed, young_override=sequence_young(N, k, seed))
    return sys_k, sequence_rhs(sys_k.positions, k, seed)
