"""Shared helpers for the parity tests: map the solver's padded block order to the oracle's
partition-sorted order (the reference's `permutation`, MASSolver.cu:86-114)."""

from __future__ import annotations

import numpy as np

from oracle import oracle as O


def oracle_for(system, solver, block_dim: int = 3):
    """Oracle built on the same partition as `solver` (after factorize)."""
    padded = solver.ordering()
    perm, offsets = O.partition_from_padded(padded)
    return O.MasOracle(system.outer, system.inner, system.vals, system.n, block_dim, perm, offsets), padded


def real_to_padded_nodes(padded: np.ndarray, perm: np.ndarray) -> np.ndarray:
    """r2p[real] = padded node, where real = oracle's permuted block id."""
    r2p = np.empty(perm.size, dtype=np.int64)
    r2p[perm] = padded
    return r2p


def padded_to_oracle(vec_padded: np.ndarray, r2p: np.ndarray, bd: int) -> np.ndarray:
    return vec_padded.reshape(-1, bd)[r2p].reshape(-1)


def oracle_to_padded(vec_real: np.ndarray, r2p: np.ndarray, bd: int, nodes: int) -> np.ndarray:
    out = np.zeros((nodes, bd))
    out[r2p] = vec_real.reshape(-1, bd)
    return out.reshape(-1)


def packed_to_dense(packed: np.ndarray, N: int) -> np.ndarray:
    M = np.zeros((N, N))
    iu = np.triu_indices(N)
    M[iu] = packed
    M = M + M.T - np.diag(np.diag(M))
    return M
