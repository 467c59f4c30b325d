"""SNP-block jackknife and rank-revealing normal-equation solves on the GPU.

Mirrors the numerical core of SUMMIT's downstream fits: contiguous jackknife
blocks (``inference/jackknife.py:109-214``), the symmetric spectral solve of
``context/fit.py:435-525`` (symmetrize, eigendecompose, keep eigenvalues above
max(100 eps scale, rtol leading), solve on the kept subspace), and delete-one
replicate standard errors (``inference/gxe.py:2052-2057``).  All arithmetic on
the device in FP64 (liblds); there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import check, ptr

DEFAULT_SOLVE_RTOL = 1.0e-10


def equal_count_block_boundaries(M: int, B: int):
    starts, ends = np.empty(B, np.int64), np.empty(B, np.int64)
    check(_lib.load().lds_block_boundaries(int(M), int(B), None, 1, ptr(starts), ptr(ends)))
    return starts, ends


def weighted_contiguous_block_boundaries(mass, B: int, *, min_snps: int = 1):
    mass = np.ascontiguousarray(mass, dtype=np.float64).ravel()
    starts, ends = np.empty(B, np.int64), np.empty(B, np.int64)
    check(_lib.load().lds_block_boundaries(mass.size, int(B), ptr(mass), int(min_snps),
                                           ptr(starts), ptr(ends)))
    return starts, ends


def solve_normal_equations(matrix, rhs, rtol: float | None = None,
                           require_full_rank: bool = True) -> dict:
    """Solve one system, or a stack (matrix n x K x K, rhs n x K)."""
    A = np.asarray(matrix, dtype=np.float64)
    b = np.asarray(rhs, dtype=np.float64)
    single = A.ndim == 2
    if single:
        A, b = A[None], b[None]
    n, K = A.shape[0], A.shape[1]
    if A.shape != (n, K, K) or b.shape != (n, K):
        raise ValueError("Normal-equation shapes are incompatible.")
    sys_ = np.ascontiguousarray(np.concatenate([A.reshape(n, K * K), b], axis=1))
    x = np.empty((n, K))
    rank = np.empty(n, dtype=np.int32)
    eig = np.empty((n, K))
    check(_lib.load().lds_sym_solve(ptr(sys_), n, K,
                                    float(DEFAULT_SOLVE_RTOL if rtol is None else rtol),
                                    int(bool(require_full_rank)), ptr(x), ptr(rank), ptr(eig), 0))
    if single:
        return {"coefficients": x[0], "rank": int(rank[0]), "eigenvalues": eig[0]}
    return {"coefficients": x, "rank": rank, "eigenvalues": eig}


def jackknife_normal_equations(terms, starts, ends, rtol: float | None = None) -> dict:
    """terms: M x (K*K + K) per-SNP [vec(A_j), b_j].  Returns the full solution,
    delete-one-block replicates, their SE and covariance."""
    T = np.ascontiguousarray(terms, dtype=np.float64)
    M, P = T.shape
    K = int(round((-1 + np.sqrt(1 + 4 * P)) / 2))
    if K * K + K != P:
        raise ValueError("terms must have K*K + K columns")
    s = np.ascontiguousarray(starts, dtype=np.int64)
    e = np.ascontiguousarray(ends, dtype=np.int64)
    B = s.size
    theta, reps = np.empty(K), np.empty((B, K))
    se, cov = np.empty(K), np.empty((K, K))
    check(_lib.load().lds_jackknife_normal_equations(
        ptr(T), M, K, ptr(s), ptr(e), B, float(DEFAULT_SOLVE_RTOL if rtol is None else rtol),
        ptr(theta), ptr(reps), ptr(se), ptr(cov), 0))
    return {"theta": theta, "replicates": reps, "se": se, "cov": cov}
