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


# ---------------------------------------------------------------------------
# Drop-in for solve_context_normal_equations (context/fit.py:474-525) and its
# _rank_diagnostics (:435-471): the same result fields, errors and messages,
# with the eigendecomposition, the retained-subspace solve and the residual
# computed on the device (lds_sym_solve_diag).
# ---------------------------------------------------------------------------
from dataclasses import dataclass  # noqa: E402


@dataclass(frozen=True)
class SymmetricRankDiagnostics:
    """Fields of the reference's ``SymmetricRankDiagnostics`` (context/oracle.py:67-74)."""
    symmetry_error: float
    eigenvalues: np.ndarray
    singular_values: np.ndarray
    rank: int
    condition_number: float
    tolerance: float
    null_space: np.ndarray


@dataclass(frozen=True)
class ContextSolveResult:
    """Fields of the reference's ``ContextSolveResult`` (context/fit.py:119-130)."""
    coefficients: np.ndarray
    diagnostics: SymmetricRankDiagnostics
    rank: int
    condition_number: float
    solve_residual: np.ndarray
    relative_residual: float
    minimum_gram_eigenvalue: float
    retained_directions: np.ndarray
    null_space: np.ndarray
    relative_tolerance: float
    absolute_tolerance: float


class ContextRankError(ValueError):
    """A declared normal system is not identifiable (context/fit.py:228-240)."""

    def __init__(self, message: str, *, diagnostics: SymmetricRankDiagnostics,
                 component_names=()):
        super().__init__(message)
        self.diagnostics = diagnostics
        self.component_names = tuple(component_names)


def _finite_float64(name: str, value, ndim: int) -> np.ndarray:
    array = np.asarray(value, dtype=np.float64)
    if array.ndim != ndim:
        raise ValueError(f"{name} must be {ndim}-dimensional; got {array.shape}.")
    if not np.all(np.isfinite(array)):
        raise ValueError(f"{name} contains non-finite values.")
    return array


def _readonly(a: np.ndarray) -> np.ndarray:
    a = np.array(a, dtype=np.float64, copy=True)
    a.setflags(write=False)
    return a


def solve_context_normal_equations(equations, *, rtol: float | None = None,
                                   require_full_rank: bool = True) -> ContextSolveResult:
    """Rank-revealing symmetric solve of ``equations.matrix @ x = equations.rhs``.

    ``equations`` is the reference's ``ContextNormalEquations`` or any object
    with ``matrix`` (n x n) and ``rhs`` (n) attributes (``component_names``
    optional).  Follows context/fit.py:474-525: symmetrize, eigendecompose,
    keep |lambda| > max(100 eps scale, rtol |lambda|_max), solve on the kept
    eigenvectors with Rayleigh-quotient eigenvalues.  The directional
    target/source systems (``target_source``), which the reference solves by
    SVD in context/target_jackknife.py, are not handled here.  n <= 96.
    """
    if getattr(equations, "target_source", False):
        raise ValueError("Directional target/source normal systems are solved by SVD "
                         "(context/target_jackknife.py); this solver handles symmetric systems.")
    matrix = _finite_float64("normal matrix", equations.matrix, ndim=2)
    rhs = _finite_float64("normal RHS", equations.rhs, ndim=1)
    if matrix.shape[0] != matrix.shape[1] or rhs.shape != (matrix.shape[0],):
        raise ValueError("Normal-equation shapes are incompatible.")
    relative_tolerance = DEFAULT_SOLVE_RTOL if rtol is None else float(rtol)
    if not np.isfinite(relative_tolerance) or relative_tolerance <= 0.0:
        raise ValueError("rtol must be finite and positive.")
    n = matrix.shape[0]
    names = tuple(getattr(equations, "component_names", ()) or ())
    scale = max(float(np.max(np.abs(matrix), initial=0.0)), 1.0)
    absolute_tolerance = 100.0 * np.finfo(np.float64).eps * scale
    if n == 0:
        # (the reference fails on an empty system when it reads its smallest eigenvalue)
        raise ValueError("Normal-equation system is empty.")
    system = np.ascontiguousarray(np.concatenate([matrix.reshape(-1), rhs]))
    x = np.empty(n)
    rank = np.empty(1, dtype=np.int32)
    eig = np.empty(n)
    vecs = np.empty((n, n))
    resid = np.empty(n)
    asym = np.empty(1)
    tol = np.empty(1)
    status = np.empty(1, dtype=np.int32)
    check(_lib.load().lds_sym_solve_diag(ptr(system), 1, n, relative_tolerance, ptr(x), ptr(rank),
                                         ptr(eig), ptr(vecs), ptr(resid), ptr(asym), ptr(tol),
                                         ptr(status)))
    asymmetry = float(asym[0])
    if status[0] & 1:
        raise ValueError(f"Normal matrix has material asymmetry ({asymmetry:.6g}).")
    tolerance = float(tol[0])
    retained = np.abs(eig) > tolerance
    r = int(rank[0])
    singular_values = np.sort(np.abs(eig))[::-1]
    leading = float(singular_values[0])
    condition = (float("inf") if r < n or r == 0
                 else float(leading / np.min(np.abs(eig[retained]))))
    diag = SymmetricRankDiagnostics(
        symmetry_error=asymmetry, eigenvalues=_readonly(eig),
        singular_values=_readonly(singular_values), rank=r, condition_number=condition,
        tolerance=tolerance, null_space=_readonly(vecs[:, ~retained]))
    if require_full_rank and r != n:
        raise ContextRankError(
            "Contextual normal system is not identifiable: "
            f"rank {r} of {n} at tolerance {tolerance:.6g}.",
            diagnostics=diag, component_names=names)
    return ContextSolveResult(
        coefficients=_readonly(x), diagnostics=diag, rank=r, condition_number=condition,
        solve_residual=_readonly(resid),
        relative_residual=float(np.linalg.norm(resid) / max(1.0, np.linalg.norm(rhs))),
        minimum_gram_eigenvalue=float(eig[0]), retained_directions=_readonly(vecs[:, retained]),
        null_space=diag.null_space, relative_tolerance=relative_tolerance,
        absolute_tolerance=float(absolute_tolerance))
