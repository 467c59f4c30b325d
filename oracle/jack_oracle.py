"""ORACLE — numpy restatement of the jackknife / normal-equation numerics
(test infrastructure only): the symmetric spectral solve of
context/fit.py:435-525 and the delete-one replicate SE of
inference/gxe.py:2052-2057.  Pinned to tests/golden/jackknife_golden.npz,
which the reference's own Python wrote."""
from __future__ import annotations

import numpy as np


def solve(matrix, rhs, rtol=1e-10):
    A = np.asarray(matrix, dtype=np.float64)
    b = np.asarray(rhs, dtype=np.float64)
    scale = max(float(np.max(np.abs(A), initial=0.0)), 1.0)
    if float(np.max(np.abs(A - A.T), initial=0.0)) > 2.0e-10 * scale:
        raise ValueError("Normal matrix has material asymmetry")
    S = 0.5 * (A + A.T)
    lam, V = np.linalg.eigh(S)
    tol = max(100.0 * np.finfo(np.float64).eps * scale, rtol * float(np.max(np.abs(lam))))
    keep = np.abs(lam) > tol
    Vk = V[:, keep]
    if Vk.shape[1] == 0:
        return np.zeros_like(b), 0
    ev = np.einsum("ni,nm,mi->i", Vk, S, Vk)
    return Vk @ ((Vk.T @ b) / ev), int(keep.sum())


def jackknife(terms, starts, ends, rtol=1e-10):
    M, P = terms.shape
    K = int(round((-1 + np.sqrt(1 + 4 * P)) / 2))
    tot = terms.sum(0)
    theta = solve(tot[:K * K].reshape(K, K), tot[K * K:], rtol)[0]
    reps = []
    for s, e in zip(starts, ends):
        d = tot - terms[s:e].sum(0)
        reps.append(solve(d[:K * K].reshape(K, K), d[K * K:], rtol)[0])
    reps = np.asarray(reps)
    B = reps.shape[0]
    c = reps.mean(0)
    return theta, reps, np.sqrt((B - 1.0) / B * ((reps - c) ** 2).sum(0))
