"""Golden vectors for the jackknife / normal-equation row, written by the
reference's own Python (src/summit/inference/jackknife.py block boundaries,
src/summit/context/fit.py solve_context_normal_equations, the replicate SE of
src/summit/inference/gxe.py:2052-2057), imported from the reference tree
named by the SUMMIT_REFERENCE_DIR environment variable.

    SUMMIT_REFERENCE_DIR=<SUMMIT checkout> python tests/golden/make_golden_jackknife.py
"""
from __future__ import annotations

import os
import sys
from pathlib import Path

import numpy as np

if not os.environ.get("SUMMIT_REFERENCE_DIR"):
    raise SystemExit("set SUMMIT_REFERENCE_DIR to the SUMMIT source tree")
REF = Path(os.environ["SUMMIT_REFERENCE_DIR"]) / "src"
sys.path.insert(0, str(REF))

from summit.context import fit as F  # noqa: E402
from summit.inference import jackknife as J  # noqa: E402

HERE = Path(__file__).resolve().parent


def solve(A, b, rtol=None):
    K = A.shape[0]
    eq = F.ContextNormalEquations(
        matrix=A, rhs=b, traces=np.zeros(K), component_names=tuple(f"c{i}" for i in range(K)),
        genetic_count=K, annotation_masses=np.ones(1), deleted_groups=(),
        reference_genetic_gram=np.eye(K), transferred_genetic_gram=np.eye(K), reference_n=1000,
        study_n=1000)
    r = F.solve_context_normal_equations(eq, rtol=rtol, require_full_rank=False)
    return r.coefficients, r.rank


def main():
    rng = np.random.default_rng(20261203)
    out = {}
    # block boundaries
    for i, (M, B) in enumerate([(1000, 200), (777, 13), (5, 5), (100_003, 200)]):
        s, e = J._equal_count_block_boundaries(M, B)
        out[f"eq{i}_M"], out[f"eq{i}_B"], out[f"eq{i}_starts"], out[f"eq{i}_ends"] = M, B, s, e
    mass = rng.gamma(2.0, 1.0, size=1000)
    mass[::17] = 0.0
    mass[5] = np.nan
    for i, (B, ms) in enumerate([(37, 3), (200, 1), (10, 50)]):
        s, e = J._weighted_contiguous_block_boundaries(mass, B, min_snps=ms)
        out[f"w{i}_B"], out[f"w{i}_min"], out[f"w{i}_starts"], out[f"w{i}_ends"] = B, ms, s, e
    out["mass"] = mass
    # normal-equation solves: well conditioned, larger, rank deficient, scaled
    systems = []
    X = rng.normal(size=(50, 5))
    systems.append((X.T @ X, rng.normal(size=5)))
    X = rng.normal(size=(400, 24))
    systems.append((X.T @ X / 400.0, rng.normal(size=24)))
    X = rng.normal(size=(30, 4)) @ rng.normal(size=(4, 6))
    systems.append((X.T @ X, rng.normal(size=6)))
    X = rng.normal(size=(60, 7))
    systems.append((1e6 * (X.T @ X), 1e3 * rng.normal(size=7)))
    for i, (A, b) in enumerate(systems):
        x, rank = solve(A, b)
        out[f"s{i}_A"], out[f"s{i}_b"], out[f"s{i}_x"], out[f"s{i}_rank"] = A, b, x, rank
    # jackknife over per-SNP normal-equation contributions
    M, K, B = 600, 4, 20
    Xs = rng.normal(size=(M, K))
    y = Xs @ np.array([0.5, -1.0, 0.25, 2.0]) + rng.normal(size=M)
    terms = np.hstack([np.einsum("ji,jk->jik", Xs, Xs).reshape(M, K * K), Xs * y[:, None]])
    s, e = J._equal_count_block_boundaries(M, B)
    A_all = terms[:, :K * K].sum(0).reshape(K, K)
    b_all = terms[:, K * K:].sum(0)
    theta, _ = solve(A_all, b_all)
    reps = []
    for bb in range(B):
        keep = np.ones(M, bool)
        keep[s[bb]:e[bb]] = False
        reps.append(solve(terms[keep, :K * K].sum(0).reshape(K, K), terms[keep, K * K:].sum(0))[0])
    reps = np.asarray(reps)
    center = reps.mean(axis=0)
    se = np.sqrt((B - 1.0) / B * np.sum((reps - center) ** 2, axis=0))
    out.update({"jk_terms": terms, "jk_starts": s, "jk_ends": e, "jk_theta": theta,
                "jk_reps": reps, "jk_se": se})
    np.savez(HERE / "jackknife_golden.npz", **out)
    print("wrote", HERE / "jackknife_golden.npz")


if __name__ == "__main__":
    main()
