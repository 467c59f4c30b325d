"""GPU: FP64 rank-revealing solves and the SNP-block jackknife against golden
vectors written by the reference's own Python (tests/golden/jackknife_golden.npz)."""
from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
G = np.load(Path(__file__).parent / "golden" / "jackknife_golden.npz")


@pytest.mark.parametrize("i", range(4))
def test_solve_matches_reference(i):
    from summit_b200.jackknife import solve_normal_equations

    r = solve_normal_equations(G[f"s{i}_A"], G[f"s{i}_b"], require_full_rank=False)
    assert r["rank"] == int(G[f"s{i}_rank"])
    x = G[f"s{i}_x"]
    np.testing.assert_allclose(r["coefficients"], x, rtol=1e-9, atol=1e-12 * np.abs(x).max())
    lam = np.linalg.eigvalsh(0.5 * (G[f"s{i}_A"] + G[f"s{i}_A"].T))
    np.testing.assert_allclose(r["eigenvalues"], lam, rtol=1e-9, atol=1e-12 * np.abs(lam).max())


def test_solve_batch_and_errors():
    from summit_b200.jackknife import solve_normal_equations

    A = np.stack([G["s0_A"], 2.0 * G["s0_A"]])
    b = np.stack([G["s0_b"], G["s0_b"]])
    r = solve_normal_equations(A, b)
    np.testing.assert_allclose(r["coefficients"][1], 0.5 * r["coefficients"][0], rtol=1e-12)
    with pytest.raises(RuntimeError, match="not identifiable"):
        solve_normal_equations(G["s2_A"], G["s2_b"], require_full_rank=True)
    bad = G["s0_A"].copy()
    bad[0, 1] += 1.0
    with pytest.raises(RuntimeError, match="asymmetry"):
        solve_normal_equations(bad, G["s0_b"])


def test_jackknife_matches_reference():
    from summit_b200.jackknife import jackknife_normal_equations

    r = jackknife_normal_equations(G["jk_terms"], G["jk_starts"], G["jk_ends"])
    np.testing.assert_allclose(r["theta"], G["jk_theta"], rtol=1e-10)
    np.testing.assert_allclose(r["replicates"], G["jk_reps"], rtol=1e-10)
    np.testing.assert_allclose(r["se"], G["jk_se"], rtol=1e-8)
    np.testing.assert_allclose(np.sqrt(np.diag(r["cov"])), r["se"], rtol=1e-12)
