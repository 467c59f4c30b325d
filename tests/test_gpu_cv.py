"""GPU: near-field control-variate outputs of a windowed plan against the oracle.

The oracle recomputes, in FP64 from its standardized genotypes and its own
probe streams, the near-field sums C (per V-tile) and their known means mu:
  c_ji = (x_j . x_i) inv_j / (N - ddof),  a_jkv = sum_{|i-j|<=D, same window} c_ji annot_ik z_iv.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu


def _window_probes(oracle, ws, m, step, seed, v0, V):
    from summit_b200.session import window_seed

    Z = np.zeros((m, V))
    for w in range(len(ws) - 1):
        a, b = int(ws[w]), int(ws[w + 1])
        for s in range(0, b - a, step):
            L = min(step, b - a - s)
            Z[a + s: a + s + L] = oracle.probes(window_seed(seed, w), s, v0, L, V)
    return Z


@pytest.mark.parametrize("D", [4, 8])
def test_cv_near_outputs_match_oracle(small_bed, oracle, D):
    from summit_b200.session import GwSession, WinPlan

    n, m, packed = small_bed["n"], small_bed["m"], small_bed["rows"]
    ws = np.array([0, 60, 200, 201, 333, 410], dtype=np.int64)
    rng = np.random.default_rng(5)
    annot = np.ones((m, 3))
    annot[:, 1] = rng.random(m) < 0.3
    annot[:, 2] = rng.random(m) < 0.5
    seed, nvecs, step = 99, 24, 50
    sess = GwSession(packed, n)
    plan = WinPlan(sess, annot, ws, nvecs, step, seed, "rademacher", vtile=12)
    plan.set_cv(annot, split_tiles=True, band=D)
    plan.execute()
    out = plan.cv_outputs()
    res = plan.results()
    tiles = plan.tiles()
    assert tiles == [12, 12]
    # the slices add up to the plain sums
    np.testing.assert_allclose(out["meansq"].sum(0), res["meansq_accum"], rtol=1e-13, atol=0)

    X = oracle.standardize(packed, n, 0, m)[0]
    inv = oracle.inv_resvar(X, 1e-10)
    win = np.repeat(np.arange(len(ws) - 1), np.diff(ws))
    assert rel_err(out["xx"], oracle.band_products(packed, n, D)) < 1e-13
    mu = np.zeros((m, 3))
    v0 = 0
    for t, V in enumerate(tiles):
        Z = _window_probes(oracle, ws, m, step, seed, v0, V)
        C = np.zeros((m, 3))
        for j in range(m):
            nb = [i for i in range(max(0, j - D), min(m, j + D + 1)) if win[i] == win[j]]
            c = (X[:, nb].T @ X[:, j]) * inv[j] / (n - 1)
            w = c[:, None] * annot[nb]                # (neighbours, K)
            a = Z[nb].T @ w                            # (V, K)
            C[j] = (a ** 2).sum(0)
            if t == 0:
                mu[j] = (w ** 2).sum(0)
        assert rel_err(out["C"][t], C) < 1e-11, f"tile {t}"
        v0 += V
    assert rel_err(out["mu"], mu) < 1e-11
    plan.close()
    sess.close()


def test_cv_plan_results_unchanged(small_bed):
    """Adding the control-variate outputs leaves the plain LD scores as they were."""
    from summit_b200.session import GwSession, WinPlan

    n, m, packed = small_bed["n"], small_bed["m"], small_bed["rows"]
    ws = np.array([0, 150, 410], dtype=np.int64)
    annot = np.ones((m, 2))
    annot[::3, 1] = 0
    sess = GwSession(packed, n)
    a = WinPlan(sess, annot, ws, 20, 40, 3, "rademacher", vtile=10)
    b = WinPlan(sess, annot, ws, 20, 40, 3, "rademacher", vtile=10)
    b.set_cv(annot, split_tiles=True, band=8)
    a.execute()
    b.execute()
    np.testing.assert_array_equal(a.results()["ldscore"], b.results()["ldscore"])
    assert b.cv_ms() >= 0.0
