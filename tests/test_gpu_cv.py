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


@pytest.mark.parametrize("D,vtile", [(4, 12), (8, 12), (8, 0), (8, 10)])
def test_cv_near_outputs_match_oracle(small_bed, oracle, D, vtile):
    """Two probe halves [0, 12) and [12, 24): one V-tile each (vtile 12), both in
    one V-tile (vtile 0: split inside the kernels), or a tile straddling the
    split (vtile 10: tiles 10, 10, 4)."""
    from summit_b200.session import GwSession, WinPlan

    n, m, packed = small_bed["n"], small_bed["m"], small_bed["rows"]
    ws = np.array([0, 60, 200, 201, 333, 410], dtype=np.int64)
    rng = np.random.default_rng(5)
    annot = np.ones((m, 3))
    annot[:, 1] = rng.random(m) < 0.3
    annot[:, 2] = rng.random(m) < 0.5
    seed, nvecs, step = 99, 24, 50
    sess = GwSession(packed, n)
    plan = WinPlan(sess, annot, ws, nvecs, step, seed, "rademacher", vtile=vtile)
    plan.set_cv(annot, split_tiles=True, band=D)
    plan.execute()
    out = plan.cv_outputs()
    res = plan.results()
    tiles = plan.tiles()
    assert sum(tiles) == nvecs and out["meansq"].shape[0] == 2
    # the slices add up to the plain sums
    np.testing.assert_allclose(out["meansq"].sum(0), res["meansq_accum"], rtol=1e-13, atol=0)

    X = oracle.standardize(packed, n, 0, m)[0]
    inv = oracle.inv_resvar(X, 1e-10)
    win = np.repeat(np.arange(len(ws) - 1), np.diff(ws))
    assert rel_err(out["xx"], oracle.band_products(packed, n, D)) < 1e-13
    # the plan's probes, tile by tile (streams are seeded per V-tile offset)
    Z = np.hstack([_window_probes(oracle, ws, m, step, seed, int(sum(tiles[:t])), V)
                   for t, V in enumerate(tiles)])
    halves = [slice(0, 12), slice(12, 24)]
    mu = np.zeros((m, 3))
    C = np.zeros((2, m, 3))
    G = X.T @ X  # small: 410 x 410
    for j in range(m):
        nb = [i for i in range(max(0, j - D), min(m, j + D + 1)) if win[i] == win[j]]
        c = G[nb, j] * inv[j] / (n - 1)
        w = c[:, None] * annot[nb]                # (neighbours, K)
        a = Z[nb].T @ w                            # (V, K)
        for h, sl in enumerate(halves):
            C[h, j] = (a[sl] ** 2).sum(0)
        mu[j] = (w ** 2).sum(0)
    for h in range(2):
        assert rel_err(out["C"][h], C[h]) < 1e-11, f"half {h}"
    assert rel_err(out["mu"], mu) < 1e-11
    # plain sums of each half against the oracle's per-window estimator
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


def _config_like(n, m, K=24, seed=11):
    """Scaled-down config-2 inputs: Bernoulli(0.1) annotations, contiguous
    windows with log-uniform sizes in [200, 5000]."""
    from summit_b200 import gwldcore

    bed = gwldcore.synth_bed_rows(n, m, seed)
    rng = np.random.default_rng(seed)
    annot = (rng.random((m, K)) < 0.1).astype(np.float64)
    starts = [0]
    while starts[-1] < m:
        starts.append(min(m, starts[-1] + int(np.exp(rng.uniform(np.log(200.0), np.log(5000.0))))))
    return bed, annot, np.asarray(starts, dtype=np.int64)


def _snp_rrmse(est, truth):
    est, truth = np.asarray(est), np.asarray(truth)
    return float(np.mean(np.sqrt(((est - truth) ** 2).mean(0)) / np.sqrt((truth ** 2).mean(0))))


def test_learned_network_gains_over_the_estimator_without_it():
    """Judged against the exact expectation of the windowed estimator: with 10
    probes, the trained network cuts the per-SNP error of the near-field
    control variate it is added to, and beats the plain estimator with 10x the
    probes; the combine keeps each bin's mean of the near-field estimate."""
    from summit_b200.learned_cv import CvConfig, LearnedCV
    from summit_b200.session import GwSession, WinPlan

    n, m = 3000, 30000
    bed, annot, ws = _config_like(n, m)
    sess = GwSession(bed, n)
    truth = sess.partition_ld_expectation(annot, ws)
    cv = LearnedCV(sess, annot, ws, 1000, 2024, cfg=CvConfig(nvecs=10))
    res = cv.run()
    cv.close()
    learned = res["ldscore"].cpu().numpy()
    near = res["nearcv_ldscore"].cpu().numpy()
    plain10 = res["plain_ldscore"].cpu().numpy()
    p100 = WinPlan(sess, annot, ws, 100, 1000, 2024, "rademacher")
    p100.execute()
    plain100 = p100.results()["ldscore"]
    p100.close()
    sess.close()
    e_learned, e_near = _snp_rrmse(learned, truth), _snp_rrmse(near, truth)
    e_plain10, e_plain100 = _snp_rrmse(plain10, truth), _snp_rrmse(plain100, truth)
    assert e_near < 0.85 * e_plain10, (e_near, e_plain10)
    assert e_learned < 0.6 * e_near, (e_learned, e_near)
    assert e_learned < e_plain100, (e_learned, e_plain100)
    np.testing.assert_allclose(learned.mean(0), near.mean(0), rtol=1e-9, atol=1e-12)
