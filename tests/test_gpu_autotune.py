"""GPU: the autotuner times real tilings of a windowed plan, every candidate
gives the same LD scores bit for bit, and a plan built from the tuned record
reproduces the default plan's scores."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_tune_and_tuned_plan(tmp_path):
    from summit_b200 import autotune, gwldcore
    from summit_b200.session import GwSession, WinPlan

    n, m = 2048, 20_000
    packed = gwldcore.synth_bed_rows(n, m, 17)
    rng = np.random.default_rng(2)
    cuts = np.sort(rng.choice(np.arange(1, m), 30, replace=False))
    ws = np.concatenate([[0], cuts, [m]]).astype(np.int64)
    annot = (rng.random((m, 5)) < 0.3).astype(np.float64)
    annot[:, 0] = 1.0
    sess = GwSession(packed, n)
    cache = autotune.TuneCache(tmp_path / "tune.json")
    cands = [{"p1_sb_per_cta": 4, "batch_gb": 8.0},
             {"p1_sb_per_cta": 16, "batch_gb": 0.05}]
    rec = autotune.tune_windowed(sess, annot, ws, 50, 1000, 3, candidates=cands, cache=cache)
    assert rec["config"] in cands and rec["ms"] > 0 and len(rec["trials"]) == 2
    plan = autotune.tuned_win_plan(sess, annot, ws, 50, 1000, 3, cache=cache,
                                   tune_if_missing=False)
    plan.execute()
    got = plan.results()["ldscore"]
    plan.close()
    ref = WinPlan(sess, annot, ws, 50, 1000, 3)
    ref.execute()
    want = ref.results()["ldscore"]
    ref.close()
    sess.close()
    np.testing.assert_array_equal(got, want)


def test_phase2_bins_per_cta_do_not_change_scores():
    """Bins per phase-2 CTA (one bin, the grouped default, all bins, and a
    count that leaves the tile's last CTA with fewer bins and MMA groups) give
    the same scores bit for bit, in work order and in grid order."""
    from summit_b200 import gwldcore
    from summit_b200.session import GwSession, WinPlan

    n, m, k = 1536, 9_000, 7
    packed = gwldcore.synth_bed_rows(n, m, 23)
    rng = np.random.default_rng(5)
    cuts = np.sort(rng.choice(np.arange(1, m), 12, replace=False))
    ws = np.concatenate([[0], cuts, [m]]).astype(np.int64)
    annot = (rng.random((m, k)) < 0.4).astype(np.float64)
    annot[:, 0] = 1.0
    sess = GwSession(packed, n)
    got = {}
    for nb, chunk in ((1, 4), (0, 4), (k, 2), (3, 0), (5, 1)):
        plan = WinPlan(sess, annot, ws, 50, 1000, 9)
        plan.set_p2_bins(nb)
        plan.set_p2_order(chunk)
        plan.execute()
        got[(nb, chunk)] = plan.results()["ldscore"]
        plan.close()
    sess.close()
    base = got[(1, 4)]
    assert np.all(np.isfinite(base)) and np.any(base != 0)
    for key, val in got.items():
        np.testing.assert_array_equal(val, base, err_msg=str(key))
