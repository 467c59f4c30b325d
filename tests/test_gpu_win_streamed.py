"""GPU: the one-call windowed estimate with the upload streamed in chunks
(lds_win_ldscore) equals one windowed plan over the whole resident image bit
for bit: same window seeds (global window index), same HWE imputation draws
(global SNP index), same per-window sketch digits."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _plan_result(packed, n, annot, ws, nvecs, step, seed, dist, impute, rows=None, vtile=None):
    from summit_b200.session import GwSession, WinPlan

    sess = GwSession(packed, n, impute_mode=impute, impute_seed=6, row_sel=rows)
    plan = WinPlan(sess, annot, ws, nvecs, step, seed, dist, vtile=vtile)
    plan.execute()
    res = plan.results()
    plan.close()
    sess.close()
    return res


@pytest.mark.parametrize("chunks", [1, 2, 3, 100])
@pytest.mark.parametrize("impute,rows_sel", [("mean", False), ("hwe", True)])
def test_streamed_equals_resident_plan(small_bed, chunks, impute, rows_sel):
    from summit_b200.session import windowed_ldscore

    n, m, packed = small_bed["n"], small_bed["m"], small_bed["rows"]
    ws = np.array([0, 60, 200, 201, 333, 410], dtype=np.int64)  # includes a 1-SNP window
    assert ws[-1] == m
    rng = np.random.default_rng(12)
    annot = np.ones((m, 3))
    annot[:, 1] = rng.random(m) < 0.3
    annot[:, 2] = rng.random(m)
    rows = np.sort(rng.choice(n, n - 37, replace=False)) if rows_sel else None
    want = _plan_result(packed, n, annot, ws, 24, 50, 4242, "rademacher", impute, rows, vtile=16)
    got = windowed_ldscore(packed, n, annot, ws, 24, 50, 4242, "rademacher", vtile=16,
                           impute_mode=impute, impute_seed=6, row_sel=rows, chunks=chunks,
                           meansq=True)
    np.testing.assert_array_equal(got["ldscore"], want["ldscore"])
    np.testing.assert_array_equal(got["meansq_accum"], want["meansq_accum"])
    np.testing.assert_array_equal(got["inv"], want["inv"])


def test_streamed_many_windows_and_batches():
    """A larger image: 60 windows over 24k SNPs in 5 chunks, two V-tiles,
    Gaussian probes; ldscore only (meansq and inv not requested)."""
    from summit_b200 import gwldcore
    from summit_b200.session import windowed_ldscore

    n, m = 2048, 24_000
    packed = gwldcore.synth_bed_rows(n, m, 91)
    rng = np.random.default_rng(5)
    cuts = np.sort(rng.choice(np.arange(1, m), 59, replace=False))
    ws = np.concatenate([[0], cuts, [m]]).astype(np.int64)
    annot = (rng.random((m, 4)) < 0.4).astype(np.float64)
    annot[:, 0] = 1.0
    want = _plan_result(packed, n, annot, ws, 100, 500, 77, "gaussian", "mean", vtile=64)
    got = windowed_ldscore(packed, n, annot, ws, 100, 500, 77, "gaussian", vtile=64, chunks=5)
    np.testing.assert_array_equal(got["ldscore"], want["ldscore"])
    assert got["meansq_accum"] is None and got["inv"] is None


def test_streamed_rejects_bad_windows(small_bed):
    from summit_b200.session import windowed_ldscore

    n, m, packed = small_bed["n"], small_bed["m"], small_bed["rows"]
    annot = np.ones((m, 1))
    with pytest.raises(RuntimeError):
        windowed_ldscore(packed, n, annot, np.array([0, 100, m - 1]), 8, 50, 1)
    with pytest.raises(RuntimeError):
        windowed_ldscore(packed, n, annot, np.array([0, 100, 100, m]), 8, 50, 1)
    with pytest.raises(ValueError):
        windowed_ldscore(packed, n, annot[:-1], np.array([0, m]), 8, 50, 1)


def test_streamed_after_clearing_the_device_cache(small_bed):
    """The chunk pool is released by lds_clear_device_cache and rebuilt by the
    next call: results stay identical across calls."""
    from summit_b200 import _lib
    from summit_b200.session import windowed_ldscore

    n, m, packed = small_bed["n"], small_bed["m"], small_bed["rows"]
    ws = np.array([0, 100, 250, m], dtype=np.int64)
    annot = np.ones((m, 2))
    annot[::3, 1] = 0.0
    a = windowed_ldscore(packed, n, annot, ws, 16, 50, 5, chunks=3)["ldscore"]
    _lib.load().lds_clear_device_cache()
    b = windowed_ldscore(packed, n, annot, ws, 16, 50, 5, chunks=3)["ldscore"]
    c = windowed_ldscore(packed, n, annot, ws, 16, 50, 5, chunks=2,
                         tiling={"p1_sb_per_cta": 64})["ldscore"]
    np.testing.assert_array_equal(a, b)
    np.testing.assert_array_equal(a, c)
