"""GPU: windowed + partitioned stochastic LD scores.

Window w's estimate is the genome-wide estimator on the window's SNPs with
probe root window_seed(seed, w), so each window is checked against the
reference's own compiled code run on that window's sub-fileset."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu


def _sub_fileset(tmp_path, packed, n, a, b, name):
    from summit_b200 import bedfile

    return bedfile.write_plink(tmp_path / name, packed=packed[a:b], n=n)


@pytest.mark.parametrize("impute", ["mean", "hwe"])
def test_windows_match_reference_per_window(tmp_path, small_bed, reference, oracle, impute):
    from summit_b200.session import GwSession, WinPlan, window_seed

    n, m, packed = small_bed["n"], small_bed["m"], small_bed["rows"]
    ws = np.array([0, 60, 200, 201, 333, 410], dtype=np.int64)  # includes a 1-SNP window
    rng = np.random.default_rng(12)
    annot = np.ones((m, 2))
    annot[:, 1] = rng.random(m) < 0.3
    seed, nvecs, step = 4242, 24, 50
    sess = GwSession(packed, n, impute_mode=impute, impute_seed=6)
    plan = WinPlan(sess, annot, ws, nvecs, step, seed, "rademacher", vtile=16, with_mc=True)
    plan.execute()            # graph capture + launch
    first = plan.results()
    plan.execute()            # graph launch
    res = plan.results()
    np.testing.assert_array_equal(first["ldscore"], res["ldscore"])
    for w in range(len(ws) - 1):
        a, b = int(ws[w]), int(ws[w + 1])
        pre = _sub_fileset(tmp_path, packed, n, a, b, f"w{impute}{w}")
        kw = dict(nvecs=nvecs, step=step, seed=window_seed(seed, w), dist="rademacher", vtile=16,
                  impute=impute, impute_seed=6, with_mc=True)
        if impute == "mean":
            ref = reference.gw_ldscore(pre, n, b - a, annot[a:b], **kw)
        else:
            # HWE draws are seeded by the SNP's index in the fileset, which a
            # sub-fileset would renumber: use the oracle on the full image.
            ref = oracle.gw_ldscore(packed, n, annot[a:b], snp0=a, **kw)
        assert rel_err(res["ldscore"][a:b], ref["ldscore"]) < 1e-6, f"window {w}"
        assert rel_err(res["meansq_accum"][a:b], ref["meansq_accum"]) < 1e-6, f"window {w}"
    plan.close()
    sess.close()


def test_windowed_batches_agree(small_bed):
    """Splitting the windows into several batches does not change the result."""
    from summit_b200.session import GwSession, WinPlan

    n, m, packed = small_bed["n"], small_bed["m"], small_bed["rows"]
    ws = np.array([0, 100, 180, 300, 410], dtype=np.int64)
    annot = np.ones((m, 3))
    annot[::4, 2] = 0
    sess = GwSession(packed, n)
    one = WinPlan(sess, annot, ws, 16, 64, 7, "gaussian", batch_gb=100.0)
    many = WinPlan(sess, annot, ws, 16, 64, 7, "gaussian", batch_gb=1e-6)  # one window per batch
    one.execute()
    many.execute()
    a, b = one.results(), many.results()
    np.testing.assert_allclose(a["ldscore"], b["ldscore"], rtol=1e-13, atol=1e-13)
