"""GPU: exact windowed LD scores (tcgen05 int8 Gram products, FP64 epilogue)
against the reference's own winldcore.cpp compiled unchanged and against the
oracle, including SNPs that are monomorphic or entirely missing."""
from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def refwin():
    from oracle.oracle import REF_WIN_SO, ReferenceWindowed

    if not REF_WIN_SO.exists():
        pytest.skip("reference checker oracle/_ref/libref_winld.so not built (make -C oracle ref)")
    return ReferenceWindowed()


def _bp(m, seed=3):
    rng = np.random.default_rng(seed)
    return np.cumsum(rng.integers(1, 2000, size=m)).astype(np.int64) + 10_000


@pytest.mark.parametrize("impute", ["mean", "hwe"])
@pytest.mark.parametrize("kb", [20.0, 150.0, 1e6])
def test_windowed_ld_matches_reference(small_bed, refwin, impute, kb):
    from summit_b200 import winldcore

    n, m, prefix = small_bed["n"], small_bed["m"], small_bed["prefix"]
    bp = _bp(m)
    rng = np.random.default_rng(1)
    annot = np.column_stack([np.ones(m), rng.random(m) < 0.3, rng.random(m)])
    seed = 17 if impute == "hwe" else None
    ref = refwin.compute_windowed_ld_chr(prefix, 0, m, bp, annot, kb, 64, impute_mode=impute,
                                         impute_seed=seed)
    gpu = winldcore.compute_windowed_ld_chr(prefix, prefix + ".fam", 0, m, bp, annot, kb, 64,
                                            impute_mode=impute, impute_seed=seed)
    assert gpu.shape == ref.shape and gpu.flags.f_contiguous
    assert rel_err(gpu, ref) < 1e-11


@pytest.mark.parametrize("impute", ["mean", "hwe"])
@pytest.mark.parametrize("rows_sel", [False, True])
def test_windowed_ld_with_covariates_matches_reference(small_bed, refwin, impute, rows_sel):
    """Covariates: genotypes projected by (I - C R) and restandardized per
    panel, corr_dim = N - p (winldcore.cpp:340-366, :853)."""
    from summit_b200 import winldcore

    n, prefix = small_bed["n"], small_bed["prefix"]
    rng = np.random.default_rng(21)
    rows = np.sort(rng.choice(n, 280, replace=False)) if rows_sel else None
    N = n if rows is None else rows.size
    a, b = 10, 390
    bp = _bp(b - a, seed=6)
    annot = np.column_stack([np.ones(b - a), rng.random(b - a) < 0.4])
    C = np.column_stack([np.ones(N), rng.normal(size=N), rng.normal(size=N)])
    R = np.linalg.pinv(C)
    seed = 5 if impute == "hwe" else None
    ref = refwin.compute_windowed_ld_chr(prefix, a, b, bp, annot, 120.0, 64, row_sel=rows, C=C,
                                         R=R, impute_mode=impute, impute_seed=seed)
    gpu = winldcore.compute_windowed_ld_chr(prefix, prefix + ".fam", a, b, bp, annot, 120.0, 64,
                                            row_sel=rows, C=C, R=R, impute_mode=impute,
                                            impute_seed=seed)
    assert rel_err(gpu, ref) < 1e-10
    with pytest.raises(RuntimeError, match="C/R shape mismatch"):
        winldcore.compute_windowed_ld_chr(prefix, prefix + ".fam", a, b, bp, annot, 120.0, 64,
                                          row_sel=rows, C=C[:-1], R=R[:, :-1])


def test_windowed_ld_subrange_and_row_selection(small_bed, refwin):
    from summit_b200 import winldcore

    n, prefix = small_bed["n"], small_bed["prefix"]
    rows = np.sort(np.random.default_rng(9).choice(n, 250, replace=False))
    a, b = 37, 301
    bp = _bp(b - a, seed=5)
    annot = np.ones((b - a, 2))
    annot[::4, 1] = 0.0
    ref = refwin.compute_windowed_ld_chr(prefix, a, b, bp, annot, 100.0, 50, row_sel=rows)
    gpu = winldcore.compute_windowed_ld_chr(prefix, prefix + ".fam", a, b, bp, annot, 100.0, 50,
                                            row_sel=rows)
    assert rel_err(gpu, ref) < 1e-11


@pytest.mark.parametrize("key", ["mean_narrow", "mean_wide", "hwe_narrow", "hwe_wide"])
def test_windowed_ld_hardcall_golden(tmp_path, key):
    """Monomorphic and all-missing SNPs contribute -1/(N-2) per partner, as in
    the reference (tests/golden/hardcalls_winld.npz)."""
    from summit_b200 import bedfile, winldcore

    d = np.load(Path(__file__).parent / "golden" / "hardcalls_winld.npz")
    impute, width = key.split("_")
    prefix = bedfile.write_plink(tmp_path / key, packed=d["packed"], n=12)
    gpu = winldcore.compute_windowed_ld_chr(prefix, prefix + ".fam", 0, 7, d["bp"], d["annot"],
                                            0.15 if width == "narrow" else 1000.0, 4,
                                            impute_mode=impute, impute_seed=17)
    np.testing.assert_allclose(gpu, d[key], rtol=1e-12, atol=1e-13)


def test_partition_window_ld_matches_oracle(small_bed, oracle):
    """Plain r^2 over partition windows (the stochastic estimator's expectation)
    on a resident image, including a one-SNP window and a sub-range."""
    from oracle.oracle import windowed_ld_exact
    from summit_b200.session import GwSession

    n, m, packed = small_bed["n"], small_bed["m"], small_bed["rows"]
    ws = np.array([0, 60, 200, 201, 333, 410])
    win = np.repeat(np.arange(ws.size - 1), np.diff(ws))
    lo, hi = ws[win], ws[win + 1]
    rng = np.random.default_rng(4)
    annot = np.column_stack([np.ones(m), rng.random(m) < 0.2])
    sess = GwSession(packed, n)
    gpu = sess.window_ld(lo, hi, annot)
    X = oracle.standardize(packed, n, 0, m)[0]
    ref = windowed_ld_exact(X, annot, lo, hi, restandardize=True, corr_dim=None)
    assert rel_err(gpu, ref) < 1e-11
    again = sess.window_ld(lo, hi, annot)
    np.testing.assert_array_equal(gpu, again)  # deterministic
    a, b = 130, 290
    sub = sess.window_ld(np.clip(lo[a:b], a, b), np.clip(hi[a:b], a, b), annot[a:b], row0=a, row1=b)
    ref_sub = windowed_ld_exact(X[:, a:b], annot[a:b], np.clip(lo[a:b], a, b) - a,
                                np.clip(hi[a:b], a, b) - a, restandardize=True, corr_dim=None)
    assert rel_err(sub, ref_sub) < 1e-11
    sess.close()


def test_partition_expectation_is_the_stochastic_mean(small_bed):
    """The windowed stochastic estimator with many probes approaches the exact
    expectation SNP by SNP (relative RMS error ~ sqrt(2/B))."""
    from summit_b200.session import GwSession, WinPlan

    n, m, packed = small_bed["n"], small_bed["m"], small_bed["rows"]
    ws = np.array([0, 150, 410], dtype=np.int64)
    annot = np.ones((m, 1))
    sess = GwSession(packed, n)
    truth = sess.partition_ld_expectation(annot, ws)
    B = 4096
    plan = WinPlan(sess, annot, ws, B, 100, 77, "rademacher")
    plan.execute()
    est = plan.results()["ldscore"]
    plan.close()
    sess.close()
    # sd(meansq / B) <= sqrt(2/B) E[meansq / B] and E[meansq / B] = truth + M_w/(N-1)
    sd = np.sqrt(2.0 / B) * (truth + np.diff(ws).max() / (n - 1.0))
    z = (est - truth) / sd
    assert np.sqrt(np.mean(z ** 2)) < 1.5
    assert abs(np.mean(z)) < 1.0
