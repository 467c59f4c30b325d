"""CPU: the oracle's exact windowed LD scores against the reference's own
winldcore.cpp compiled unchanged (oracle/_ref/libref_winld.so)."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import rel_err


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
@pytest.mark.parametrize("kb,chunk", [(50.0, 64), (200.0, 100), (1e6, 1000)])
def test_oracle_windowed_matches_reference(oracle, refwin, small_bed, impute, kb, chunk):
    from oracle.oracle import bp_window_bounds, windowed_ld_exact

    n, m = small_bed["n"], small_bed["m"]
    bp = _bp(m)
    rng = np.random.default_rng(1)
    annot = np.column_stack([np.ones(m), rng.random(m) < 0.3, rng.random(m)])
    seed = 17 if impute == "hwe" else None
    ref = refwin.compute_windowed_ld_chr(small_bed["prefix"], 0, m, bp, annot, kb, chunk,
                                         impute_mode=impute, impute_seed=seed)
    X = oracle.standardize(small_bed["rows"], n, 0, m, None, 0, impute, seed or 0)[0]
    lo, hi = bp_window_bounds(bp, kb)
    ours = windowed_ld_exact(X, annot, lo, hi, restandardize=(impute == "mean"), corr_dim=n - 1)
    assert rel_err(ours, ref) < 1e-12


def test_oracle_windowed_row_selection_and_subrange(oracle, refwin, small_bed):
    """A chromosome slice [chr_start, chr_end) and a sample subset."""
    from oracle.oracle import bp_window_bounds, windowed_ld_exact

    n, m = small_bed["n"], small_bed["m"]
    rows = np.sort(np.random.default_rng(9).choice(n, 250, replace=False))
    a, b = 37, 301
    bp = _bp(b - a, seed=5)
    annot = np.ones((b - a, 2))
    annot[::4, 1] = 0.0
    ref = refwin.compute_windowed_ld_chr(small_bed["prefix"], a, b, bp, annot, 100.0, 50,
                                         row_sel=rows)
    X = oracle.standardize(small_bed["rows"], n, a, b, rows, 0, "mean", 0)[0]
    lo, hi = bp_window_bounds(bp, 100.0)
    ours = windowed_ld_exact(X, annot, lo, hi, restandardize=True, corr_dim=rows.size - 1)
    assert rel_err(ours, ref) < 1e-12


def test_reference_windowed_rejects_unsorted_positions(refwin, small_bed):
    bp = _bp(small_bed["m"])[::-1].copy()
    with pytest.raises(RuntimeError, match="BP not sorted"):
        refwin.compute_windowed_ld_chr(small_bed["prefix"], 0, small_bed["m"], bp,
                                       np.ones((small_bed["m"], 1)), 100.0, 64)


@pytest.mark.parametrize("key", ["mean_narrow", "mean_wide", "hwe_narrow", "hwe_wide"])
def test_oracle_windowed_matches_golden_hardcalls(oracle, key):
    """Hard calls with missing, monomorphic and all-missing SNPs
    (tests/golden/hardcalls_winld.npz, written by the reference's winldcore)."""
    from pathlib import Path

    from oracle.oracle import bp_window_bounds, windowed_ld_exact

    d = np.load(Path(__file__).parent / "golden" / "hardcalls_winld.npz")
    impute, width = key.split("_")
    packed, annot, bp = d["packed"], d["annot"], d["bp"]
    m, n = packed.shape[0], 12
    X = oracle.standardize(packed, n, 0, m, None, 0, impute, 17)[0]
    lo, hi = bp_window_bounds(bp, 0.15 if width == "narrow" else 1000.0)
    ours = windowed_ld_exact(X, annot, lo, hi, restandardize=(impute == "mean"), corr_dim=n - 1)
    np.testing.assert_allclose(ours, d[key], rtol=1e-12, atol=1e-13)


def test_dropin_windowed_argument_checks_match_reference():
    """Argument errors of the GPU drop-in are raised before any device work,
    with the reference's messages (winldcore.cpp:798-852)."""
    from summit_b200 import winldcore

    ones = np.ones((3, 1))
    bp = np.array([1, 2, 3], dtype=np.int64)
    with pytest.raises(RuntimeError, match="chr_end must be >= chr_start"):
        winldcore.compute_windowed_ld_chr("x", "x.fam", 3, 0, bp, ones, 1.0, 10)
    with pytest.raises(RuntimeError, match="Chromosome slice is empty"):
        winldcore.compute_windowed_ld_chr("x", "x.fam", 2, 2, bp[:0], ones[:0], 1.0, 10)
    with pytest.raises(RuntimeError, match="chunk_size must be > 0"):
        winldcore.compute_windowed_ld_chr("x", "x.fam", 0, 3, bp, ones, 1.0, 0)
    with pytest.raises(RuntimeError, match="finite positive BP window"):
        winldcore.compute_windowed_ld_chr("x", "x.fam", 0, 3, bp, ones, -1.0, 10)
    with pytest.raises(RuntimeError, match="BP not sorted"):
        winldcore.compute_windowed_ld_chr("x", "x.fam", 0, 3, bp[::-1].copy(), ones, 1.0, 10)
    with pytest.raises(RuntimeError, match="bp length mismatch"):
        winldcore.compute_windowed_ld_chr("x", "x.fam", 0, 3, bp[:2], ones, 1.0, 10)
    with pytest.raises(RuntimeError, match="C/R shape mismatch"):
        winldcore.compute_windowed_ld_chr("x", "x.fam", 0, 3, bp, ones, 1.0, 10,
                                          row_sel=np.arange(4), C=np.ones((5, 1)),
                                          R=np.ones((1, 5)))
    with pytest.raises(RuntimeError, match="impute_mode"):
        winldcore.compute_windowed_ld_chr("x", "x.fam", 0, 3, bp, ones, 1.0, 10,
                                          impute_mode="median")
