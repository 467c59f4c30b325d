"""Exact neighbour products (lds_nn_band) against the oracle.

The integer sums must match bit for bit; the FP64 products x_j . x_{j+d} must
match the oracle's standardized genotypes (which are pinned to the reference's
genotype.cpp standardization) to FP64 rounding.
"""
from __future__ import annotations

import numpy as np
import pytest

from oracle.oracle import band_counts
from summit_b200 import bedfile

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("D", [0, 1, 8, 15])
def test_band_counts_exact(small_bed, D):
    from summit_b200.session import GwSession

    s = GwSession(small_bed["rows"], small_bed["n"])
    xx, cnt = s.nn_band(D, with_counts=True)
    want = band_counts(small_bed["geno"], D)
    assert np.array_equal(cnt.astype(np.int64), want)
    s.close()


@pytest.mark.parametrize("impute", ["mean", "hwe"])
def test_band_products_match_oracle(small_bed, oracle, impute):
    from summit_b200.session import GwSession

    D = 8
    s = GwSession(small_bed["rows"], small_bed["n"], impute_mode=impute, impute_seed=17)
    xx = s.nn_band(D)
    want = oracle.band_products(small_bed["rows"], small_bed["n"], D, impute=impute,
                                impute_seed=17)
    scale = np.abs(want[:, 0]).max()
    assert np.max(np.abs(xx - want)) <= 1e-12 * scale
    s.close()


def test_band_row_selection_and_ragged(oracle):
    """Sample subset, N not a multiple of 16 and M not a multiple of the SNP tile."""
    from summit_b200.session import GwSession

    n, m, D = 1037, 131, 8
    geno = bedfile.synth_genotypes(n, m, seed=99)
    rows = bedfile.pack_bed_rows(geno)
    sel = np.arange(3, n, 2, dtype=np.int64)
    s = GwSession(rows, n, row_sel=sel)
    xx, cnt = s.nn_band(D, with_counts=True)
    assert np.array_equal(cnt.astype(np.int64), band_counts(geno[:, sel], D))
    want = oracle.band_products(rows, n, D, rows=sel)
    assert np.max(np.abs(xx - want)) <= 1e-12 * np.abs(want[:, 0]).max()
    s.close()
