"""CPU: the oracle restatement (oracle/lds_oracle.cpp) against the reference's
own native code compiled unchanged (oracle/_ref) and against golden fixtures
produced by it (tests/golden/make_golden.py).  This pins the checker that the
GPU tests use."""
from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

from conftest import rel_err

GOLDEN = Path(__file__).resolve().parent / "golden"


@pytest.mark.parametrize("impute", ["mean", "hwe"])
def test_hardcall_fixture_matches_golden(oracle, impute):
    """Hard calls with missing, monomorphic and all-missing SNPs
    (reference tests/test_pgen_gwld.py:139-151)."""
    gold = np.load(GOLDEN / "hardcalls_gw.npz")
    packed = gold["packed"]
    n = 12
    annot = np.ones((packed.shape[0], 1))
    o = oracle.gw_ldscore(packed, n, annot, nvecs=64, step=3, seed=991, dist="rademacher",
                          impute=impute, impute_seed=17, with_mc=True)
    np.testing.assert_allclose(o["inv"], gold[f"{impute}_inv"], rtol=1e-13, atol=0)
    np.testing.assert_allclose(o["meansq_accum"], gold[f"{impute}_meansq"], rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(o["ldscore"], gold[f"{impute}_ldscore"], rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(o["mc_per_snp_sumsq"], gold[f"{impute}_mc"], rtol=1e-12, atol=1e-12)


@pytest.mark.parametrize("dist", ["gaussian", "spherical"])
def test_synthetic_fixture_matches_golden(oracle, dist):
    gold = np.load(GOLDEN / "synth_gw.npz")
    o = oracle.gw_ldscore(gold["packed"], 97, gold["annot"], nvecs=24, step=40, seed=31, dist=dist,
                          vtile=16, impute="mean", with_mc=True)
    assert rel_err(o["meansq_accum"], gold[f"{dist}_meansq"]) < 1e-13
    assert rel_err(o["ldscore"], gold[f"{dist}_ldscore"]) < 1e-13
    assert rel_err(o["mc_aggregate_sumsq"], gold[f"{dist}_mc_agg"]) < 1e-13


@pytest.mark.parametrize("impute", ["mean", "hwe"])
@pytest.mark.parametrize("dist", ["rademacher", "gaussian", "spherical"])
def test_oracle_matches_compiled_reference(oracle, reference, small_bed, impute, dist):
    n, m = small_bed["n"], small_bed["m"]
    rng = np.random.default_rng(1)
    annot = np.ones((m, 3))
    annot[:, 1] = rng.random(m) < 0.4
    annot[:, 2] = rng.random(m) * (rng.random(m) < 0.5)
    kw = dict(nvecs=20, step=50, seed=5, dist=dist, impute=impute, impute_seed=3, with_mc=True,
              vtile=8)
    r = reference.gw_ldscore(small_bed["prefix"], n, m, annot, **kw)
    o = oracle.gw_ldscore(small_bed["rows"], n, annot, **kw)
    assert rel_err(o["inv"], r["inv"]) < 1e-14
    assert rel_err(o["meansq_accum"], r["meansq_accum"]) < 1e-13
    assert rel_err(o["mc_per_snp_sumsq"], r["mc_per_snp_sumsq"]) < 1e-13


def test_oracle_row_selection_matches_reference(oracle, reference, small_bed):
    n, m = small_bed["n"], small_bed["m"]
    sel = np.sort(np.random.default_rng(4).choice(n, 150, replace=False)).astype(np.int64)
    annot = np.ones((m, 1))
    kw = dict(nvecs=12, step=64, seed=9, dist="rademacher", impute="hwe", impute_seed=2, rows=sel)
    r = reference.gw_ldscore(small_bed["prefix"], n, m, annot, **kw)
    o = oracle.gw_ldscore(small_bed["rows"], n, annot, **kw)
    assert rel_err(o["meansq_accum"], r["meansq_accum"]) < 1e-13


def test_reference_phase2_geno_exact_matrix(reference):
    """The compiled reference reproduces the exact matrix oracle of the
    reference's own tests/test_gwld_mc.py:44-127 (pins the harness)."""
    geno = np.asfortranarray([[0.2, -0.4, 0.8, 0.1], [1.1, 0.3, -0.2, 0.5], [-0.7, 0.9, 0.4, -0.6],
                              [0.6, -1.2, 0.7, 0.3], [0.1, 0.8, -0.5, 1.0]])
    xz = np.asfortranarray([[0.3, -0.1, 0.7, 0.2, 0.5, -0.4], [1.0, 0.6, -0.2, 0.8, -0.3, 0.9],
                            [-0.5, 0.4, 0.1, -0.7, 0.2, 0.3], [0.9, -0.8, 0.3, 0.4, 0.7, -0.1],
                            [0.2, 0.5, -0.6, 1.1, -0.9, 0.6]])
    inv = np.asarray([1.0, 0.75, 1.25, 0.6])
    bins, probes, n_denom = 2, 3, 6
    work = geno.T @ xz
    y = np.empty((4, probes, bins))
    for k in range(bins):
        y[:, :, k] = np.square(work[:, k * probes:(k + 1) * probes]) * np.square(inv[:, None]) / 25.0
    point = np.zeros((4, bins))
    agg = np.zeros(bins)
    per = np.zeros((4, bins))
    reference.phase2_geno(geno, 0, inv, probes, xz, point, n_denom, agg, per)
    np.testing.assert_allclose(point, y.sum(axis=1), rtol=2e-14, atol=2e-14)
    np.testing.assert_allclose(per, np.square(y).sum(axis=1), rtol=2e-14, atol=2e-14)
    np.testing.assert_allclose(agg, np.square(y).sum(axis=(0, 1)), rtol=2e-14, atol=2e-14)


def test_oracle_integer_products(oracle):
    from summit_b200 import bedfile

    g = bedfile.synth_genotypes(50, 7, seed=3)
    rows = bedfile.pack_bed_rows(g)
    y = np.asfortranarray(np.random.default_rng(0).integers(-127, 128, size=(50, 5), dtype=np.int8))
    out, obs = oracle.int_products(rows, 50, y)
    gv = np.where(g < 0, 0, g).astype(np.int64)
    np.testing.assert_array_equal(out, gv @ y.astype(np.int64))
    np.testing.assert_array_equal(obs, (g >= 0).astype(np.int64) @ y.astype(np.int64))
