"""GPU parity on the reference's own edge cases and at the workloads' shapes.

Checkers (no oracle restatement in between):
* the golden fixture tests/golden/hardcalls_gw.npz, written by the
  reference's own gwldcore.cpp (tests/golden/make_golden.py) from the hard
  calls of its tests/test_pgen_gwld.py:139-151 (missing, monomorphic and
  all-missing SNPs);
* the reference's gwldcore.cpp compiled unchanged (oracle/_ref), run with
  the same probes at N = 5,000 x M = 20,000, B = 20 Rademacher, FP64 (the
  parity configuration compared against the native CPU backend), and on one
  2,000-SNP window at N = 50,000, K = 24, B = 50 (the windowed workload's
  sample count and probe count).

Tolerances: LD-score sums (meansq_accum, non-negative sums of squares) are
held element by element to |gpu - ref| <= 1e-6 |ref| (the exact zeros of
monomorphic and all-missing SNPs must be zero on both sides up to 1e-12 of
the largest value); residual variances to 1e-13; fourth-moment sums to 1e-5.
"""
from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

from conftest import assert_rel_elementwise, dropin_gw_ldscore, rel_err

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden"
LD_RTOL = 1e-6


@pytest.fixture(scope="module")
def gw():
    from summit_b200 import gwldcore

    gwldcore.set_slices(4)
    return gwldcore


@pytest.mark.parametrize("impute", ["mean", "hwe"])
def test_hardcall_golden_through_session(gw, impute):
    gold = np.load(GOLDEN / "hardcalls_gw.npz")
    packed, n = gold["packed"], 12
    annot = np.ones((packed.shape[0], 1))
    out = gw.gw_ldscore(packed, n, annot, 64, 3, 991, rand_dist="rademacher", impute_mode=impute,
                        impute_seed=17, with_mc=True)
    np.testing.assert_allclose(out["inv"], gold[f"{impute}_inv"], rtol=1e-13, atol=0)
    assert_rel_elementwise(out["meansq_accum"], gold[f"{impute}_meansq"], LD_RTOL, "meansq")
    assert_rel_elementwise(out["mc_per_snp_sumsq"], gold[f"{impute}_mc"], 10 * LD_RTOL, "mc")
    # LD scores = meansq / B - M_k / (N - 1): compare on the meansq scale.
    np.testing.assert_allclose(out["ldscore"], gold[f"{impute}_ldscore"], rtol=0,
                               atol=LD_RTOL * np.max(np.abs(gold[f"{impute}_meansq"])) / 64)


@pytest.mark.parametrize("impute", ["mean", "hwe"])
def test_hardcall_golden_through_dropin(gw, tmp_path, impute):
    from summit_b200 import bedfile

    gold = np.load(GOLDEN / "hardcalls_gw.npz")
    packed, n = gold["packed"], 12
    m = packed.shape[0]
    prefix = bedfile.write_plink(tmp_path / f"hc_{impute}", packed=packed, n=n)
    annot = np.ones((m, 1))
    ours = dropin_gw_ldscore(gw, prefix, n, m, annot, 64, 3, 991, "rademacher", impute,
                             np.float64, 64, impute_seed=17)
    np.testing.assert_allclose(ours["inv"], gold[f"{impute}_inv"], rtol=1e-13, atol=0)
    assert_rel_elementwise(ours["meansq"], gold[f"{impute}_meansq"], LD_RTOL, "meansq")
    assert_rel_elementwise(ours["mc_snp"], gold[f"{impute}_mc"], 10 * LD_RTOL, "mc")


@pytest.fixture(scope="module")
def config1(tmp_path_factory, gw):
    """N = 5,000 x M = 20,000 synthetic fileset (1 % MCAR missing)."""
    from summit_b200 import bedfile

    n, m = 5000, 20000
    rows = gw.synth_bed_rows(n, m, seed=1)
    prefix = bedfile.write_plink(tmp_path_factory.mktemp("cfg1") / "cfg1", packed=rows, n=n)
    return {"n": n, "m": m, "rows": rows, "prefix": prefix}


@pytest.mark.parametrize("impute", ["mean", "hwe"])
def test_config1_full_shape_session_matches_reference(gw, reference, config1, impute):
    n, m = config1["n"], config1["m"]
    annot = np.ones((m, 1))
    kw = dict(impute_seed=3)
    ref = reference.gw_ldscore(config1["prefix"], n, m, annot, 20, 1000, 2024, dist="rademacher",
                               vtile=20, impute=impute, with_mc=True, **kw)
    out = gw.gw_ldscore(config1["rows"], n, annot, 20, 1000, 2024, rand_dist="rademacher",
                        vtile=20, impute_mode=impute, with_mc=True, **kw)
    assert rel_err(out["inv"], ref["inv"]) < 1e-13
    assert_rel_elementwise(out["meansq_accum"], ref["meansq_accum"], LD_RTOL, "meansq_accum")
    assert_rel_elementwise(out["mc_per_snp_sumsq"], ref["mc_per_snp_sumsq"], 10 * LD_RTOL, "mc")


def test_config1_full_shape_dropin_matches_reference(gw, reference, config1):
    n, m, prefix = config1["n"], config1["m"], config1["prefix"]
    annot = np.ones((m, 1))
    ref = reference.gw_ldscore(prefix, n, m, annot, 20, 1000, 2024, dist="rademacher", vtile=20,
                               impute="mean", impute_seed=4, with_mc=True)
    ours = dropin_gw_ldscore(gw, prefix, n, m, annot, 20, 1000, 2024, "rademacher", "mean",
                             np.float64, 20)
    assert rel_err(ours["inv"], ref["inv"]) < 1e-13
    assert_rel_elementwise(ours["meansq"], ref["meansq_accum"], LD_RTOL, "meansq_accum")
    assert_rel_elementwise(ours["mc_snp"], ref["mc_per_snp_sumsq"], 10 * LD_RTOL, "mc")


def test_window_at_workload_shape_matches_reference(gw, reference, tmp_path):
    """One 2,000-SNP window of the windowed workload's shape (N = 50,000, 24
    Bernoulli(0.1) annotation bins, B = 50 Rademacher probes, 1,000-SNP
    blocks) through the windowed plan, against the reference's genome-wide
    estimator on the window's SNPs with the window's probe root."""
    from summit_b200 import bedfile
    from summit_b200.session import GwSession, WinPlan, window_seed

    n, m, K, B = 50_000, 2_000, 24, 50
    rows = gw.synth_bed_rows(n, m, seed=77)
    rng = np.random.default_rng(5)
    annot = (rng.random((m, K)) < 0.1).astype(np.float64)
    annot[:, 0] = 1.0
    seed = 31
    sess = GwSession(rows, n)
    plan = WinPlan(sess, annot, np.array([0, m], dtype=np.int64), B, 1000, seed, "rademacher")
    plan.execute()
    res = plan.results()
    plan.close()
    sess.close()
    prefix = bedfile.write_plink(tmp_path / "win", packed=rows, n=n)
    ref = reference.gw_ldscore(prefix, n, m, annot, B, 1000, window_seed(seed, 0),
                               dist="rademacher", vtile=B, impute="mean")
    assert_rel_elementwise(res["meansq_accum"], ref["meansq_accum"], LD_RTOL, "meansq_accum")


def test_bad_bed_magic_is_rejected(gw, tmp_path):
    """genotype.cpp:384-389: anything but 6C 1B 01 (SNP-major) is refused with
    the reference's message."""
    from summit_b200 import bedfile

    geno = bedfile.synth_genotypes(40, 10, seed=3)
    prefix = bedfile.write_plink(tmp_path / "bad", geno)
    raw = bytearray(Path(prefix + ".bed").read_bytes())
    raw[2] = 0x00  # individual-major mode
    Path(prefix + ".bed").write_bytes(bytes(raw))
    ms = np.zeros((10, 1))
    with pytest.raises(RuntimeError, match="Invalid BED magic/mode"):
        gw.phase2_accum_XtXz_bed(bed_prefix=prefix, fam_path=prefix + ".fam", blk_start=0,
                                 blk_end=10, ddof=1, inv_left=np.ones(10), tile_nvecs=4,
                                 Xz2d=np.zeros((40, 4), order="F"), meansq_accum=ms, N_denom=40,
                                 impute_mode="mean")
    from summit_b200 import winldcore

    with pytest.raises(RuntimeError, match="Invalid BED magic/mode"):
        winldcore.compute_maf_bed(prefix, prefix + ".fam", 10, 5)


def test_rewritten_file_invalidates_the_device_cache(gw, tmp_path):
    """The device image is cached by file identity (dev, inode, size, mtime,
    ctime; genotype.cpp:50-97): a fileset rewritten in place with new
    genotypes must not be served from the cache."""
    import os
    import time

    from summit_b200 import bedfile

    n, m = 300, 64
    prefix = str(tmp_path / "rw")
    rng = np.random.default_rng(1)
    inv = np.ones(m)
    Xz = np.asfortranarray(rng.standard_normal((n, 8)))

    def phase2(p):
        ms = np.zeros((m, 1))
        gw.phase2_accum_XtXz_bed(bed_prefix=p, fam_path=p + ".fam", blk_start=0, blk_end=m,
                                 ddof=1, inv_left=inv, tile_nvecs=8, Xz2d=Xz, meansq_accum=ms,
                                 N_denom=n, impute_mode="mean")
        return ms

    bedfile.write_plink(prefix, bedfile.synth_genotypes(n, m, seed=11))
    first = phase2(prefix)
    again = phase2(prefix)
    np.testing.assert_array_equal(first, again)
    time.sleep(0.01)
    bedfile.write_plink(prefix, bedfile.synth_genotypes(n, m, seed=12))
    os.utime(prefix + ".bed")
    rewritten = phase2(prefix)
    fresh_prefix = bedfile.write_plink(tmp_path / "fresh", bedfile.synth_genotypes(n, m, seed=12))
    np.testing.assert_array_equal(rewritten, phase2(fresh_prefix))
    assert not np.array_equal(rewritten, first)
