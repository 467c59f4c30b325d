"""GPU parity tests for the genome-wide LD-score path (liblds.so through its C ABI).

The checker is the oracle (our FP64 restatement, itself pinned to the
reference's compiled code in test_oracle_pins.py) and, for the drop-in
per-block functions, the reference's own compiled gwldcore.cpp.

Tolerances: integer products are compared bit for bit.  LD scores carry the
representation error of 4 int8 digits of the floating operands (28 bits), far
below the 1e-6 relative bound asserted here.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import (assert_rel_elementwise, dropin_gw_ldscore, max_rel_elementwise,
                      rel_err)

pytestmark = pytest.mark.gpu

LD_RTOL = 1e-6


@pytest.fixture(scope="module")
def gw():
    from summit_b200 import gwldcore

    gwldcore.set_slices(4)
    return gwldcore


def test_tensor_core_products_are_exact(gw, oracle):
    from summit_b200 import bedfile

    rng = np.random.default_rng(5)
    n, L, Q = 1000, 300, 37  # none of them a tile multiple
    geno = bedfile.synth_genotypes(n, L, seed=99)
    rows = bedfile.pack_bed_rows(geno)
    y = np.asfortranarray(rng.integers(-127, 128, size=(n, Q), dtype=np.int8))
    g_gpu, o_gpu = gw.debug_xt_products(rows, n, y)
    g_ref, o_ref = oracle.int_products(rows, n, y)
    np.testing.assert_array_equal(g_gpu, g_ref)
    np.testing.assert_array_equal(o_gpu, o_ref)


def test_tcgen05_products_are_exact(gw, oracle):
    """The tcgen05 phase-2 kernel's integer core: per-digit int8 products
    accumulated in TMEM, recombined exactly (Horner in int64)."""
    from summit_b200 import bedfile

    rng = np.random.default_rng(6)
    n, L, V = 1000, 300, 50  # 200 digit columns -> N = 208 per MMA
    geno = bedfile.synth_genotypes(n, L, seed=98)
    rows = bedfile.pack_bed_rows(geno)
    y4 = np.asfortranarray(rng.integers(-127, 128, size=(n, 4 * V), dtype=np.int8))
    g_gpu, o_gpu = gw.debug_xt_products_umma(rows, n, y4)
    g_ref, o_ref = oracle.int_products(rows, n, y4)
    horner = lambda a: ((a[:, 0::4] * 128 + a[:, 1::4]) * 128 + a[:, 2::4]) * 128 + a[:, 3::4]
    np.testing.assert_array_equal(g_gpu, horner(g_ref))
    np.testing.assert_array_equal(o_gpu, horner(o_ref))


@pytest.mark.parametrize("V", [8, 50, 64, 100])
def test_tcgen05_and_mma_sync_paths_agree(gw, oracle, small_bed, V):
    n, m, rows = small_bed["n"], small_bed["m"], small_bed["rows"]
    annot = np.ones((m, 2))
    annot[::2, 1] = 0
    out = {}
    for impl in ("tcgen05", "mma"):
        gw.set_p2_kernel(impl)
        out[impl] = gw.gw_ldscore(rows, n, annot, V, 128, 21, vtile=V, with_mc=True)
    gw.set_p2_kernel("tcgen05")
    ora = oracle.gw_ldscore(rows, n, annot, V, 128, 21, vtile=V, with_mc=True)
    assert rel_err(out["tcgen05"]["meansq_accum"], out["mma"]["meansq_accum"]) < 1e-12
    assert rel_err(out["tcgen05"]["ldscore"], ora["ldscore"]) < LD_RTOL


def test_device_synthetic_generator_matches_numpy(gw):
    from summit_b200 import bedfile

    n, m = 517, 64
    dev = gw.synth_bed_rows(n, m, seed=31337)
    host = bedfile.pack_bed_rows(bedfile.synth_genotypes(n, m, seed=31337))
    np.testing.assert_array_equal(dev, host)


@pytest.mark.parametrize("impute", ["mean", "hwe"])
@pytest.mark.parametrize("dist", ["rademacher", "gaussian", "spherical"])
def test_session_matches_oracle(gw, oracle, small_bed, impute, dist):
    n, m, rows = small_bed["n"], small_bed["m"], small_bed["rows"]
    rng = np.random.default_rng(3)
    annot = np.ones((m, 3))
    annot[:, 1] = rng.random(m) < 0.3
    annot[:, 2] = rng.random(m) * (rng.random(m) < 0.5)  # continuous, some zeros
    kw = dict(nvecs=40, seed=11, vtile=16, impute_seed=5)
    gpu = gw.gw_ldscore(rows, n, annot, step_size=97, rand_dist=dist, impute_mode=impute,
                        with_mc=True, **kw)
    ora = oracle.gw_ldscore(rows, n, annot, step=97, dist=dist, impute=impute, with_mc=True, **kw)
    # Residual variances are summed from code counts instead of sample by
    # sample, so they agree to rounding (the sequential FP64 sum's order).
    assert rel_err(gpu["inv"], ora["inv"]) < 1e-13
    assert_rel_elementwise(gpu["meansq_accum"], ora["meansq_accum"], LD_RTOL, "meansq_accum")
    assert rel_err(gpu["ldscore"], ora["ldscore"]) < LD_RTOL
    assert rel_err(gpu["mc_per_snp_sumsq"], ora["mc_per_snp_sumsq"]) < 10 * LD_RTOL
    assert rel_err(gpu["mc_aggregate_sumsq"], ora["mc_aggregate_sumsq"]) < 10 * LD_RTOL


def test_session_float_path_inputs(gw, oracle, small_bed):
    n, m, rows = small_bed["n"], small_bed["m"], small_bed["rows"]
    annot = np.ones((m, 1))
    gpu = gw.gw_ldscore(rows, n, annot, 30, 64, 17, rand_dist="gaussian", dtype=np.float32)
    ora = oracle.gw_ldscore(rows, n, annot, 30, 64, 17, dist="gaussian", as_float=True)
    assert rel_err(gpu["ldscore"], ora["ldscore"]) < LD_RTOL


def test_session_row_selection(gw, oracle, small_bed):
    n, m, rows = small_bed["n"], small_bed["m"], small_bed["rows"]
    sel = np.sort(np.random.default_rng(8).choice(n, size=201, replace=False)).astype(np.int64)
    annot = np.ones((m, 1))
    gpu = gw.gw_ldscore(rows, n, annot, 20, 50, 3, row_sel=sel, impute_mode="hwe", impute_seed=9)
    ora = oracle.gw_ldscore(rows, n, annot, 20, 50, 3, rows=sel, impute="hwe", impute_seed=9)
    assert rel_err(gpu["ldscore"], ora["ldscore"]) < LD_RTOL


def test_session_is_deterministic(gw, small_bed):
    n, m, rows = small_bed["n"], small_bed["m"], small_bed["rows"]
    annot = np.ones((m, 2))
    a = gw.gw_ldscore(rows, n, annot, 25, 64, 1, with_mc=True)
    b = gw.gw_ldscore(rows, n, annot, 25, 64, 1)
    np.testing.assert_array_equal(a["ldscore"], b["ldscore"])


@pytest.mark.parametrize("impute", ["mean", "hwe"])
def test_dropin_blockwise_matches_reference(gw, reference, small_bed, impute):
    """The per-block drop-in functions against the reference's own compiled
    gwldcore.cpp, both driven by the reference driver's call sequence."""
    prefix, n, m = small_bed["prefix"], small_bed["n"], small_bed["m"]
    annot = np.ones((m, 2))
    annot[1::2, 1] = 0
    ours = dropin_gw_ldscore(gw, prefix, n, m, annot, 24, 100, 77, "rademacher", impute, np.float64, 16)
    ref = reference.gw_ldscore(prefix, n, m, annot, 24, 100, 77, dist="rademacher", vtile=16,
                               impute=impute, impute_seed=4, with_mc=True)
    assert rel_err(ours["inv"], ref["inv"]) < 1e-13
    assert_rel_elementwise(ours["meansq"], ref["meansq_accum"], LD_RTOL, "meansq_accum")
    assert_rel_elementwise(ours["mc_snp"], ref["mc_per_snp_sumsq"], 10 * LD_RTOL, "mc_per_snp")


def test_dropin_float32_overload(gw, reference, oracle, small_bed):
    """float32 arrays through the drop-in per-block entries.

    The float32 path draws float probes, stores the sketch and the sums in
    float32, and computes in exact integer digits.  Its FP64-arithmetic
    counterpart on the same float inputs is the oracle with float inputs;
    against it our float32 result is held to 1e-6 per element, and it must be
    at least as close as the reference's own float32 run (float32 BLAS)."""
    prefix, n, m, rows = small_bed["prefix"], small_bed["n"], small_bed["m"], small_bed["rows"]
    annot = np.ones((m, 1))
    ours = dropin_gw_ldscore(gw, prefix, n, m, annot, 16, 128, 5, "spherical", "mean", np.float32,
                             16)
    ref32 = reference.gw_ldscore(prefix, n, m, annot, 16, 128, 5, dist="spherical", vtile=16,
                                 dtype=np.float32)
    exact = oracle.gw_ldscore(rows, n, annot, 16, 128, 5, dist="spherical", vtile=16,
                              as_float=True)
    assert ours["meansq"].dtype == np.float32
    assert_rel_elementwise(ours["meansq"], exact["meansq_accum"], LD_RTOL, "float32 meansq")
    err_ours = max_rel_elementwise(ours["meansq"], exact["meansq_accum"])
    err_ref = max_rel_elementwise(ref32["meansq_accum"], exact["meansq_accum"])
    assert err_ours <= max(err_ref, 1e-7), (err_ours, err_ref)


@pytest.mark.parametrize("n,m", [(333, 410), (1000, 2600)])
def test_synthetic_image_equals_uploaded_rows(gw, n, m):
    """The image generated on the device equals the one uploaded from the same
    generator's host rows: identical statistics and identical estimates."""
    from summit_b200.session import GwSession

    rows = gw.synth_bed_rows(n, m, 77)
    a, b = GwSession(rows, n), GwSession.synthetic(n, m, 77)
    sa, sb = a.stats(), b.stats()
    np.testing.assert_array_equal(sa["mean"], sb["mean"])
    np.testing.assert_array_equal(sa["sdinv"], sb["sdinv"])
    annot = np.ones((m, 2))
    annot[::3, 1] = 0
    ra = a.plan(annot, 20, 250, 5)
    rb = b.plan(annot, 20, 250, 5)
    ra.execute()
    rb.execute()
    np.testing.assert_array_equal(ra.results()["ldscore"], rb.results()["ldscore"])
    for x in (ra, rb, a, b):
        x.close()


@pytest.mark.parametrize("impute", ["mean", "hwe"])
def test_tiles_without_missing_calls_skip_the_o_plane(gw, oracle, impute):
    """Phase 2 skips the observed-count products of 128-SNP tiles whose SNPs
    have no missing call (their O^T y equals the sketch digits' column sums).
    An image mixing complete and incomplete tiles, in the genome-wide session
    and the windowed plan, against the oracle (HWE-completed images have no
    missing call at all: every tile skips)."""
    from summit_b200 import bedfile
    from summit_b200.session import GwSession, WinPlan, window_seed

    n, m = 300, 700
    geno = bedfile.synth_genotypes(n, m, seed=606)
    full = bedfile.synth_genotypes(n, m, seed=606, missing=False)
    geno[:256] = full[:256]        # two complete tiles, then tiles with missing calls
    geno[400:520] = full[400:520]  # a complete run that straddles tile boundaries
    rows = bedfile.pack_bed_rows(geno)
    annot = np.ones((m, 2))
    annot[::3, 1] = 0.0
    kw = dict(nvecs=24, seed=5, vtile=24, impute_seed=3)
    got = gw.gw_ldscore(rows, n, annot, step_size=100, impute_mode=impute, with_mc=True, **kw)
    want = oracle.gw_ldscore(rows, n, annot, step=100, impute=impute, with_mc=True, **kw)
    assert_rel_elementwise(got["meansq_accum"], want["meansq_accum"], LD_RTOL, "session")
    assert rel_err(got["mc_per_snp_sumsq"], want["mc_per_snp_sumsq"]) < 10 * LD_RTOL
    ws = np.array([0, 130, 460, 700], dtype=np.int64)
    sess = GwSession(rows, n, impute_mode=impute, impute_seed=3)
    plan = WinPlan(sess, annot, ws, 24, 100, 9, "rademacher")
    plan.execute()
    res = plan.results()
    plan.close()
    sess.close()
    for w in range(len(ws) - 1):
        a, b = int(ws[w]), int(ws[w + 1])
        ref = oracle.gw_ldscore(rows, n, annot[a:b], nvecs=24, step=100, seed=window_seed(9, w),
                                impute=impute, impute_seed=3, snp0=a)
        assert_rel_elementwise(res["meansq_accum"][a:b], ref["meansq_accum"], LD_RTOL,
                               f"window {w}")
