"""GPU: the remaining gwldcore drop-in entries (row-major phase 1, Mailman
phase 2, sketch column sums and projections, dosage standardization) against
the reference's own gwldcore.cpp compiled unchanged."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dt", [np.float64, np.float32])
@pytest.mark.parametrize("impute", ["mean", "hwe"])
def test_phase1_rowmajor_matches_reference(small_bed, reference, dt, impute):
    from summit_b200 import gwldcore

    n, m, prefix = small_bed["n"], small_bed["m"], small_bed["prefix"]
    rng = np.random.default_rng(2)
    K, V, a, b = 2, 12, 50, 170
    annot = np.ones((b - a, K), dtype=dt)
    annot[::3, 1] = 0
    inv = (0.5 + rng.random(b - a)).astype(dt)
    start = rng.normal(size=(n, K * V)).astype(dt)  # the row-major entry accumulates
    ref = np.ascontiguousarray(start.copy())
    gpu = np.ascontiguousarray(start.copy())
    kw = dict(impute_mode=impute, impute_seed=9 if impute == "hwe" else None)
    reference.phase1_bed_rowmajor(prefix, a, b, annot, inv, 3, V, 5, "rademacher", 77, ref, **kw)
    gwldcore.phase1_compute_Xz_bed_chunk_rowmajor(prefix, prefix + ".fam", a, b, annot_blk=annot,
                                                  inv_right=inv, v_start=3, v_count=V,
                                                  kmax_hint=5, seed=77, Xz2d_chunk=gpu, **kw)
    # 4 int8 digits per floating operand: ~4e-9 of the column maximum
    assert rel_err(gpu, ref) < (1e-6 if dt == np.float32 else 1e-7)


@pytest.mark.parametrize("dt", [np.float64, np.float32])
def test_phase2_mailman_rowmajor_matches_reference(small_bed, reference, dt):
    from summit_b200 import gwldcore

    n, m, prefix = small_bed["n"], small_bed["m"], small_bed["prefix"]
    rng = np.random.default_rng(3)
    V, K, a, b = 10, 2, 20, 300
    Xz = np.ascontiguousarray(rng.normal(size=(n, K * V)).astype(dt))
    sums = reference.col_sums_rowmajor(Xz)
    inv = (0.5 + rng.random(b - a)).astype(dt)
    ms_r = np.zeros((m, K), dtype=dt)
    ms_g = np.zeros((m, K), dtype=dt)
    mc_r, mc_g = np.zeros((m, K)), np.zeros((m, K))
    reference.phase2_mailman_rowmajor(prefix, a, b, inv, V, Xz, ms_r, sums, n, impute_seed=5,
                                      mc_per_snp=mc_r)
    gwldcore.phase2_accum_XtXz_bed_mailman_rowmajor(prefix, prefix + ".fam", a, b, inv_left=inv,
                                                    tile_nvecs=V, Xz2d=Xz, meansq_accum=ms_g,
                                                    sum_Xz=sums, N_denom=n, impute_seed=5,
                                                    mc_per_snp_sumsq=mc_g)
    assert rel_err(ms_g, ms_r) < 1e-6
    assert rel_err(mc_g, mc_r) < 1e-6
    # the column-major Mailman entry gives the same numbers
    ms_f = np.zeros((m, K), dtype=dt)
    gwldcore.phase2_accum_XtXz_bed_mailman(prefix, prefix + ".fam", a, b, inv_left=inv,
                                           tile_nvecs=V, Xz2d=np.asfortranarray(Xz),
                                           meansq_accum=ms_f, N_denom=n, impute_seed=5)
    assert rel_err(ms_f, ms_r) < 1e-6


@pytest.mark.parametrize("dt", [np.float64, np.float32])
def test_col_sums_and_projections_match_reference(reference, dt):
    from summit_b200 import gwldcore

    rng = np.random.default_rng(4)
    n, q, p = 777, 37, 3
    X = np.ascontiguousarray(rng.normal(size=(n, q)).astype(dt))
    np.testing.assert_array_equal(gwldcore.compute_col_sums_rowmajor(X),
                                  reference.col_sums_rowmajor(X))
    Cm = np.asfortranarray(rng.normal(size=(n, p)).astype(dt))
    Rm = np.asfortranarray(np.linalg.pinv(Cm.astype(np.float64)).astype(dt))
    tol = 1e-5 if dt == np.float32 else 1e-12
    Xr, Xg = X.copy(), X.copy()
    sr = reference.project_rowmajor(Xr, Cm, Rm)
    sg = gwldcore.project_rowmajor_inplace_and_col_sums(Xg, Cm, Rm)
    assert rel_err(Xg, Xr) < tol
    assert np.max(np.abs(sg - sr)) < tol * np.max(np.abs(X)) * n
    Xf_r, Xf_g = np.asfortranarray(X), np.asfortranarray(X).copy(order="F")
    Xf_r = Xf_r.copy(order="F")
    reference.project_colmajor(Xf_r, Cm, Rm)
    gwldcore.project_colmajor_inplace(Xf_g, Cm, Rm)
    assert rel_err(Xf_g, Xf_r) < tol
    # without covariates the row-major call only sums
    Xn = X.copy()
    np.testing.assert_array_equal(gwldcore.project_rowmajor_inplace_and_col_sums(Xn), sr * 0 +
                                  reference.col_sums_rowmajor(X))
    np.testing.assert_array_equal(Xn, X)


@pytest.mark.parametrize("dt", [np.float64, np.float32])
def test_standardize_dosage_matches_reference(reference, dt):
    from summit_b200 import gwldcore

    rng = np.random.default_rng(6)
    n, L = 501, 23
    G = rng.uniform(0, 2, size=(n, L)).astype(dt)
    G[rng.random((n, L)) < 0.05] = -9.0
    G[:, 4] = 1.0           # monomorphic
    G[:, 5] = -9.0          # all missing
    Gr = np.asfortranarray(G.copy())
    Gg = np.asfortranarray(G.copy())
    nr = reference.standardize_dosage(Gr)
    ng = gwldcore.standardize_dosage_inplace(Gg)
    assert nr == ng
    np.testing.assert_array_equal(Gg, Gr)
    bad = np.asfortranarray(G.copy())
    bad[0, 0] = 3.5
    with pytest.raises(RuntimeError, match="out-of-range"):
        gwldcore.standardize_dosage_inplace(bad)


def _covariates(n, p=3, seed=12):
    rng = np.random.default_rng(seed)
    C = np.linalg.qr(np.column_stack([np.ones(n)] + [rng.normal(size=n) for _ in range(p - 1)]))[0]
    return np.asfortranarray(C), np.asfortranarray(C.T)


@pytest.mark.parametrize("dt", [np.float64, np.float32])
def test_residual_variances_with_covariates_match_reference(small_bed, reference, dt):
    """precompute_residual_variances_bed with C, R and snp_var_out, and the
    phase-1 fused residual variances with C, R and the covariate Gram."""
    from summit_b200 import gwldcore

    n, m, prefix = small_bed["n"], small_bed["m"], small_bed["prefix"]
    C, R = _covariates(n)
    sv_r, sv_g = np.zeros(m), np.zeros(m)
    inv_r = reference.resvar_bed_cov(prefix, m, 100, C, R, dtype=dt, snp_var=sv_r)
    inv_g, mu22 = gwldcore.precompute_residual_variances_bed(
        prefix, prefix + ".fam", m, 100, C=C, R=R, impute_mode="mean", snp_var_out=sv_g, dtype=dt)
    assert mu22 is None
    tol = 1e-6 if dt == np.float32 else 1e-9
    assert rel_err(inv_g, inv_r) < tol
    assert np.max(np.abs(sv_g - sv_r)) < tol
    a, b, V, K = 30, 230, 8, 2
    annot = np.ones((b - a, K), dtype=dt)
    gram = (C.T @ C).astype(dt)
    for g in (None, gram):
        Xr = np.zeros((n, K * V), dtype=dt, order="F")
        Xg = np.zeros((n, K * V), dtype=dt, order="F")
        fr = reference.phase1_bed_cov(prefix, a, b, annot, 0, V, 31, Xr, C, R, g)
        fg = np.empty(b - a, dtype=dt)
        gwldcore.phase1_compute_Xz_bed_chunk(prefix, prefix + ".fam", a, b, annot_blk=annot,
                                             inv_right=None, v_start=0, v_count=V, kmax_hint=1,
                                             seed=31, Xz2d_chunk=Xg, C=C, R=R, impute_mode="mean",
                                             resvar_gram=g, inv_out=fg)
        assert rel_err(fg, fr) < tol
        assert rel_err(Xg, Xr) < (1e-6 if dt == np.float32 else 1e-7)
