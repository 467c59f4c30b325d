"""GPU: gwldcore entries for dense genotype blocks, covariate projections
inside phase 1 / phase 2, the legacy direct phase 2, GRM panel products, the
mu22 moments and the binary block corrections, each against the reference's
own gwldcore.cpp compiled unchanged.

Tolerances: the dense entries compute in FP64 on the device (reference FP64:
1e-10; float32 overloads: the reference accumulates in float, 1e-4).  The
BED entries carry the 4-digit int8 representation (~4e-9 of a column's
maximum): 1e-6.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu


def _cov(n, p=3, seed=12, symmetric=True):
    rng = np.random.default_rng(seed)
    C = np.column_stack([np.ones(n)] + [rng.normal(size=n) for _ in range(p - 1)])
    R = np.linalg.pinv(C)
    if not symmetric:
        R = R + 0.05 * rng.normal(size=R.shape) / np.sqrt(n)  # C R no longer symmetric
    return np.asfortranarray(C), np.asfortranarray(R)


def _dense(n, L, dt, seed=3):
    rng = np.random.default_rng(seed)
    g = rng.binomial(2, rng.uniform(0.05, 0.5, size=L), size=(n, L)).astype(np.float64)
    g = (g - g.mean(0)) / np.where(g.std(0) > 0, g.std(0), 1.0)
    return np.asfortranarray(g.astype(dt))


def _tol(dt):
    return 1e-4 if dt == np.float32 else 1e-10


@pytest.fixture(autouse=True)
def _fresh_reference_caches(reference):
    """The reference caches phase-1 CSR lists keyed by the annotation and
    inverse-sd buffer ADDRESSES (gwldcore.cpp:1065-1100); numpy reuses freed
    addresses between tests, so a stale list would be returned.  Clear it."""
    reference.clear_caches()
    yield


@pytest.mark.parametrize("dt", [np.float64, np.float32])
@pytest.mark.parametrize("fused", [False, True])
def test_phase1_geno_matches_reference(reference, dt, fused):
    from summit_b200 import gwldcore

    n, L, K, V = 301, 90, 3, 20
    rng = np.random.default_rng(5)
    G = _dense(n, L, dt)
    annot = (rng.random((L, K)) < 0.5).astype(dt)
    annot[:, 0] = 1
    annot[:, 2] = 0  # an empty bin keeps its columns
    inv = (0.5 + rng.random(L)).astype(dt)
    start = rng.normal(size=(n, K * V)).astype(dt)
    Xr = np.asfortranarray(start.copy())
    Xg = np.asfortranarray(start.copy())
    br = np.array([1, 0, 0], dtype=np.uint8)
    bg = br.copy()
    C, R = _cov(n)
    kw = dict(C=C.astype(dt), R=R.astype(dt), gram=(C.T @ C).astype(dt)) if fused else {}
    fr = np.empty(L, dtype=dt) if fused else None
    fg = np.empty(L, dtype=dt) if fused else None
    reference.phase1_geno_cov(np.asfortranarray(G.copy()), 200, annot, None if fused else inv, 4,
                              V, 99, Xr, br, C=kw.get("C"), R=kw.get("R"), gram=kw.get("gram"),
                              inv_out=fr)
    gwldcore.phase1_compute_Xz_geno_chunk(G, 200, annot_blk=annot,
                                          inv_right=None if fused else inv, v_start=4, v_count=V,
                                          kmax_hint=1, seed=99, Xz2d_chunk=Xg, bin_init_mask=bg,
                                          C=kw.get("C"), R=kw.get("R"),
                                          resvar_gram=kw.get("gram"), inv_out=fg)
    np.testing.assert_array_equal(bg, br)
    if fused:
        assert rel_err(fg, fr) < _tol(dt)
    assert rel_err(Xg, Xr) < _tol(dt)
    np.testing.assert_array_equal(Xg[:, 2 * V:], start[:, 2 * V:])


@pytest.mark.parametrize("dt", [np.float64, np.float32])
@pytest.mark.parametrize("cov", [False, True])
def test_phase2_geno_matches_reference(reference, dt, cov):
    from summit_b200 import gwldcore

    n, L, K, V, M = 287, 70, 2, 16, 120
    rng = np.random.default_rng(6)
    Gr = _dense(n, L, dt, seed=4)
    Gg = np.asfortranarray(Gr.copy())
    Xz = np.asfortranarray(rng.normal(size=(n, K * V)).astype(dt))
    inv = (0.5 + rng.random(L)).astype(dt)
    C, R = _cov(n, symmetric=False)
    C, R = (C.astype(dt), R.astype(dt)) if cov else (None, None)
    ms_r = np.zeros((M, K), dtype=dt)
    ms_g = np.zeros((M, K), dtype=dt)
    agg_r, agg_g = np.zeros(K), np.zeros(K)
    mc_r, mc_g = np.zeros((M, K)), np.zeros((M, K))
    reference.phase2_geno_cov(Gr, 30, inv, V, Xz, ms_r, n, C, R, agg_r, mc_r)
    gwldcore.phase2_accum_XtXz_geno(Gg, 30, inv_left=inv, tile_nvecs=V, Xz2d=Xz,
                                    meansq_accum=ms_g, C=C, R=R, N_denom=n,
                                    mc_aggregate_sumsq=agg_g, mc_per_snp_sumsq=mc_g)
    assert rel_err(Gg, Gr) < _tol(dt)  # the projection is applied to the caller's block
    assert rel_err(ms_g, ms_r) < _tol(dt)
    assert rel_err(mc_g, mc_r) < 10 * _tol(dt)
    assert rel_err(agg_g, agg_r) < 10 * _tol(dt)


@pytest.mark.parametrize("mailman", [False, True])
@pytest.mark.parametrize("symmetric", [True, False])
def test_phase2_bed_with_covariates_matches_reference(small_bed, reference, mailman, symmetric):
    from summit_b200 import gwldcore

    n, m, prefix = small_bed["n"], small_bed["m"], small_bed["prefix"]
    rng = np.random.default_rng(7)
    V, K, a, b = 12, 2, 40, 330
    Xz = np.asfortranarray(rng.normal(size=(n, K * V)))
    inv = 0.5 + rng.random(b - a)
    C, R = _cov(n, symmetric=symmetric)
    ms_r, ms_g = np.zeros((m, K)), np.zeros((m, K))
    mc_r, mc_g = np.zeros((m, K)), np.zeros((m, K))
    reference.phase2_bed_cov(prefix, a, b, inv, V, Xz, ms_r, n, C, R, mailman=mailman,
                             mc_per_snp=mc_r)
    if mailman:
        gwldcore.phase2_accum_XtXz_bed_mailman(prefix, prefix + ".fam", a, b, inv_left=inv,
                                               tile_nvecs=V, Xz2d=Xz, meansq_accum=ms_g, C=C, R=R,
                                               N_denom=n, mc_per_snp_sumsq=mc_g)
    else:
        gwldcore.phase2_accum_XtXz_bed(prefix, prefix + ".fam", a, b, inv_left=inv, tile_nvecs=V,
                                       Xz2d=Xz, meansq_accum=ms_g, C=C, R=R, N_denom=n,
                                       impute_mode="mean", mc_per_snp_sumsq=mc_g)
    assert rel_err(ms_g, ms_r) < 1e-6
    assert rel_err(mc_g, mc_r) < 1e-5


def test_phase1_bed_project_right_matches_reference(small_bed, reference):
    from summit_b200 import gwldcore

    n, m, prefix = small_bed["n"], small_bed["m"], small_bed["prefix"]
    rng = np.random.default_rng(8)
    K, V, a, b = 2, 10, 60, 250
    annot = np.ones((b - a, K))
    annot[::2, 1] = 0
    inv = 0.5 + rng.random(b - a)
    C, R = _cov(n, symmetric=False)
    start = np.asfortranarray(rng.normal(size=(n, K * V)))
    Xr, Xg = start.copy(order="F"), start.copy(order="F")
    br = np.array([1, 0], dtype=np.uint8)
    bg = br.copy()
    reference.phase1_bed_projright(prefix, a, b, annot, inv, 2, V, 17, Xr, C, R, bin_init=br)
    gwldcore.phase1_compute_Xz_bed_chunk(prefix, prefix + ".fam", a, b, annot_blk=annot,
                                         inv_right=inv, v_start=2, v_count=V, kmax_hint=1,
                                         seed=17, Xz2d_chunk=Xg, bin_init_mask=bg,
                                         project_right=True, C=C, R=R, impute_mode="mean")
    np.testing.assert_array_equal(bg, br)
    assert rel_err(Xg, Xr) < 1e-7
    with pytest.raises(RuntimeError, match="incompatible with project_right"):
        gwldcore.phase1_compute_Xz_bed_chunk(prefix, prefix + ".fam", a, b, annot_blk=annot,
                                             inv_right=None, v_start=2, v_count=V, kmax_hint=1,
                                             seed=17, Xz2d_chunk=Xg, project_right=True, C=C, R=R,
                                             impute_mode="mean", inv_out=np.empty(b - a))


@pytest.mark.parametrize("cov", [False, True])
def test_phase2_legacy_matches_reference(small_bed, reference, cov):
    from summit_b200 import gwldcore

    n, m, prefix = small_bed["n"], small_bed["m"], small_bed["prefix"]
    rng = np.random.default_rng(9)
    V, K, a, b = 14, 3, 0, 200
    Xz = np.asfortranarray(rng.normal(size=(n, K * V)))
    inv = 0.5 + rng.random(b - a)
    C, R = _cov(n) if cov else (None, None)
    ms_r, ms_g = np.full((m, K), 0.25), np.full((m, K), 0.25)
    reference.phase2_legacy(prefix, a, b, inv, V, Xz, ms_r, n, C, R)
    gwldcore.phase2_compute_XtXz_bed(prefix, prefix + ".fam", a, b, inv_left=inv, nvecs=V,
                                     vchunk=V, Xz2d=Xz, meansq=ms_g, C=C, R=R, N_denom=n,
                                     impute_mode="mean")
    assert rel_err(ms_g, ms_r) < 1e-6


@pytest.mark.parametrize("dt", [np.float64, np.float32])
@pytest.mark.parametrize("mode", ["mean", "hwe", "mailman"])
def test_apply_grm_matches_reference(small_bed, reference, dt, mode):
    from summit_b200 import gwldcore

    n, m, prefix = small_bed["n"], small_bed["m"], small_bed["prefix"]
    rng = np.random.default_rng(10)
    Q, nsnps = 9, 380
    pin = np.asfortranarray(rng.normal(size=(n, Q)).astype(dt))
    inv = (0.5 + rng.random(m)).astype(dt)
    inv[5] = 0.0  # dropped from the GRM
    C, R = _cov(n)
    C, R = C.astype(dt), R.astype(dt)
    for cv in (False, True):
        kw = dict(C=C, R=R) if cv else {}
        if mode == "mailman":
            want = reference.apply_grm(prefix, nsnps, 100, inv, pin, impute_seed=4, mailman=True,
                                       **kw)
            got = np.zeros((n, Q), dtype=dt, order="F")
            gwldcore.apply_grm_bed_panel_mailman(prefix, prefix + ".fam", nsnps, 100,
                                                 inv_all=inv, panel_in=pin, panel_out=got,
                                                 impute_seed=4, **kw)
        else:
            want = reference.apply_grm(prefix, nsnps, 100, inv, pin, impute_mode=mode,
                                       impute_seed=4, **kw)
            got = np.zeros((n, Q), dtype=dt, order="F")
            gwldcore.apply_grm_bed_panel(prefix, prefix + ".fam", nsnps, 100, inv_all=inv,
                                         panel_in=pin, panel_out=got, impute_mode=mode,
                                         impute_seed=4, **kw)
        assert rel_err(got, want) < (1e-4 if dt == np.float32 else 1e-6)


@pytest.mark.parametrize("dt", [np.float64, np.float32])
@pytest.mark.parametrize("cov", [False, True])
def test_mu22_matches_reference(small_bed, reference, dt, cov):
    from summit_b200 import gwldcore

    n, m, prefix = small_bed["n"], small_bed["m"], small_bed["prefix"]
    rng = np.random.default_rng(11)
    B = 4
    annot = (rng.random((m, B)) < 0.4).astype(dt)
    annot[:, 0] = 1
    annot[:, 3] = 0  # empty bin: zero row and column
    C, R = _cov(n) if cov else (None, None)
    if cov:
        C, R = C.astype(dt), R.astype(dt)
    inv_r, mu_r = reference.resvar_mu22(prefix, m, 100, annot, C, R, dtype=dt)
    inv_g, mu_g = gwldcore.precompute_residual_variances_bed(
        prefix, prefix + ".fam", m, 100, compute_mu22=True, annot_all=annot, C=C, R=R,
        impute_mode="mean")
    assert inv_g.dtype == dt
    assert rel_err(inv_g, inv_r) < (1e-6 if dt == np.float32 else 1e-9)
    assert rel_err(mu_g, mu_r) < (1e-5 if dt == np.float32 else 1e-9)
    np.testing.assert_array_equal(mu_g[3], 0.0)


@pytest.mark.parametrize("adt", [np.float64, np.float32])
def test_block_corrections_match_reference(reference, adt):
    from summit_b200 import gwldcore

    rng = np.random.default_rng(12)
    M, B = 5000, 6
    meansq = rng.gamma(2.0, 1.0, size=(M, B))
    annot = (rng.random((M, B)) < 0.3).astype(adt)
    annot[:, 5] = 0
    mu22 = rng.random((B, B)) + 1.0
    want = reference.block_corrections(meansq, mu22, annot, 4000, 1.7)
    got = gwldcore.compute_block_corrections_binary(meansq, mu22, annot, 4000, 1.7)
    for g, w in zip(got, want):
        np.testing.assert_allclose(g, w, rtol=1e-12, atol=0)
    with pytest.raises(RuntimeError, match="N must be > 1"):
        gwldcore.compute_block_corrections_binary(meansq, mu22, annot, 1, 1.0)
