"""Generalized per-SNP GxE packed products (generalized_gxe_variant.inc:
1749-1988).  CPU: the Mailman mean pack's statistics are pinned to the
reference's genotype.cpp, and the reference's own packed_source_product /
packed_target_product (gxeldcore.cpp compiled unchanged, oracle/_ref) are
checked against the FP64 products of those genotypes.  GPU: liblds's source
and target products against the reference's products on the same fileset,
missing calls included (int8 digits: 1e-6 of each column's largest value)."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import rel_err


def _pack_genotypes(geno, ddof=1):
    """X' (N x M) of the reference's convention: inv_j (g - mu_j) on observed
    calls, 0 on missing, inv_j = sqrt((N - ddof) / M2_j) (1 without spread)."""
    G = geno.astype(np.float64)  # M x N, negative = missing
    ok = G >= 0
    g = np.where(ok, G, 0.0)
    nobs = ok.sum(1)
    mu = np.where(nobs > 0, g.sum(1) / np.maximum(nobs, 1), 0.0)
    m2 = (g * g).sum(1) - g.sum(1) ** 2 / np.maximum(nobs, 1)
    m2[(m2 < 0) & (m2 > -1e-12)] = 0.0
    N = G.shape[1]
    inv = np.where((m2 > 0) & (N - ddof > 0), np.sqrt((N - ddof) / np.where(m2 > 0, m2, 1.0)), 1.0)
    X = np.where(ok, (g - mu[:, None]) * inv[:, None], 0.0)
    return X.T, mu, inv, nobs


def test_pack_statistics_match_reference(small_bed, reference):
    n, m, prefix, geno = small_bed["n"], small_bed["m"], small_bed["prefix"], small_bed["geno"]
    mean, inv, obs = reference.mailman_mean_stats(prefix + ".bed", n, 0, m, ddof=1)
    _, mu, iv, nobs = _pack_genotypes(geno)
    np.testing.assert_array_equal(obs, nobs)
    np.testing.assert_allclose(mean, mu, rtol=1e-15, atol=0)
    np.testing.assert_allclose(inv, iv, rtol=1e-15, atol=0)


@pytest.fixture(scope="module")
def ref_gxe():
    from oracle.oracle import REF_GXE_SO, ReferenceGxe

    if not REF_GXE_SO.exists():
        pytest.skip("reference checker oracle/_ref/libref_gxe.so not built (make -C oracle ref)")
    return ReferenceGxe()


def test_reference_products_match_fp64_formula(small_bed, ref_gxe):
    """The reference's packed products equal -X'^T-style FP64 products of the
    mean-imputed, scaled genotypes (sign convention out = mu sum - raw)."""
    n, geno, prefix = small_bed["n"], small_bed["geno"], small_bed["prefix"]
    X, _, _, _ = _pack_genotypes(geno)
    rng = np.random.default_rng(4)
    a, b, cols = 37, 301, 23
    rhs_s = rng.normal(size=(b - a, cols))
    rhs_t = rng.normal(size=(n, cols))
    src, tgt = ref_gxe.generalized_products(prefix + ".bed", n, a, b, rhs_s, rhs_t)
    assert rel_err(src, -X[:, a:b] @ rhs_s) < 1e-13
    assert rel_err(tgt, -X[:, a:b].T @ rhs_t) < 1e-13


def _colwise_rel(got, ref) -> float:
    scale = np.maximum(np.max(np.abs(ref), axis=0), 1e-300)
    return float(np.max(np.max(np.abs(got - ref), axis=0) / scale))


@pytest.mark.gpu
@pytest.mark.parametrize("a,b,cols", [(37, 301, 23), (0, 410, 64), (128, 129, 5)])
def test_generalized_products_on_device(small_bed, ref_gxe, a, b, cols):
    from summit_b200.gxeldcore import generalized_source_product, generalized_target_product
    from summit_b200.session import GwSession

    n, prefix = small_bed["n"], small_bed["prefix"]
    rng = np.random.default_rng(4 + a)
    sess = GwSession(small_bed["rows"], n, impute_mode="mean")
    rhs_s = rng.normal(size=(b - a, cols))
    rhs_t = rng.normal(size=(n, cols))
    src = generalized_source_product(sess.block(a, b), rhs_s)
    tgt = generalized_target_product(sess.block(a, b), rhs_t)
    src_ref, tgt_ref = ref_gxe.generalized_products(prefix + ".bed", n, a, b, rhs_s, rhs_t)
    assert _colwise_rel(src, src_ref) < 1e-6
    assert _colwise_rel(tgt, tgt_ref) < 1e-6
    sess.close()


@pytest.mark.gpu
def test_generalized_products_reject_bad_inputs(small_bed):
    from summit_b200.gxeldcore import generalized_source_product, generalized_target_product
    from summit_b200.session import GwSession

    n = small_bed["n"]
    rng = np.random.default_rng(4)
    sess = GwSession(small_bed["rows"], n, impute_mode="mean")
    a, b, cols = 37, 301, 23
    rhs_s = rng.normal(size=(b - a, cols))
    rhs_t = rng.normal(size=(n, cols))
    with pytest.raises(RuntimeError, match="mis-sized"):
        generalized_source_product(sess.block(a, b), rhs_s[1:])
    hwe = GwSession(small_bed["rows"], n, impute_mode="hwe", impute_seed=3)
    with pytest.raises(RuntimeError, match="mean-imputed"):
        generalized_target_product(hwe.block(a, b), rhs_t)
    sess.close()
    hwe.close()
