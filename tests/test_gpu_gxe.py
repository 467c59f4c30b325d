"""GPU: SUMMIT-GxE multi-environment products (drop-in gxeldcore) against the
reference's own gxeldcore.cpp compiled unchanged.

The GPU computes the genotype products on int8 tensor cores with 4-digit
operand splits; the stated tolerance against the reference's FP64 BLAS is
1e-6 relative (measured ~1e-8)."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu
TOL = 1e-6


@pytest.fixture(scope="module")
def refgxe():
    from oracle.oracle import REF_GXE_SO, ReferenceGxe

    if not REF_GXE_SO.exists():
        pytest.skip("reference checker oracle/_ref/libref_gxe.so not built (make -C oracle ref)")
    return ReferenceGxe()


def _kernels(refgxe, d, K):
    from summit_b200 import gxeldcore

    args = (d["environments"], d["feature_basis"], d["power_indices"], d["power_offsets"],
            d["ranks"], d["gram_values"], d["gram_offsets"], d["e2_gram_values"],
            d["common_basis"], d["directions"], 1, K)
    return refgxe.kernel(*args), gxeldcore.MultiEnvironmentKernel(*args, 2)


def test_philox_rademacher_matches_numpy():
    from oracle.gxe_oracle import philox_keys, rademacher_block
    from summit_b200 import gxeldcore

    keys = philox_keys(91, 1000, range(11))
    for rows in (1, 7, 8, 64, 1001, 20000):
        np.testing.assert_array_equal(gxeldcore.numpy_philox_rademacher_block(keys, rows, 2),
                                      rademacher_block(91, 1000, rows, range(11)))


# B = 40 gives 160 digit columns per group: the target's CTAs then take 8
# groups each, walked in 256-column MMA groups that split groups.
@pytest.mark.parametrize("T,env_start,K,is_sqrt,B", [(3, 0, 1, False, 6), (2, 1, 2, True, 6),
                                                    (2, 0, 2, False, 40)])
def test_gxe_products_match_reference(oracle, refgxe, small_bed, T, env_start, K, is_sqrt, B):
    from oracle.gxe_oracle import design, rademacher_block
    from summit_b200.session import GwSession

    n, m, packed = small_bed["n"], small_bed["m"], small_bed["rows"]
    X = oracle.standardize(packed, n, 0, m)[0]
    E = 3
    d = design(n, E, seed=4, categorical=1)
    ref, gpu = _kernels(refgxe, d, K)
    sess = GwSession(packed, n)
    rng = np.random.default_rng(8)
    cols = T * 2 * K * B
    blocks = [(0, 150), (150, 151), (151, m)]  # includes a one-SNP block
    target_r = np.asfortranarray(rng.normal(size=(n, cols)))
    target_g = target_r.copy(order="F")
    scales = {}
    for (a, b) in blocks:
        L = b - a
        z = rademacher_block(77, a, L, range(B))
        ann = rng.random((L, K)) + 0.05
        ann[::5, 0] = 0.0
        if is_sqrt:
            ann = np.sqrt(ann)
        sx = 0.5 + rng.random((L, T))
        sw = 0.5 + rng.random((L, T))
        scales[(a, b)] = (sx, sw)
        ref.source_block(target_r, X[:, a:b], z, ann, sx, sw, env_start, is_sqrt)
        assert gpu.source_block(target_g, sess.block(a, b), z, ann, sx, sw, env_start,
                                annotation_is_sqrt=is_sqrt) == 0
    assert rel_err(target_g, target_r) < TOL
    lr = ref.project_sources(target_r, K * B, env_start)
    lg = gpu.project_sources(target_g, K * B, env_start)
    assert lg.shape == lr.shape and np.all(lg < 1e-12)
    assert rel_err(target_g, target_r) < TOL
    from summit_b200.gxeldcore import prepare_protected_row_weighted_pair

    w = d["environments"][:, env_start:env_start + T]
    pair_r = ref.pair(target_r, w)
    pair_g = prepare_protected_row_weighted_pair(target_g, w, 2)
    assert (pair_g.rows, pair_g.columns) == (n, cols)
    accs_r = [np.zeros((E * m, K)) for _ in range(4)]
    accs_g = [np.zeros((E * m, K)) for _ in range(4)]
    for (a, b) in blocks:
        sx, sw = scales[(a, b)]
        ref.target_score_block(X[:, a:b], pair_r, sx, sw, accs_r, a, m, B, env_start)
        gpu.target_score_block(sess.block(a, b), pair_g, sx, sw, *accs_g, a, m, B, env_start)
    ref.normalize_scores(accs_r, B)
    gpu.normalize_scores(*accs_g, B)
    for name, r_, g_ in zip(("xx", "xw", "wx", "ww"), accs_r, accs_g):
        assert rel_err(g_, r_) < TOL, name
    refgxe.lib.refg_pair_destroy(pair_r)
    sess.close()


def test_gxe_rejects_invalid_inputs(small_bed):
    from oracle.gxe_oracle import design
    from summit_b200 import gxeldcore
    from summit_b200.session import GwSession

    n, m, packed = small_bed["n"], small_bed["m"], small_bed["rows"]
    d = design(n, 2, seed=1)
    k = gxeldcore.MultiEnvironmentKernel(d["environments"], d["feature_basis"],
                                         d["power_indices"], d["power_offsets"], d["ranks"],
                                         d["gram_values"], d["gram_offsets"], d["e2_gram_values"],
                                         d["common_basis"], d["directions"], 1, 1, 2)
    sess = GwSession(packed, n)
    L, B = 10, 3
    target = np.zeros((n, 2 * 1 * B), order="F")
    z = np.ones((L, B))
    bad = np.ones((L, 1))
    bad[3, 0] = 0.0
    with pytest.raises(RuntimeError, match="invalid values"):
        k.source_block(target, sess.block(0, L), z, np.ones((L, 1)), bad, np.ones((L, 1)), 0)
    with pytest.raises(TypeError, match="float64"):
        k.source_block(target, np.zeros((n, L), dtype=np.float32), z, np.ones((L, 1)),
                       np.ones((L, 1)), np.ones((L, 1)), 0)
    with pytest.raises(RuntimeError, match="rows do not match"):
        k.source_block(target, np.zeros((n - 1, L)), z, np.ones((L, 1)), np.ones((L, 1)),
                       np.ones((L, 1)), 0)
    with pytest.raises(RuntimeError, match="mis-sized"):
        k.source_block(np.zeros((n, 5), order="F"), sess.block(0, L), z, np.ones((L, 1)),
                       np.ones((L, 1)), np.ones((L, 1)), 0)
    sess.close()


@pytest.mark.parametrize("T,env_start,K", [(3, 0, 1), (2, 1, 2)])
def test_gxe_dense_genotype_dropin_matches_reference(oracle, refgxe, small_bed, T, env_start, K):
    """The reference builder's call sequence (GenomewideEnvLDScore.native_source_block /
    native_target_score_block, gxe_multi.py:3066-3230) with the reference's own
    argument: dense N x L FP64 standardized genotype blocks, the same arrays
    handed to the reference's compiled gxeldcore.cpp and to the shim."""
    from oracle.gxe_oracle import design, rademacher_block
    from summit_b200.gxeldcore import prepare_protected_row_weighted_pair

    n, m, packed = small_bed["n"], small_bed["m"], small_bed["rows"]
    X = oracle.standardize(packed, n, 0, m)[0]
    E = 3
    d = design(n, E, seed=5, categorical=1)
    ref, gpu = _kernels(refgxe, d, K)
    rng = np.random.default_rng(9)
    B = 5
    cols = T * 2 * K * B
    blocks = [(0, 97), (97, 98), (98, m)]
    target_r = np.zeros((n, cols), order="F")
    target_g = np.zeros((n, cols), order="F")
    scales = {}
    for (a, b) in blocks:
        L = b - a
        z = rademacher_block(11, a, L, range(B))
        ann = rng.random((L, K)) + 0.05
        ann[::7, 0] = 0.0
        sx = 0.5 + rng.random((L, T))
        sw = 0.5 + rng.random((L, T))
        scales[(a, b)] = (sx, sw)
        geno = np.asfortranarray(X[:, a:b], dtype=np.float64)
        ref.source_block(target_r, geno, z, ann, sx, sw, env_start, False)
        assert gpu.source_block(target_g, geno, z, ann, sx, sw, env_start) == 0
    assert rel_err(target_g, target_r) < 1e-12
    ref.project_sources(target_r, K * B, env_start)
    gpu.project_sources(target_g, K * B, env_start)
    assert rel_err(target_g, target_r) < 1e-12
    w = d["environments"][:, env_start:env_start + T]
    pair_r = ref.pair(target_r, w)
    pair_g = prepare_protected_row_weighted_pair(target_g, w, 2)
    accs_r = [np.zeros((E * m, K)) for _ in range(4)]
    accs_g = [np.zeros((E * m, K)) for _ in range(4)]
    for (a, b) in blocks:
        sx, sw = scales[(a, b)]
        geno = np.asfortranarray(X[:, a:b], dtype=np.float64)
        ref.target_score_block(geno, pair_r, sx, sw, accs_r, a, m, B, env_start)
        gpu.target_score_block(geno, pair_g, sx, sw, *accs_g, a, m, B, env_start)
    ref.normalize_scores(accs_r, B)
    gpu.normalize_scores(*accs_g, B)
    for name, r_, g_ in zip(("xx", "xw", "wx", "ww"), accs_r, accs_g):
        assert rel_err(g_, r_) < 1e-12, name
    refgxe.lib.refg_pair_destroy(pair_r)
