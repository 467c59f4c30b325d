"""CPU: the GxE oracle restatement against the reference's own gxeldcore.cpp
compiled unchanged (oracle/_ref/libref_gxe.so), and the reference's NumPy-Philox
probes against NumPy itself."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import rel_err


@pytest.fixture(scope="module")
def refgxe():
    from oracle.oracle import REF_GXE_SO, ReferenceGxe

    if not REF_GXE_SO.exists():
        pytest.skip("reference checker oracle/_ref/libref_gxe.so not built (make -C oracle ref)")
    return ReferenceGxe()


def _kernel(refgxe, d, K):
    return refgxe.kernel(d["environments"], d["feature_basis"], d["power_indices"],
                         d["power_offsets"], d["ranks"], d["gram_values"], d["gram_offsets"],
                         d["e2_gram_values"], d["common_basis"], d["directions"], 1, K)


def test_reference_philox_matches_numpy(refgxe):
    from oracle.gxe_oracle import philox_keys, rademacher_block

    keys = philox_keys(91, 3000, range(7))
    for rows in (1, 5, 8, 33, 1000):
        np.testing.assert_array_equal(refgxe.philox_rademacher(keys, rows),
                                      rademacher_block(91, 3000, rows, range(7)))


@pytest.mark.parametrize("T,env_start,K,is_sqrt", [(3, 0, 1, False), (2, 1, 2, True)])
def test_oracle_gxe_matches_reference(oracle, refgxe, small_bed, T, env_start, K, is_sqrt):
    import oracle.gxe_oracle as go

    n, m = small_bed["n"], small_bed["m"]
    X = oracle.standardize(small_bed["rows"], n, 0, m)[0]
    E = 3
    d = go.design(n, E, seed=4, categorical=1)
    rng = np.random.default_rng(8)
    B, L0, L1 = 6, 40, 170
    G = X[:, L0:L1]
    L = L1 - L0
    z = go.rademacher_block(91, L0, L, range(B))
    ann = rng.random((L, K)) + 0.1
    if is_sqrt:
        ann = np.sqrt(ann)
    sx = 0.5 + rng.random((L, T))
    sw = 0.5 + rng.random((L, T))
    cols = T * 2 * K * B
    ker = _kernel(refgxe, d, K)
    ref_t = np.asfortranarray(rng.normal(size=(n, cols)))
    ora_t = ref_t.copy(order="F")
    ker.source_block(ref_t, G, z, ann, sx, sw, env_start, is_sqrt)
    go.source_block(ora_t, G, z, ann, sx, sw, d["environments"], env_start, is_sqrt)
    assert rel_err(ora_t, ref_t) < 1e-12
    ref_leak = ker.project_sources(ref_t, K * B, env_start)
    ora_leak = go.project_sources(ora_t, K * B, env_start, d["common_basis"], d["directions"],
                                  d["fixed_bases"])
    assert rel_err(ora_t, ref_t) < 1e-11
    assert np.all(ref_leak < 1e-12) and np.all(ora_leak < 1e-12)
    wts = d["environments"][:, env_start:env_start + T]
    pair = ker.pair(ref_t, wts)
    opair = go.row_weighted_pair(ora_t, wts)
    rows = E * m
    racc = [np.zeros((rows, K)) for _ in range(4)]
    oacc = [np.zeros((rows, K)) for _ in range(4)]
    for (a, b) in [(0, 100), (100, m)]:
        ker.target_score_block(X[:, a:b], pair, sx[:b - a] if b - a <= L else np.ones((b - a, T)),
                               sw[:b - a] if b - a <= L else np.ones((b - a, T)), racc, a, m, B,
                               env_start)
        go.target_score_block(X[:, a:b], opair, sx[:b - a] if b - a <= L else np.ones((b - a, T)),
                              sw[:b - a] if b - a <= L else np.ones((b - a, T)), oacc, a, m, B,
                              env_start, d["ranks"], K)
    ker.normalize_scores(racc, B)
    go.normalize_scores(oacc, B)
    for r_, o_ in zip(racc, oacc):
        assert rel_err(o_, r_) < 1e-11
    refgxe.lib.refg_pair_destroy(pair)


def test_reference_rejects_leaky_projection(refgxe, small_bed):
    """A panel that keeps a component along the environment's fixed-effect
    basis after projection is an error (gxeldcore.cpp:11717-11722)."""
    import oracle.gxe_oracle as go

    n = small_bed["n"]
    d = go.design(n, 2, seed=1)
    ker = _kernel(refgxe, d, 1)
    # a directions array that differs from the fixed-effect basis leaves leakage
    bad = dict(d)
    bad["directions"] = np.asfortranarray(np.random.default_rng(0).normal(size=(n, 2)))
    ker_bad = _kernel(refgxe, bad, 1)
    panel = np.asfortranarray(np.random.default_rng(1).normal(size=(n, 4)))
    with pytest.raises(RuntimeError, match="excessive leakage"):
        ker_bad.project_sources(panel.copy(order="F"), 2, 0)
    assert ker.project_sources(panel.copy(order="F"), 2, 0).max() < 1e-12
