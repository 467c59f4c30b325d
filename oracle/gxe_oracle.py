"""ORACLE — FP64 numpy restatement of the SUMMIT-GxE multi-environment
products (test infrastructure; only tests/ and bench.py's CPU leg use it).

Follows MultiEnvironmentKernel in src/native/gxeldcore.cpp:
* source_block        :11008-11240
* project_sources     :11583-11729
* prepare_protected_row_weighted_pair :9808-9870
* target_score_block  :11731-11936
* normalize_scores    :12490-12557
and the probe streams of src/summit/ldscore/gwe_ldscore.py:524-530
(_make_seed) and :2484-2505 (_generate_random_block, NumPy Philox).
``design`` returns the package's synthetic kernel inputs
(summit_b200.gxe.synthetic_design).
"""
from __future__ import annotations

import numpy as np

MASK64 = 0xFFFFFFFFFFFFFFFF


def mix64(x: int) -> int:
    x = (x + 0x9E3779B97F4A7C15) & MASK64
    x = ((x ^ (x >> 30)) * 0xBF58476D1CE4E5B9) & MASK64
    x = ((x ^ (x >> 27)) * 0x94D049BB133111EB) & MASK64
    return (x ^ (x >> 31)) & MASK64


def make_seed(root: int, block: int, probe_id: int) -> int:
    """gwe_ldscore.py:524-530."""
    s = 0x1234ABCD
    s ^= mix64(int(root))
    s ^= mix64(int(block) + 0x9E37)
    s ^= mix64(int(probe_id) + 0x85EB)
    return s & MASK64


def philox_keys(root: int, block: int, probe_ids) -> np.ndarray:
    """NumPy Philox keys of the per-(block, probe) streams (P x 2 uint64)."""
    return np.asarray([np.random.Philox(make_seed(root, block, int(p))).state["state"]["key"]
                       for p in probe_ids], dtype=np.uint64)


def rademacher_block(root: int, block: int, L: int, probe_ids) -> np.ndarray:
    """_generate_random_block for rand_dist='rademacher' (L x P, column-major)."""
    Z = np.empty((L, len(probe_ids)), order="F")
    for q, p in enumerate(probe_ids):
        g = np.random.Generator(np.random.Philox(make_seed(root, block, int(p))))
        Z[:, q] = 2.0 * g.integers(0, 2, size=L, dtype=np.int8).astype(np.float64) - 1.0
    return Z


def source_block(target, genotype, probes, annotation, scale_x, scale_w, env, environment_start,
                 annotation_is_sqrt=False):
    L, B = probes.shape
    K = annotation.shape[1]
    T = scale_x.shape[1]
    cols = K * B
    sq = annotation if annotation_is_sqrt else np.sqrt(np.maximum(annotation, 0.0))
    for e in range(T):
        for k in range(K):
            wx = sq[:, k, None] * probes * scale_x[:, e, None]
            ww = sq[:, k, None] * probes * scale_w[:, e, None]
            a = e * 2 * cols + k * B
            target[:, a:a + B] += genotype @ wx
            target[:, a + cols:a + cols + B] += env[:, environment_start + e, None] * (genotype @ ww)


def project_sources(panel, columns_per_environment, environment_start, common, directions,
                    fixed_bases):
    """fixed_bases[e]: N x rank_e basis the leakage is measured on."""
    n = panel.shape[0]
    tile = panel.shape[1] // (2 * columns_per_environment)
    if common.shape[1]:
        panel -= common @ (common.T @ panel)
    for e in range(tile):
        seg = slice(e * 2 * columns_per_environment, (e + 1) * 2 * columns_per_environment)
        d = directions[:, environment_start + e]
        coef = d @ panel[:, seg]
        mean = panel[:, seg].sum(axis=0) / n
        panel[:, seg] -= d[:, None] * coef[None, :] + mean[None, :]
    leak = np.zeros(tile)
    for e in range(tile):
        seg = panel[:, e * 2 * columns_per_environment:(e + 1) * 2 * columns_per_environment]
        den = (seg * seg).sum(axis=0)
        co = fixed_bases[environment_start + e].T @ seg
        rel = np.sqrt((co * co).sum(axis=0) / den)
        if not np.all(np.isfinite(rel)) or rel.max() > 1e-9:
            raise RuntimeError("Multi-environment native source projection has excessive leakage")
        leak[e] = rel.max()
    return leak


def row_weighted_pair(right, row_weights):
    groups = row_weights.shape[1]
    per = right.shape[1] // groups
    w = np.repeat(row_weights, per, axis=1)
    return np.asfortranarray(np.hstack([right, w * right]))


def target_score_block(genotype, pair, scale_x, scale_w, accs, block_start, total_variants,
                       probe_count, environment_start, ranks, K):
    n, L = genotype.shape
    T = scale_x.shape[1]
    B = probe_count
    cols = K * B
    pair_cols = T * 2 * cols
    out = genotype.T @ pair
    xx, xw, wx, ww = accs
    for e in range(T):
        env = environment_start + e
        df = float(n - ranks[env])
        sc = 1.0 / (df * df)
        rows = env * total_variants + block_start + np.arange(L)
        for k in range(K):
            a = e * 2 * cols + k * B
            b = a + cols
            sx, sw = scale_x[:, e, None], scale_w[:, e, None]
            xx[rows, k] += ((sx * out[:, a:a + B]) ** 2).sum(1) * sc
            xw[rows, k] += ((sx * out[:, b:b + B]) ** 2).sum(1) * sc
            wx[rows, k] += ((sw * out[:, pair_cols + a:pair_cols + a + B]) ** 2).sum(1) * sc
            ww[rows, k] += ((sw * out[:, pair_cols + b:pair_cols + b + B]) ** 2).sum(1) * sc


def normalize_scores(accs, probe_count):
    for a in accs:
        a *= 1.0 / float(probe_count)


def design(n: int, E: int, seed: int = 0, n_cov: int = 1, categorical: int = 0):
    """Synthetic kernel inputs (summit_b200.gxe.synthetic_design)."""
    from summit_b200.gxe import synthetic_design

    return synthetic_design(n, E, seed, n_cov, categorical)
