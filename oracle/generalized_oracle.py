"""CPU restatement of the device pieces of the generalized per-variant GxE
estimator.  Test infrastructure only: the tests use it as the checker of
summit_b200.generalized_gxe's host-side algebra (standing in for the device
products) and of the device probe stream; no product path imports it.

* global_probe_sign / global_probes: the reference's counter-based Rademacher
  stream (ldscore/generalized_gxe_variant.py:60-103, 114-152);
* source_product / target_product: the dense products of pass 1
  (generalized_gxe_pass1.py:683-700, base += G (sqrt(a) o Z)) and pass 2
  (generalized_gxe_pass2.py:619, G^T rhs) on a decoded standardized block;
* component_diagonal: the pass-2 component-kernel diagonal numerators
  (generalized_gxe_pass2.py:528-572), projected-feature form.
"""
from __future__ import annotations

import numpy as np

MASK64 = (1 << 64) - 1


def splitmix64(value: int) -> int:
    value = (value + 0x9E3779B97F4A7C15) & MASK64
    value = ((value ^ (value >> 30)) * 0xBF58476D1CE4E5B9) & MASK64
    value = ((value ^ (value >> 27)) * 0x94D049BB133111EB) & MASK64
    return (value ^ (value >> 31)) & MASK64


def namespace_key(namespace: str) -> int:
    value = 0xCBF29CE484222325
    for byte in namespace.encode("utf-8"):
        value ^= byte
        value = (value * 0x100000001B3) & MASK64
    return value


def global_probe_sign(root_seed: int, variant: int, probe: int, key: int) -> float:
    state = splitmix64((root_seed ^ key ^ 0x9E3779B97F4A7C15) & MASK64)
    state ^= splitmix64((variant + 0xD2B74407B1CE6E93) & MASK64)
    state ^= splitmix64((probe + 0xCA5A826395121157) & MASK64)
    return 1.0 if (splitmix64(state) >> 63) else -1.0


def global_probes(root_seed: int, variants, probes, namespace: str) -> np.ndarray:
    key = namespace_key(namespace)
    out = np.empty((len(variants), len(probes)), order="F")
    for c, p in enumerate(probes):
        for r, v in enumerate(variants):
            out[r, c] = global_probe_sign(root_seed, int(v), int(p), key)
    return out


def source_product(X: np.ndarray, j0: int, j1: int, annot_blk: np.ndarray,
                   z: np.ndarray) -> np.ndarray:
    blk = X[:, j0:j1]
    k_count = annot_blk.shape[1]
    return np.asfortranarray(np.concatenate(
        [blk @ (np.sqrt(annot_blk[:, k])[:, None] * z) for k in range(k_count)], axis=1))


def target_product(X: np.ndarray, j0: int, j1: int, Y: np.ndarray) -> np.ndarray:
    return np.asfortranarray(X[:, j0:j1].T @ Y)


def component_diagonal(X: np.ndarray, j0: int, j1: int, annot_blk, basis, fixed, coef,
                       numerator: np.ndarray) -> None:
    blk = X[:, j0:j1]
    q_count = basis.shape[1]
    pairs = [(q, q) for q in range(q_count)] + [
        (q, r) for q in range(q_count - 1) for r in range(q + 1, q_count)]
    p_count = len(pairs)
    feats = []
    for q in range(q_count):
        f = basis[:, q, None] * blk
        if fixed.shape[1]:
            f = f - fixed @ coef[:, q, :].T
        feats.append(f)
    for p, (q, r) in enumerate(pairs):
        factor = 1.0 if q == r else 2.0
        prod = (factor * feats[q] * feats[r]) @ annot_blk   # N x K
        for k in range(annot_blk.shape[1]):
            numerator[k * p_count + p] += prod[:, k]


def project_sources(base: np.ndarray, basis: np.ndarray, fixed: np.ndarray):
    """Pass 1's projection (generalized_gxe_pass1.py:718-757): contextual
    sources (K, Q, B, N) = w - fixed (fixed^T w) with w = basis[:, q] * base[k]
    (base (K, B, N)), and the maximum absolute and relative leakage of
    fixed^T p (zero without fixed effects)."""
    k_count, b_count, n = base.shape
    q_count = basis.shape[1]
    contextual = np.empty((k_count, q_count, b_count, n))
    max_abs = max_rel = 0.0
    for k in range(k_count):
        for q in range(q_count):
            weighted = base[k] * basis[:, q]
            if not fixed.shape[1]:
                contextual[k, q] = weighted
                continue
            projected = weighted - (weighted @ fixed) @ fixed.T
            contextual[k, q] = projected
            leakage = projected @ fixed
            max_abs = max(max_abs, float(np.max(np.abs(leakage), initial=0.0)))
            max_rel = max(max_rel, float(np.linalg.norm(leakage)
                                         / max(1.0, float(np.linalg.norm(projected)))))
    return contextual, max_abs, max_rel


def assemble_rhs(rows: np.ndarray, basis: np.ndarray, fam_t, fam_s) -> np.ndarray:
    """Pass 2's right-hand side (generalized_gxe_pass2.py:401-415): N x K*B*F,
    column (k*B + b)*F + f = basis[:, t] * sources[k, s][b] for family
    f = (fam_t[f], fam_s[f]); rows is the (K, Q, B, N) source array."""
    k_count, _, b_count, n = rows.shape
    f_count = len(fam_t)
    rhs = np.empty((n, k_count * b_count * f_count))
    for k in range(k_count):
        for b in range(b_count):
            for f in range(f_count):
                rhs[:, (k * b_count + b) * f_count + f] = basis[:, fam_t[f]] * rows[k, fam_s[f], b]
    return rhs


def pass2_scores(X: np.ndarray, rhs: np.ndarray, k_count: int, b_count: int, f_count: int,
                 p_count: int, term_off, term_f1, term_f2, residual_rank: float,
                 annot: np.ndarray):
    """Per-variant pass-2 scores and the directed numerator from dense
    products (generalized_gxe_pass2.py:600-693): cross = X^T rhs / rr, column
    (k*B + b)*F + f; directional[j, tp, k*P + sp] = (1/B) sum over the terms of
    (tp, sp) of sum_b cross[j, (k,b,f1)] cross[j, (k,b,f2)]."""
    cross = (X.T @ rhs / residual_rank).reshape(X.shape[1], k_count, b_count, f_count)
    m, c_count = X.shape[1], k_count * p_count
    directional = np.zeros((m, p_count, c_count))
    for tp in range(p_count):
        for sp in range(p_count):
            acc = np.zeros((m, k_count))
            for t in range(term_off[tp * p_count + sp], term_off[tp * p_count + sp + 1]):
                acc += np.einsum("jkb,jkb->jk", cross[:, :, :, term_f1[t]],
                                 cross[:, :, :, term_f2[t]])
            directional[:, tp, np.arange(k_count) * p_count + sp] = acc / b_count
    directed = np.einsum("vk,vpc->kpc", annot, directional).reshape(c_count, c_count)
    return directional, directed
