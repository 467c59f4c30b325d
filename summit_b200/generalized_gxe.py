"""Generalized per-variant GxE LD scores: the exact two-pass estimator on the GPU.

Mirrors ``GeneralizedGxEPass1Executor.execute`` (ldscore/generalized_gxe_pass1.py:
586-800) and ``GeneralizedGxEPass2Executor.execute`` (generalized_gxe_pass2.py:
441-860) over a resident genotype image (``GwSession``), whose standardized
genotypes are the decoded blocks the reference's genotype operator supplies:

* pass 1: base_k = X (sqrt(a_k) o Z) on the phase-1 tensor-core kernel
  (Z the global variant x probe Rademacher stream, generated on the device),
  contextual_{k,q} = P (phi_q o base_k) with P = I - F F^T, and the reference's
  projection-leakage check;
* pass 2: cross_{t,s,k} = X^T (phi_t o contextual_{k,s}) / (N - R) on the
  phase-2 tensor-core kernel (one family per unordered (t, s) when there are no
  fixed effects, every ordered pair otherwise), the per-variant orientation
  products averaged over probes (directional scores, M x P x K*P), the directed
  numerator, and the component-kernel diagonals on the device.

Pairs are ordered diagonal first, then lexicographic off-diagonals, with kernel
factor 1 on the diagonal and 2 off it; components are annotation-major
(component k * P + p), as in context/spec.py.  There is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib
from ._lib import check, ptr

PROBE_NAMESPACE = "summit.generalized_gxe.variant_ldscore.reference"
_MASK64 = (1 << 64) - 1


def probe_namespace_key(namespace: str) -> int:
    """FNV-1a key of a probe namespace (generalized_gxe_variant.py:69-78)."""
    if not isinstance(namespace, str) or not namespace:
        raise ValueError("probe namespace must be a nonempty string")
    value = 0xCBF29CE484222325
    for byte in namespace.encode("utf-8"):
        value ^= byte
        value = (value * 0x100000001B3) & _MASK64
    return value


@dataclass(frozen=True)
class GlobalVariantProbeSpec:
    """Fields of the reference's spec (generalized_gxe_variant.py:155-174)."""
    root_seed: int
    probe_offset: int
    probe_count: int
    namespace: str = PROBE_NAMESPACE

    def __post_init__(self) -> None:
        for name in ("root_seed", "probe_offset", "probe_count"):
            value = getattr(self, name)
            if isinstance(value, bool) or not isinstance(value, int):
                raise ValueError(f"{name} must be an integer")
        if self.root_seed < 0 or self.root_seed > _MASK64:
            raise ValueError("root_seed must be in uint64 range")
        if self.probe_offset < 0 or self.probe_count < 1:
            raise ValueError("probe_offset must be nonnegative and probe_count positive")
        probe_namespace_key(self.namespace)


def global_variant_probes(spec: GlobalVariantProbeSpec, variant_start: int,
                          variant_count: int) -> np.ndarray:
    """Signs for variants [variant_start, +count) and all of the spec's probes
    (variant_count x probe_count, Fortran order), computed on the device."""
    out = np.empty((variant_count, spec.probe_count), order="F")
    check(_lib.load().lds_global_variant_probes(
        spec.root_seed, probe_namespace_key(spec.namespace), int(variant_start),
        int(variant_count), spec.probe_offset, spec.probe_count, ptr(out)))
    return out


# Device products (liblds); one function each so that a test can stand an
# independent restatement in for them when checking the host-side algebra.
def _source_product(session, j0: int, j1: int, annot_blk: np.ndarray, z: np.ndarray) -> np.ndarray:
    """N x K*B (column k*B + b) = sum_j x_j sqrt(a_jk) z_jb over [j0, j1)."""
    k_count, b_count = annot_blk.shape[1], z.shape[1]
    out = np.empty((session.N, k_count * b_count), order="F")
    a = np.ascontiguousarray(annot_blk, dtype=np.float64)
    zf = np.asfortranarray(z, dtype=np.float64)
    check(_lib.load().lds_geno_source_product(session.handle, j0, j1, ptr(a), k_count, ptr(zf),
                                              b_count, ptr(out)))
    return out


def _target_product(session, j0: int, j1: int, Y: np.ndarray) -> np.ndarray:
    """(j1 - j0) x cols = X_[j0,j1)^T Y."""
    Yf = np.asfortranarray(Y, dtype=np.float64)
    out = np.empty((j1 - j0, Yf.shape[1]), order="F")
    check(_lib.load().lds_geno_target_product(session.handle, j0, j1, ptr(Yf), Yf.shape[1],
                                              ptr(out)))
    return out


def _component_diagonal(session, j0: int, j1: int, annot_blk, basis, fixed, coef,
                        numerator: np.ndarray) -> None:
    """numerator (K*P x N, C order) += the block's component-kernel diagonals."""
    a = np.ascontiguousarray(annot_blk, dtype=np.float64)
    r_count = fixed.shape[1]
    check(_lib.load().lds_generalized_component_diagonal(
        session.handle, j0, j1, ptr(a), a.shape[1], ptr(basis), basis.shape[1],
        ptr(fixed) if r_count else None, r_count,
        ptr(np.ascontiguousarray(coef)) if r_count else None, ptr(numerator)))


def _pass2_scores(session, rhs, k_count, b_count, f_count, p_count, term_off, term_f1, term_f2,
                  residual_rank, weights, block):
    """(directional M x P x K*P, directed K*P x K*P) of all variants: the
    right-hand side quantized once, the exact products and the per-variant
    orientation products on the device (lds_generalized_pass2)."""
    m, c_count = session.M, k_count * p_count
    directional = np.empty((m, p_count, c_count))
    directed = np.empty((c_count, c_count))
    r = np.asfortranarray(rhs, dtype=np.float64)
    a = np.ascontiguousarray(weights, dtype=np.float64)
    check(_lib.load().lds_generalized_pass2(
        session.handle, ptr(r), k_count, b_count, f_count, p_count, ptr(term_off), ptr(term_f1),
        ptr(term_f2), float(residual_rank), ptr(a), int(block), ptr(directional), ptr(directed)))
    return directional, directed


def _project_sources(base, basis, fixed):
    """Pass 1's projection on the device (lds_generalized_project): the
    contextual sources (K x Q x B x N) of the base sources (K x B x N), and the
    maximum absolute and relative leakage."""
    k_count, b_count, n = base.shape
    q_count, r_count = basis.shape[1], fixed.shape[1]
    out = np.empty((k_count, q_count, b_count, n))
    b_ = np.ascontiguousarray(base, dtype=np.float64)
    q_ = np.ascontiguousarray(basis, dtype=np.float64)
    f_ = np.ascontiguousarray(fixed, dtype=np.float64) if r_count else None
    mabs, mrel = C.c_double(0.0), C.c_double(0.0)
    check(_lib.load().lds_generalized_project(
        ptr(b_), ptr(q_), ptr(f_) if r_count else None, k_count, q_count, b_count, r_count, n,
        ptr(out), C.byref(mabs), C.byref(mrel)))
    return out, mabs.value, mrel.value


def _pass2_scores_sources(session, rows, basis, fam_t, fam_s, k_count, b_count, p_count,
                          term_off, term_f1, term_f2, residual_rank, weights, block):
    """_pass2_scores with the right-hand side formed on the device from the
    sources (K x Q x B x N rows) and the basis (lds_generalized_pass2_sources):
    only they cross PCIe, not the K*B*F columns."""
    m, c_count = session.M, k_count * p_count
    directional = np.empty((m, p_count, c_count))
    directed = np.empty((c_count, c_count))
    src = np.ascontiguousarray(rows, dtype=np.float64)
    bas = np.ascontiguousarray(basis, dtype=np.float64)
    ft = np.ascontiguousarray(fam_t, dtype=np.int32)
    fs = np.ascontiguousarray(fam_s, dtype=np.int32)
    a = np.ascontiguousarray(weights, dtype=np.float64)
    check(_lib.load().lds_generalized_pass2_sources(
        session.handle, ptr(src), int(bas.shape[1]), ptr(bas), ptr(ft), ptr(fs), k_count, b_count,
        len(ft), p_count, ptr(term_off), ptr(term_f1), ptr(term_f2), float(residual_rank), ptr(a),
        int(block), ptr(directional), ptr(directed)))
    return directional, directed


def pair_order(q_count: int) -> tuple[tuple[int, int], ...]:
    """Diagonal-first unordered basis pairs (context/spec.py ContextPairIndex)."""
    return tuple((q, q) for q in range(q_count)) + tuple(
        (q, r) for q in range(q_count - 1) for r in range(q + 1, q_count))


def _orientations(pair):
    q, r = pair
    return ((q, q),) if q == r else ((q, r), (r, q))


def _validate(session, basis, fixed, annotations):
    n, m = session.N, session.M
    basis = np.array(basis, dtype=np.float64, order="F", copy=True)
    fixed = np.array(fixed, dtype=np.float64, order="F", copy=True)
    weights = np.array(annotations, dtype=np.float64, order="C", copy=True)
    if basis.ndim != 2 or basis.shape[0] != n:
        raise ValueError("basis must have shape (N,Q)")
    if fixed.ndim != 2 or fixed.shape[0] != n:
        raise ValueError("fixed_effect_basis must have shape (N,R)")
    if weights.ndim != 2 or weights.shape[0] != m:
        raise ValueError("annotations must have shape (M,K)")
    if not (np.all(np.isfinite(basis)) and np.all(np.isfinite(fixed))
            and np.all(np.isfinite(weights))):
        raise ValueError("basis, fixed effects, and annotations must be finite")
    if np.any(weights < 0.0):
        raise ValueError("annotations must be nonnegative")
    masses = np.sum(weights, axis=0, dtype=np.float64)
    if np.any(masses <= 0.0):
        raise ValueError("annotation masses must be positive and match full annotations")
    if fixed.shape[1]:
        gram = fixed.T @ fixed
        if not np.allclose(gram, np.eye(fixed.shape[1]), rtol=2.0e-13, atol=2.0e-13):
            raise ValueError("fixed_effect_basis must be orthonormal")
    return basis, fixed, weights, masses


@dataclass(frozen=True)
class GeneralizedPass1Result:
    """The fields of GeneralizedGxEPass1Result that pass 2 and callers read."""
    contextual_sources: np.ndarray          # K x Q x N x B
    annotation_masses: np.ndarray
    pair_table: tuple[tuple[int, int], ...]
    component_table: tuple[tuple[int, int], ...]   # (annotation, pair) per component
    maximum_projection_leakage: float
    maximum_relative_projection_leakage: float
    base_sources: np.ndarray | None         # K x N x B when retained


def pass1(session, basis, fixed_effect_basis, annotations, probe_spec: GlobalVariantProbeSpec, *,
          variant_block_width: int = 65536, projection_tolerance: float = 2.0e-11,
          retain_base_sources: bool = False) -> GeneralizedPass1Result:
    """Global contextual sources (GeneralizedGxEPass1Executor.execute)."""
    basis, fixed, weights, masses = _validate(session, basis, fixed_effect_basis, annotations)
    if not np.isfinite(projection_tolerance) or projection_tolerance <= 0.0:
        raise ValueError("projection_tolerance must be positive and finite")
    if variant_block_width < 1:
        raise ValueError("variant_block_width must be positive")
    n, m = session.N, session.M
    k_count, q_count, b_count = weights.shape[1], basis.shape[1], probe_spec.probe_count
    # Sources are kept as B x N rows (the layout the device returns and pass 2
    # reads); the results expose the reference's N x B views.
    base = np.zeros((k_count, b_count, n))
    for j0 in range(0, m, variant_block_width):
        j1 = min(m, j0 + variant_block_width)
        z = global_variant_probes(probe_spec, j0, j1 - j0)
        out = _source_product(session, j0, j1, weights[j0:j1], z)
        base += out.T.reshape(k_count, b_count, n)
    contextual, max_abs, max_rel = _project_sources(base, basis, fixed)
    if max_rel > projection_tolerance:
        raise RuntimeError("contextual source projection leakage exceeds its tolerance")
    contextual = contextual.transpose(0, 1, 3, 2)
    pairs = pair_order(q_count)
    components = tuple((k, p) for k in range(k_count) for p in range(len(pairs)))
    contextual.setflags(write=False)
    return GeneralizedPass1Result(contextual, masses, pairs, components, max_abs, max_rel,
                                  base.transpose(0, 2, 1) if retain_base_sources else None)


@dataclass(frozen=True)
class GeneralizedPass2Result:
    """The numeric fields of GeneralizedGxEPass2Result."""
    directional_ldscores: np.ndarray        # M x P x K*P
    directed_numerator: np.ndarray          # C x C
    symmetric_numerator: np.ndarray
    genetic_gram: np.ndarray
    component_kernel_diagonal: np.ndarray   # C x N
    same_person: np.ndarray                 # C x C
    residual_rank: int
    presymmetry_absolute_error: float
    presymmetry_relative_error: float


def pass2(session, pass1_result: GeneralizedPass1Result, basis, fixed_effect_basis, annotations,
          *, variant_block_width: int = 65536) -> GeneralizedPass2Result:
    """Per-variant directional scores (GeneralizedGxEPass2Executor.execute)."""
    basis, fixed, weights, masses = _validate(session, basis, fixed_effect_basis, annotations)
    sources = pass1_result.contextual_sources
    k_count, q_count, n, b_count = sources.shape
    m = session.M
    if weights.shape[1] != k_count or basis.shape[1] != q_count or n != session.N:
        raise ValueError("pass-1 sources do not match the pass-2 inputs")
    if variant_block_width < 1:
        raise ValueError("variant_block_width must be positive")
    r_count = fixed.shape[1]
    residual_rank = n - r_count
    pairs = pair_order(q_count)
    p_count, c_count = len(pairs), k_count * len(pairs)
    # With P = I, X^T diag(phi_u) diag(phi_v) S is symmetric in (u, v).
    symmetric_cross = r_count == 0
    families = tuple((u, v) for u in range(q_count)
                     for v in range(u if symmetric_cross else 0, q_count))
    f_count = len(families)
    # rhs column (k * B + b) * F + f = phi_t o sources[k, s][:, b] for family
    # f = (t, s), formed on the device from the K x Q x B x N source rows
    rows = np.swapaxes(sources, 2, 3)   # contiguous for pass-1 results
    fam_t = np.array([t for t, _ in families], dtype=np.int32)
    fam_s = np.array([s for _, s in families], dtype=np.int32)
    weighted_fixed = np.asfortranarray(
        (basis[:, :, None] * fixed[:, None, :]).reshape(n, q_count * r_count)) if r_count else None
    # Orientation terms of every (target pair, source pair): products of the
    # cross sketches of families (t_right, s_left) and (t_left, s_right).
    family = {}
    for f, (u, v) in enumerate(families):
        family[(u, v)] = f
        if symmetric_cross:
            family[(v, u)] = f
    term_off, term_f1, term_f2 = [0], [], []
    for target_pair in pairs:
        for source_pair in pairs:
            for tl, tr in _orientations(target_pair):
                for sl, sr in _orientations(source_pair):
                    term_f1.append(family[(tr, sl)])
                    term_f2.append(family[(tl, sr)])
            term_off.append(len(term_f1))
    diag_num = np.zeros((c_count, n))
    for j0 in range(0, m, variant_block_width):
        j1 = min(m, j0 + variant_block_width)
        coef = None
        if r_count:
            cf = _target_product(session, j0, j1, weighted_fixed)
            coef = np.ascontiguousarray(cf.reshape(j1 - j0, q_count, r_count))
        _component_diagonal(session, j0, j1, weights[j0:j1], basis, fixed, coef, diag_num)
    directional, directed = _pass2_scores_sources(
        session, rows, basis, fam_t, fam_s, k_count, b_count, p_count,
        np.asarray(term_off, np.int32), np.asarray(term_f1, np.int32),
        np.asarray(term_f2, np.int32), float(residual_rank), weights, variant_block_width)
    if not np.all(np.isfinite(directional)):
        raise RuntimeError("per-variant directional scores are non-finite")
    pre_abs = float(np.max(np.abs(directed - directed.T), initial=0.0))
    pre_rel = pre_abs / max(1.0, float(np.max(np.abs(directed), initial=0.0)))
    symmetric = 0.5 * (directed + directed.T)
    comp_annot = np.repeat(np.arange(k_count), p_count)
    comp_masses = masses[comp_annot]
    kernel_diag = diag_num / comp_masses[:, None]
    same_raw = kernel_diag @ kernel_diag.T
    same_person = 0.5 * (same_raw + same_raw.T)
    gram = float(residual_rank ** 2) * symmetric / (comp_masses[:, None] * comp_masses[None, :])
    for name, value in (("directional_ldscores", directional), ("directed_numerator", directed),
                        ("genetic_gram", gram), ("component_kernel_diagonal", kernel_diag),
                        ("same_person", same_person)):
        if not np.all(np.isfinite(value)):
            raise RuntimeError(f"{name} is non-finite after pass 2")
    return GeneralizedPass2Result(directional, directed, symmetric, gram, kernel_diag,
                                  same_person, int(residual_rank), pre_abs, pre_rel)


def two_pass(session, basis, fixed_effect_basis, annotations, probe_spec: GlobalVariantProbeSpec,
             *, variant_block_width: int = 65536, projection_tolerance: float = 2.0e-11):
    """Both passes; returns (pass-1 result, pass-2 result)."""
    p1 = pass1(session, basis, fixed_effect_basis, annotations, probe_spec,
               variant_block_width=variant_block_width,
               projection_tolerance=projection_tolerance)
    return p1, pass2(session, p1, basis, fixed_effect_basis, annotations,
                     variant_block_width=variant_block_width)
