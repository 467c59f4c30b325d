"""Drop-in replacement for SUMMIT's native ``gwldcore`` module, backed by liblds.so.

Function names, keyword arguments, defaults, array layouts and error messages
follow the reference's nanobind bindings (``src/native/gwldcore.cpp:3656-3829``),
so ``summit.ldscore.gw_ldscore`` can import this module in place of the native
one.  The ``float32`` / ``float64`` overloads are selected from the dtype of the
sketch array, as nanobind's overload resolution does.

All genotype arithmetic runs on the GPU (sm_100a).  There is no CPU fallback:
without liblds.so or a CUDA device every compute call raises RuntimeError.

In addition to the reference's per-block functions, ``gw_ldscore`` computes a
whole genome-wide estimate in one call with the genotype image resident on
the device (same probes, blocks and V-tiles, hence the same result).
"""
from __future__ import annotations

import numpy as np

from . import _lib
from ._lib import check, enc, ptr

_REQUIRED = object()
_verbose = False


def _need(name, value):
    if value is _REQUIRED:
        raise TypeError(f"missing required argument '{name}'")
    return value


def _tsuffix(arr) -> str:
    if arr.dtype == np.float32:
        return "f32"
    if arr.dtype == np.float64:
        return "f64"
    raise TypeError("incompatible function arguments: arrays must be float32 or float64")


def _rows(row_sel):
    if row_sel is None:
        return None, 0
    r = np.asarray(row_sel)
    if r.ndim != 1 or r.dtype not in (np.int32, np.int64):
        raise RuntimeError("row_sel must be a 1D CPU array of int32 or int64 indices")
    r = np.ascontiguousarray(r, dtype=np.int64)
    return r, int(r.size)


def _rw(arr, dtype, order, name):
    """In-place arrays must already have the right dtype and layout."""
    if not isinstance(arr, np.ndarray) or arr.dtype != dtype:
        raise TypeError(f"incompatible function arguments: {name} must be a {np.dtype(dtype)} array")
    ok = arr.flags.f_contiguous if order == "F" else arr.flags.c_contiguous
    if not ok or not arr.flags.writeable:
        raise TypeError(f"incompatible function arguments: {name} must be writable and "
                        f"{'column' if order == 'F' else 'row'}-major contiguous")
    return arr


def _cov(C, R, dt, gram=None):
    """Covariate basis C (N x p) and R (p x N) as column-major arrays of dtype dt."""
    if C is None or R is None:
        if (C is None) != (R is None):
            raise RuntimeError("C and R must be provided together for fused residual variances")
        return None, None, 0, None
    Cf = np.asfortranarray(C, dtype=dt)
    Rf = np.asfortranarray(R, dtype=dt)
    p = Cf.shape[1]
    if Rf.shape != (p, Cf.shape[0]):
        raise RuntimeError("C/R shape mismatch in fused residual variances")
    G = None
    if gram is not None:
        G = np.ascontiguousarray(gram, dtype=dt)
        if G.shape != (p, p):
            raise RuntimeError("covariate Gram shape mismatch in fused residual variances")
    return Cf, Rf, p, G


def _impute(mode: str) -> int:
    if mode not in _lib.LDS_IMPUTE:
        raise RuntimeError("impute_mode must be 'mean' or 'hwe'")
    return _lib.LDS_IMPUTE[mode]


def _dist(name: str) -> int:
    # The reference treats any non-"rademacher" name as Gaussian, with
    # "spherical" rescaled (gwldcore.cpp:1693-1716).
    if name == "rademacher":
        return 0
    return 2 if name == "spherical" else 1


# ---------------------------------------------------------------------------
# Housekeeping (gwldcore.cpp:3659-3671, :3742-3746)
# ---------------------------------------------------------------------------
def set_verbose(enabled: bool) -> None:
    global _verbose
    _verbose = bool(enabled)


def set_num_threads(n: int) -> None:
    """Host threads are not used for genotype arithmetic; accepted for API parity."""


def get_max_threads() -> int:
    return 1


def prefetch_bed_block(bed_prefix, fam_path, blk_start, blk_end, ahead_blocks=1) -> None:
    """The genotype image is resident on the device after first use; nothing to prefetch."""


def clear_gwld_native_scratch() -> None:
    _lib.load().lds_clear_device_cache()


clear_phase1_native_scratch = clear_gwld_native_scratch
clear_phase2_native_scratch = clear_gwld_native_scratch
clear_gwld_genotype_scratch = clear_gwld_native_scratch
_clear_bed_mapping_cache = clear_gwld_native_scratch


def clear_phase1_csr_cache() -> None:
    """CSR lists are rebuilt per call from the arrays passed; nothing is cached."""


def _bed_mapping_cache_info() -> dict:
    return {"entries": 0, "capacity": 2, "hits": 0, "misses": 0, "evictions": 0}


# ---------------------------------------------------------------------------
# Phase 1 (gwldcore.cpp:3673-3688)
# ---------------------------------------------------------------------------
def phase1_compute_Xz_bed_chunk(bed_prefix, fam_path, blk_start, blk_end, row_sel=None, ddof=1,
                                annot_blk=_REQUIRED, inv_right=_REQUIRED, v_start=_REQUIRED,
                                v_count=_REQUIRED, kmax_hint=_REQUIRED, rand_dist="rademacher",
                                seed=None, Xz2d_chunk=_REQUIRED, bin_init_mask=None,
                                project_right=False, C=None, R=None, impute_mode="hwe",
                                impute_seed=None, resvar_gram=None, inv_out=None,
                                resvar_eps=1e-10):
    Xz = _need("Xz2d_chunk", Xz2d_chunk)
    t = _tsuffix(Xz)
    dt = Xz.dtype
    _rw(Xz, dt, "F", "Xz2d_chunk")
    if Xz.ndim != 2:
        raise RuntimeError("Xz2d_chunk shape must be (N, B*v_count)")
    if inv_out is not None:
        Cf, Rf, p, G = _cov(C, R, dt, resvar_gram)
    elif project_right:
        Cf, Rf, p = _cr(C, R, dt, Xz.shape[0], "phase1")
        G = None
    else:
        Cf, Rf, p, G = None, None, 0, None
    ann = np.ascontiguousarray(_need("annot_blk", annot_blk), dtype=dt)
    if ann.ndim != 2:
        raise RuntimeError("L mismatch")
    inv_r = None
    if inv_out is not None:
        _rw(inv_out, dt, "C", "inv_out")
        if inv_out.shape[0] != ann.shape[0]:
            raise RuntimeError("inv_out shape mismatch in phase1 fused residual variance")
    else:
        inv_r = np.ascontiguousarray(_need("inv_right", inv_right), dtype=dt)
        if inv_r.shape[0] != ann.shape[0]:
            raise RuntimeError("inv_right shape mismatch in phase1")
    if bin_init_mask is not None:
        _rw(bin_init_mask, np.uint8, "C", "bin_init_mask")
        if bin_init_mask.shape[0] != ann.shape[1]:
            raise RuntimeError("bin_init_mask shape mismatch in phase1")
    rows, nr = _rows(row_sel)
    fn = getattr(_lib.load(), f"lds_phase1_compute_Xz_bed_chunk_{t}")
    check(fn(enc(bed_prefix), enc(fam_path), int(blk_start), int(blk_end), ptr(rows), nr,
             int(ddof), ptr(ann), ann.shape[0], ann.shape[1], ptr(inv_r), int(_need("v_start", v_start)),
             int(_need("v_count", v_count)), int(_need("kmax_hint", kmax_hint)), _dist(rand_dist),
             int(seed is not None), 0 if seed is None else int(seed) & (2**64 - 1), ptr(Xz),
             Xz.shape[0], Xz.shape[1], ptr(bin_init_mask), _impute(impute_mode),
             int(impute_seed is not None), 0 if impute_seed is None else int(impute_seed),
             ptr(inv_out), float(resvar_eps), ptr(Cf), ptr(Rf), p, ptr(G), int(bool(project_right))))


def phase1_compute_Xz_geno_chunk(Geno, blk_start, annot_blk=_REQUIRED, inv_right=_REQUIRED,
                                 v_start=_REQUIRED, v_count=_REQUIRED, kmax_hint=_REQUIRED,
                                 rand_dist="rademacher", seed=None, Xz2d_chunk=_REQUIRED,
                                 bin_init_mask=None, C=None, R=None, resvar_gram=None,
                                 inv_out=None, resvar_eps=1e-10):
    """Phase 1 from a dense standardized genotype block (gwldcore.cpp:3690-3701)."""
    t = _tsuffix(Geno)
    dt = Geno.dtype
    G = _rw(Geno, dt, "F", "Geno")
    Xz = _rw(_need("Xz2d_chunk", Xz2d_chunk), dt, "F", "Xz2d_chunk")
    ann = np.ascontiguousarray(_need("annot_blk", annot_blk), dtype=dt)
    if ann.ndim != 2:
        raise RuntimeError("L mismatch")
    Cf, Rf, p, Gr = (None, None, 0, None)
    inv_r = None
    if inv_out is not None:
        _rw(inv_out, dt, "C", "inv_out")
        if inv_out.shape[0] != G.shape[1]:
            raise RuntimeError("inv_out shape mismatch in phase1 fused residual variance")
        Cf, Rf, p, Gr = _cov(C, R, dt, resvar_gram)
        if p and Cf.shape[0] != G.shape[0]:
            raise RuntimeError("C/R shape mismatch in fused residual variances")
    else:
        inv_r = np.ascontiguousarray(_need("inv_right", inv_right), dtype=dt)
        if inv_r.shape[0] != G.shape[1]:
            raise RuntimeError("inv_right shape mismatch in phase1")
    if bin_init_mask is not None:
        _rw(bin_init_mask, np.uint8, "C", "bin_init_mask")
        if bin_init_mask.shape[0] != ann.shape[1]:
            raise RuntimeError("bin_init_mask shape mismatch in phase1")
    fn = getattr(_lib.load(), f"lds_phase1_compute_Xz_geno_chunk_{t}")
    check(fn(ptr(G), G.shape[0], G.shape[1], int(blk_start), ptr(ann), ann.shape[0], ann.shape[1],
             ptr(inv_r), int(_need("v_start", v_start)), int(_need("v_count", v_count)),
             int(_need("kmax_hint", kmax_hint)), _dist(rand_dist), int(seed is not None),
             0 if seed is None else int(seed) & (2**64 - 1), ptr(Xz), Xz.shape[0], Xz.shape[1],
             ptr(bin_init_mask), ptr(Cf), ptr(Rf), p, ptr(Gr), ptr(inv_out), float(resvar_eps)))


# ---------------------------------------------------------------------------
# Phase 2 (gwldcore.cpp:3759-3770)
# ---------------------------------------------------------------------------
def phase2_accum_XtXz_bed(bed_prefix, fam_path, blk_start, blk_end, row_sel=None, ddof=1,
                          inv_left=_REQUIRED, tile_nvecs=_REQUIRED, Xz2d=_REQUIRED,
                          meansq_accum=_REQUIRED, C=None, R=None, N_denom=0, impute_mode="hwe",
                          impute_seed=None, mc_aggregate_sumsq=None, mc_per_snp_sumsq=None):
    ms = _need("meansq_accum", meansq_accum)
    t = _tsuffix(ms)
    dt = ms.dtype
    _rw(ms, dt, "C", "meansq_accum")
    Xz = np.asfortranarray(_need("Xz2d", Xz2d), dtype=dt)
    inv = np.ascontiguousarray(_need("inv_left", inv_left), dtype=dt)
    if ms.ndim != 2:
        raise RuntimeError("meansq_accum shape mismatch in phase2_accum_XtXz_bed")
    if mc_aggregate_sumsq is not None:
        _rw(mc_aggregate_sumsq, np.float64, "C", "mc_aggregate_sumsq")
        if mc_aggregate_sumsq.shape[0] != ms.shape[1]:
            raise RuntimeError("mc_aggregate_sumsq length must equal the annotation count")
    if mc_per_snp_sumsq is not None:
        _rw(mc_per_snp_sumsq, np.float64, "C", "mc_per_snp_sumsq")
        if mc_per_snp_sumsq.shape != ms.shape:
            raise RuntimeError("mc_per_snp_sumsq shape must match meansq_accum")
    Cf, Rf, p = _cr(C, R, dt, Xz.shape[0], "phase2_accum_XtXz_bed")
    rows, nr = _rows(row_sel)
    fn = getattr(_lib.load(), f"lds_phase2_accum_XtXz_bed_{t}")
    check(fn(enc(bed_prefix), enc(fam_path), int(blk_start), int(blk_end), ptr(rows), nr,
             int(ddof), ptr(inv), inv.shape[0], int(_need("tile_nvecs", tile_nvecs)), ptr(Xz),
             Xz.shape[0], Xz.shape[1], ptr(ms), ms.shape[0], ms.shape[1], int(N_denom),
             _impute(impute_mode), int(impute_seed is not None),
             0 if impute_seed is None else int(impute_seed), ptr(mc_aggregate_sumsq),
             ptr(mc_per_snp_sumsq), ptr(Cf), ptr(Rf), p))


def phase2_accum_XtXz_geno(Geno, blk_start, inv_left=_REQUIRED, tile_nvecs=_REQUIRED,
                           Xz2d=_REQUIRED, meansq_accum=_REQUIRED, C=None, R=None, N_denom=0,
                           mc_aggregate_sumsq=None, mc_per_snp_sumsq=None):
    """Phase 2 from a dense standardized genotype block (gwldcore.cpp:3772-3783);
    with C and R the block is projected in place, as the reference does."""
    t = _tsuffix(Geno)
    dt = Geno.dtype
    G = _rw(Geno, dt, "F", "Geno")
    ms = _rw(_need("meansq_accum", meansq_accum), dt, "C", "meansq_accum")
    Xz = np.asfortranarray(_need("Xz2d", Xz2d), dtype=dt)
    inv = np.ascontiguousarray(_need("inv_left", inv_left), dtype=dt)
    if ms.ndim != 2:
        raise RuntimeError("meansq_accum shape mismatch in phase2_accum_XtXz_bed")
    if mc_aggregate_sumsq is not None:
        _rw(mc_aggregate_sumsq, np.float64, "C", "mc_aggregate_sumsq")
        if mc_aggregate_sumsq.shape[0] != ms.shape[1]:
            raise RuntimeError("mc_aggregate_sumsq length must equal the annotation count")
    if mc_per_snp_sumsq is not None:
        _rw(mc_per_snp_sumsq, np.float64, "C", "mc_per_snp_sumsq")
        if mc_per_snp_sumsq.shape != ms.shape:
            raise RuntimeError("mc_per_snp_sumsq shape must match meansq_accum")
    Cf, Rf, p = _cr(C, R, dt, G.shape[0], "phase2_accum_XtXz_bed")
    fn = getattr(_lib.load(), f"lds_phase2_accum_XtXz_geno_{t}")
    check(fn(ptr(G), G.shape[0], G.shape[1], int(blk_start), ptr(inv), inv.shape[0],
             int(_need("tile_nvecs", tile_nvecs)), ptr(Xz), Xz.shape[0], Xz.shape[1], ptr(ms),
             ms.shape[0], ms.shape[1], ptr(Cf), ptr(Rf), p, int(N_denom), ptr(mc_aggregate_sumsq),
             ptr(mc_per_snp_sumsq)))


def phase2_compute_XtXz_bed(bed_prefix, fam_path, blk_start, blk_end, row_sel=None, ddof=1,
                            inv_left=_REQUIRED, nvecs=_REQUIRED, vchunk=_REQUIRED, Xz2d=_REQUIRED,
                            meansq=_REQUIRED, C=None, R=None, N_denom=0, impute_mode="hwe",
                            impute_seed=None):
    """Legacy direct phase 2 (gwldcore.cpp:3731-3740): meansq += the update / nvecs."""
    _need("vchunk", vchunk)
    ms = _need("meansq", meansq)
    t = _tsuffix(ms)
    dt = ms.dtype
    _rw(ms, dt, "C", "meansq")
    Xz = np.asfortranarray(_need("Xz2d", Xz2d), dtype=dt)
    inv = np.ascontiguousarray(_need("inv_left", inv_left), dtype=dt)
    if ms.ndim != 2:
        raise RuntimeError("meansq shape mismatch")
    Cf, Rf, p = _cr(C, R, dt, Xz.shape[0], "phase2_compute_XtXz_bed")
    rows, nr = _rows(row_sel)
    fn = getattr(_lib.load(), f"lds_phase2_compute_XtXz_bed_{t}")
    check(fn(enc(bed_prefix), enc(fam_path), int(blk_start), int(blk_end), ptr(rows), nr,
             int(ddof), ptr(inv), inv.shape[0], int(_need("nvecs", nvecs)), ptr(Xz), Xz.shape[0],
             Xz.shape[1], ptr(ms), ms.shape[0], ms.shape[1], ptr(Cf), ptr(Rf), p, int(N_denom),
             _impute(impute_mode), int(impute_seed is not None),
             0 if impute_seed is None else int(impute_seed)))


# ---------------------------------------------------------------------------
# Row-major phase 1, Mailman phase 2, sketch sums and projections
# (gwldcore.cpp:3703-3729, :3785-3805)
# ---------------------------------------------------------------------------
def phase1_compute_Xz_bed_chunk_rowmajor(bed_prefix, fam_path, blk_start, blk_end, row_sel=None,
                                         ddof=1, annot_blk=_REQUIRED, inv_right=_REQUIRED,
                                         v_start=_REQUIRED, v_count=_REQUIRED,
                                         kmax_hint=_REQUIRED, rand_dist="rademacher", seed=None,
                                         Xz2d_chunk=_REQUIRED, project_right=False, C=None, R=None,
                                         impute_mode="hwe", impute_seed=None, resvar_gram=None,
                                         inv_out=None, resvar_eps=1e-10):
    Xz = _need("Xz2d_chunk", Xz2d_chunk)
    t = _tsuffix(Xz)
    dt = Xz.dtype
    _rw(Xz, dt, "C", "Xz2d_chunk")
    if Xz.ndim != 2:
        raise RuntimeError("Xz2d_chunk shape must be (N, B*v_count)")
    if project_right:
        raise RuntimeError("project_right is not supported by the B200 backend; project Xz2d "
                           "after phase 1 (project_rowmajor_inplace_and_col_sums)")
    Cf, Rf, p, G = _cov(C, R, dt, resvar_gram) if inv_out is not None else (None, None, 0, None)
    ann = np.ascontiguousarray(_need("annot_blk", annot_blk), dtype=dt)
    inv_r = None
    if inv_out is not None:
        _rw(inv_out, dt, "C", "inv_out")
    else:
        inv_r = np.ascontiguousarray(_need("inv_right", inv_right), dtype=dt)
        if inv_r.shape[0] != ann.shape[0]:
            raise RuntimeError("inv_right shape mismatch in phase1")
    rows, nr = _rows(row_sel)
    fn = getattr(_lib.load(), f"lds_phase1_compute_Xz_bed_chunk_rowmajor_{t}")
    check(fn(enc(bed_prefix), enc(fam_path), int(blk_start), int(blk_end), ptr(rows), nr,
             int(ddof), ptr(ann), ann.shape[0], ann.shape[1], ptr(inv_r),
             int(_need("v_start", v_start)), int(_need("v_count", v_count)),
             int(_need("kmax_hint", kmax_hint)), _dist(rand_dist), int(seed is not None),
             0 if seed is None else int(seed) & (2**64 - 1), ptr(Xz), Xz.shape[0], Xz.shape[1],
             _impute(impute_mode), int(impute_seed is not None),
             0 if impute_seed is None else int(impute_seed), ptr(inv_out), float(resvar_eps),
             ptr(Cf), ptr(Rf), p, ptr(G)))


def _mailman_common(meansq_accum, Xz2d, order, inv_left, mc_aggregate_sumsq, mc_per_snp_sumsq,
                    name):
    ms = _need("meansq_accum", meansq_accum)
    t = _tsuffix(ms)
    dt = ms.dtype
    _rw(ms, dt, "C", "meansq_accum")
    Xz = _need("Xz2d", Xz2d)
    Xz = np.asfortranarray(Xz, dtype=dt) if order == "F" else np.ascontiguousarray(Xz, dtype=dt)
    inv = np.ascontiguousarray(_need("inv_left", inv_left), dtype=dt)
    if mc_aggregate_sumsq is not None:
        _rw(mc_aggregate_sumsq, np.float64, "C", "mc_aggregate_sumsq")
    if mc_per_snp_sumsq is not None:
        _rw(mc_per_snp_sumsq, np.float64, "C", "mc_per_snp_sumsq")
        if mc_per_snp_sumsq.shape != ms.shape:
            raise RuntimeError(f"mc_per_snp_sumsq shape must match meansq_accum in {name}")
    return t, ms, Xz, inv


def phase2_accum_XtXz_bed_mailman(bed_prefix, fam_path, blk_start, blk_end, row_sel=None, ddof=1,
                                  inv_left=_REQUIRED, tile_nvecs=_REQUIRED, Xz2d=_REQUIRED,
                                  meansq_accum=_REQUIRED, C=None, R=None, N_denom=0,
                                  impute_seed=None, mc_aggregate_sumsq=None,
                                  mc_per_snp_sumsq=None):
    t, ms, Xz, inv = _mailman_common(meansq_accum, Xz2d, "F", inv_left, mc_aggregate_sumsq,
                                     mc_per_snp_sumsq, "phase2_accum_XtXz_bed_mailman")
    Cf, Rf, p = _cr(C, R, ms.dtype, Xz.shape[0], "phase2_accum_XtXz_bed_mailman")
    rows, nr = _rows(row_sel)
    fn = getattr(_lib.load(), f"lds_phase2_accum_XtXz_bed_mailman_{t}")
    check(fn(enc(bed_prefix), enc(fam_path), int(blk_start), int(blk_end), ptr(rows), nr,
             int(ddof), ptr(inv), inv.shape[0], int(_need("tile_nvecs", tile_nvecs)), ptr(Xz),
             Xz.shape[0], Xz.shape[1], ptr(ms), ms.shape[0], ms.shape[1], int(N_denom),
             int(impute_seed is not None), 0 if impute_seed is None else int(impute_seed),
             ptr(mc_aggregate_sumsq), ptr(mc_per_snp_sumsq), ptr(Cf), ptr(Rf), p))


def phase2_accum_XtXz_bed_mailman_rowmajor(bed_prefix, fam_path, blk_start, blk_end,
                                           row_sel=None, ddof=1, inv_left=_REQUIRED,
                                           tile_nvecs=_REQUIRED, Xz2d=_REQUIRED,
                                           meansq_accum=_REQUIRED, sum_Xz=_REQUIRED, N_denom=0,
                                           impute_seed=None, mc_aggregate_sumsq=None,
                                           mc_per_snp_sumsq=None):
    t, ms, Xz, inv = _mailman_common(meansq_accum, Xz2d, "C", inv_left, mc_aggregate_sumsq,
                                     mc_per_snp_sumsq, "phase2_accum_XtXz_bed_mailman_rowmajor")
    sx = np.ascontiguousarray(_need("sum_Xz", sum_Xz), dtype=np.float64)
    rows, nr = _rows(row_sel)
    fn = getattr(_lib.load(), f"lds_phase2_accum_XtXz_bed_mailman_rowmajor_{t}")
    check(fn(enc(bed_prefix), enc(fam_path), int(blk_start), int(blk_end), ptr(rows), nr,
             int(ddof), ptr(inv), inv.shape[0], int(_need("tile_nvecs", tile_nvecs)), ptr(Xz),
             Xz.shape[0], Xz.shape[1], ptr(ms), ms.shape[0], ms.shape[1], ptr(sx), sx.size,
             int(N_denom), int(impute_seed is not None),
             0 if impute_seed is None else int(impute_seed), ptr(mc_aggregate_sumsq),
             ptr(mc_per_snp_sumsq)))


def compute_col_sums_rowmajor(Xz2d) -> np.ndarray:
    X = np.asarray(Xz2d)
    t = _tsuffix(X)
    X = np.ascontiguousarray(X)
    out = np.empty(X.shape[1])
    check(getattr(_lib.load(), f"lds_compute_col_sums_rowmajor_{t}")(ptr(X), X.shape[0],
                                                                       X.shape[1], ptr(out)))
    return out


def _cr(C, R, dt, N, name):
    if C is None or R is None:
        return None, None, 0
    Cf = np.asfortranarray(C, dtype=dt)
    Rf = np.asfortranarray(R, dtype=dt)
    p = Cf.shape[1]
    if Cf.shape[0] != N or Rf.shape != (p, N):
        raise RuntimeError(f"C/R shape mismatch in {name}")
    return Cf, Rf, p


def project_rowmajor_inplace_and_col_sums(Xz2d, C=None, R=None) -> np.ndarray:
    t = _tsuffix(Xz2d)
    X = _rw(Xz2d, Xz2d.dtype, "C", "Xz2d")
    Cf, Rf, p = _cr(C, R, X.dtype, X.shape[0], "project_rowmajor_inplace_and_col_sums")
    sums = np.empty(X.shape[1])
    check(getattr(_lib.load(), f"lds_project_rowmajor_inplace_and_col_sums_{t}")(
        ptr(X), X.shape[0], X.shape[1], ptr(Cf), ptr(Rf), p, ptr(sums)))
    return sums


def project_colmajor_inplace(Xz2d, C=None, R=None) -> None:
    t = _tsuffix(Xz2d)
    X = _rw(Xz2d, Xz2d.dtype, "F", "Xz2d")
    Cf, Rf, p = _cr(C, R, X.dtype, X.shape[0], "project_colmajor_inplace")
    if p == 0:
        return
    check(getattr(_lib.load(), f"lds_project_colmajor_inplace_{t}")(
        ptr(X), X.shape[0], X.shape[1], ptr(Cf), ptr(Rf), p))


def standardize_dosage_inplace(Geno, ddof=1, missing_value=-9.0, num_threads=0) -> int:
    t = _tsuffix(Geno)
    G = _rw(Geno, Geno.dtype, "F", "Geno")
    n = np.zeros(1, dtype=np.int64)
    check(getattr(_lib.load(), f"lds_standardize_dosage_inplace_{t}")(
        ptr(G), G.shape[0], G.shape[1], int(ddof), float(missing_value), ptr(n)))
    return int(n[0])


# ---------------------------------------------------------------------------
# Residual variances (gwldcore.cpp:3748-3757)
# ---------------------------------------------------------------------------
def precompute_residual_variances_bed(bed_prefix, fam_path, nsnps, step_size, row_sel=None,
                                      ddof=1, eps=1e-10, compute_mu22=False, annot_all=None,
                                      C=None, R=None, impute_mode="hwe", impute_seed=None,
                                      snp_var_out=None, dtype=np.float64):
    # dtype selects the overload; an annotation or covariate array decides it
    # when given, as the typed arrays do for the reference's two overloads
    for a in (annot_all, C):
        if isinstance(a, np.ndarray) and a.dtype in (np.float32, np.float64):
            dtype = a.dtype
            break
    t = "f32" if np.dtype(dtype) == np.float32 else "f64"
    dt = np.float32 if t == "f32" else np.float64
    out = np.empty(int(nsnps), dtype=dt)
    if C is not None and R is not None:
        Cf = np.asfortranarray(C, dtype=dt)
        Rf = np.asfortranarray(R, dtype=dt)
        p = Cf.shape[1]
        if Rf.shape != (p, Cf.shape[0]):
            raise RuntimeError("C/R shape mismatch in precompute_residual_variances_bed")
    else:
        Cf = Rf = None
        p = 0
    if snp_var_out is not None:
        _rw(snp_var_out, np.float64, "C", "snp_var_out")
        if snp_var_out.shape[0] != int(nsnps):
            raise RuntimeError("snp_var_out shape mismatch in precompute_residual_variances_bed")
    ann, B, mu22 = None, 0, None
    if compute_mu22:
        if annot_all is None:
            raise RuntimeError("annot_all must be provided when compute_mu22=True")
        ann = np.ascontiguousarray(annot_all, dtype=dt)
        if ann.ndim != 2 or ann.shape[0] != int(nsnps):
            raise RuntimeError("annot_all shape mismatch in precompute_residual_variances_bed")
        B = ann.shape[1]
        mu22 = np.zeros((B, B))
    rows, nr = _rows(row_sel)
    fn = getattr(_lib.load(), f"lds_precompute_residual_variances_bed_{t}")
    check(fn(enc(bed_prefix), enc(fam_path), int(nsnps), int(step_size), ptr(rows), nr, int(ddof),
             float(eps), _impute(impute_mode), int(impute_seed is not None),
             0 if impute_seed is None else int(impute_seed), ptr(out), ptr(Cf), ptr(Rf), p,
             ptr(snp_var_out), int(bool(compute_mu22)), ptr(ann),
             0 if ann is None else ann.shape[0], B, ptr(mu22)))
    return out, mu22


def compute_block_corrections_binary(meansq_raw, mu22, annot_all, N, d):
    """R2, rho2, bias and delta (B x B each) of binary annotations
    (gwldcore.cpp:3807-3810, impl :3569-3627)."""
    A = np.asarray(annot_all)
    t = _tsuffix(A)
    A = np.ascontiguousarray(A)
    m = np.ascontiguousarray(meansq_raw, dtype=np.float64)
    u = np.ascontiguousarray(mu22, dtype=np.float64)
    M, B = m.shape
    if u.shape != (B, B):
        raise RuntimeError("mu22 shape mismatch")
    if A.shape != (M, B):
        raise RuntimeError("annot_all shape mismatch")
    out = [np.zeros((B, B)) for _ in range(4)]
    check(getattr(_lib.load(), f"lds_compute_block_corrections_binary_{t}")(
        ptr(m), M, B, ptr(u), ptr(A), int(N), float(d), *[ptr(o) for o in out]))
    return tuple(out)


def _grm(name, bed_prefix, fam_path, nsnps, step_size, row_sel, ddof, inv_all, panel_in,
         panel_out, C, R):
    pout = _need("panel_out", panel_out)
    t = _tsuffix(pout)
    dt = pout.dtype
    _rw(pout, dt, "F", "panel_out")
    pin = np.asfortranarray(_need("panel_in", panel_in), dtype=dt)
    inv = np.ascontiguousarray(_need("inv_all", inv_all), dtype=dt)
    if pin.shape[0] != pout.shape[0]:
        raise RuntimeError(f"panel row mismatch in {name}")
    if pin.shape[1] != pout.shape[1]:
        raise RuntimeError(f"panel col mismatch in {name}")
    Cf, Rf, p = _cr(C, R, dt, pin.shape[0], name)
    rows, nr = _rows(row_sel)
    head = (enc(bed_prefix), enc(fam_path), int(nsnps), int(step_size), ptr(rows), nr, int(ddof),
            ptr(inv), inv.shape[0], ptr(pin), ptr(pout), pin.shape[0], pin.shape[1], ptr(Cf),
            ptr(Rf), p)
    return head, getattr(_lib.load(), f"lds_{name}_{t}")


def apply_grm_bed_panel(bed_prefix, fam_path, nsnps, step_size, row_sel=None, ddof=1,
                        inv_all=_REQUIRED, panel_in=_REQUIRED, panel_out=_REQUIRED, C=None,
                        R=None, impute_mode="hwe", impute_seed=None) -> None:
    """panel_out = P X D X^T P panel_in (gwldcore.cpp:3812-3820)."""
    head, fn = _grm("apply_grm_bed_panel", bed_prefix, fam_path, nsnps, step_size, row_sel, ddof,
                    inv_all, panel_in, panel_out, C, R)
    check(fn(*head, _impute(impute_mode), int(impute_seed is not None),
             0 if impute_seed is None else int(impute_seed)))


def apply_grm_bed_panel_mailman(bed_prefix, fam_path, nsnps, step_size, row_sel=None, ddof=1,
                                inv_all=_REQUIRED, panel_in=_REQUIRED, panel_out=_REQUIRED,
                                C=None, R=None, impute_seed=None) -> None:
    """Mailman form on HWE-completed genotypes (gwldcore.cpp:3821-3828)."""
    head, fn = _grm("apply_grm_bed_panel_mailman", bed_prefix, fam_path, nsnps, step_size,
                    row_sel, ddof, inv_all, panel_in, panel_out, C, R)
    check(fn(*head, int(impute_seed is not None),
             0 if impute_seed is None else int(impute_seed)))


# ---------------------------------------------------------------------------
# Whole-estimator entry (no reference counterpart as a single call; it fuses
# the per-block loop of gw_ldscore.py:1753-2222).
# ---------------------------------------------------------------------------
def gw_ldscore(bed_rows, n_total, annot, nvecs, step_size, seed, rand_dist="rademacher",
               vtile=None, ddof=1, impute_mode="mean", impute_seed=0, eps=1e-10,
               dtype=np.float64, row_sel=None, with_mc=False):
    """Genome-wide (partitioned) LD scores from an in-memory BED image.

    ``bed_rows``: (M, row_bytes) uint8 SNP-major packed rows (no header).
    ``annot``: (M, K) annotation matrix.  Returns a dict with ``ldscore``,
    ``meansq_accum``, ``inv`` and, with ``with_mc``, the MC fourth-moment sums.
    """
    bed_rows = np.ascontiguousarray(bed_rows, dtype=np.uint8)
    M, row_bytes = bed_rows.shape
    annot = np.ascontiguousarray(annot, dtype=np.float64)
    K = annot.shape[1]
    ld = np.empty((M, K))
    ms = np.empty((M, K))
    inv = np.empty(M)
    mca = np.empty(K) if with_mc else None
    mcp = np.empty((M, K)) if with_mc else None
    rows, nr = _rows(row_sel)
    lib = _lib.load()
    check(lib.lds_gw_ldscore(ptr(bed_rows), row_bytes, int(n_total), M, ptr(rows), nr, ptr(annot),
                             K, int(nvecs), int(step_size), int(vtile or 0), int(seed),
                             _dist(rand_dist), int(ddof), _impute(impute_mode), int(impute_seed),
                             float(eps), int(np.dtype(dtype) == np.float32), ptr(ld), ptr(ms),
                             ptr(inv), ptr(mca), ptr(mcp)))
    return {"ldscore": ld, "meansq_accum": ms, "inv": inv, "mc_aggregate_sumsq": mca,
            "mc_per_snp_sumsq": mcp}


def last_timings() -> dict:
    """Device times (ms) of the last gw_ldscore call."""
    buf = np.zeros(4)
    _lib.load().lds_last_timings(ptr(buf), 4)
    return {"prepare_ms": buf[0], "phase1_ms": buf[1], "phase2_ms": buf[2], "total_ms": buf[3]}


def debug_xt_products(bed_rows, n, y):
    """Exact int64 (G^T y, O^T y) from the tensor-core kernel (verification)."""
    bed_rows = np.ascontiguousarray(bed_rows, dtype=np.uint8)
    y = np.asfortranarray(y, dtype=np.int8)
    L = bed_rows.shape[0]
    Q = y.shape[1]
    g = np.empty((L, Q), dtype=np.int64)
    o = np.empty((L, Q), dtype=np.int64)
    check(_lib.load().lds_debug_xt_products(ptr(bed_rows), bed_rows.shape[1], int(n), L, ptr(y), Q,
                                            ptr(g), ptr(o)))
    return g, o


def debug_xt_products_umma(bed_rows, n, y4):
    """Exact Horner-combined int64 products from the tcgen05 kernel (verification).

    ``y4``: (n, 4*V) int8, column 4 v + t = digit t of probe v."""
    bed_rows = np.ascontiguousarray(bed_rows, dtype=np.uint8)
    y4 = np.asfortranarray(y4, dtype=np.int8)
    L = bed_rows.shape[0]
    V = y4.shape[1] // 4
    g = np.empty((L, V), dtype=np.int64)
    o = np.empty((L, V), dtype=np.int64)
    check(_lib.load().lds_debug_xt_products_umma(ptr(bed_rows), bed_rows.shape[1], int(n), L,
                                                 ptr(y4), V, ptr(g), ptr(o)))
    return g, o


def set_p2_kernel(impl: str) -> None:
    """Phase-2 kernel for plans created afterwards: "tcgen05" (default) or "mma"."""
    check(_lib.load().lds_set_p2_kernel({"mma": 0, "tcgen05": 1}[impl]))


def set_slices(s: int) -> None:
    check(_lib.load().lds_set_slices(int(s)))


def synth_bed_rows(n: int, m: int, seed: int, missing: bool = True, out=None) -> np.ndarray:
    """Synthetic packed BED rows generated on the device (same bytes as bedfile.py).

    ``out``: optional C-contiguous (m, ceil(n/4)) uint8 array to fill (e.g. the
    numpy view of a pinned torch tensor)."""
    from .bedfile import allele_freqs, hwe_thresholds

    p = allele_freqs(seed, m)
    t0, t1 = hwe_thresholds(p)
    shape = (m, (n + 3) // 4)
    if out is None:
        out = np.empty(shape, dtype=np.uint8)
    elif out.shape != shape or out.dtype != np.uint8 or not out.flags["C_CONTIGUOUS"]:
        raise ValueError(f"out must be a C-contiguous uint8 array of shape {shape}")
    check(_lib.load().lds_synth_bed(int(n), int(m), int(seed), ptr(np.ascontiguousarray(t0)),
                                    ptr(np.ascontiguousarray(t1)), int(missing), ptr(out)))
    return out
