"""ctypes binding of liblds.so (declarations in include/lds.h).

The library is built in-tree by ``summit_b200.build`` (nvcc, sm_100a).  There is
no fallback: if the shared object is missing, importing the compute API raises.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

PKG = Path(__file__).resolve().parent
# SUMMIT_B200_CHECKED=1 loads the bounds-checked build (python -m
# summit_b200.build --checked) instead.
LIB_PATH = PKG / ("liblds_checked.so" if os.environ.get("SUMMIT_B200_CHECKED") == "1"
                  else "liblds.so")

LDS_DIST = {"rademacher": 0, "gaussian": 1, "normal": 1, "spherical": 2}
LDS_IMPUTE = {"mean": 0, "hwe": 1}

_p = C.c_void_p
_i64 = C.c_int64
_u64 = C.c_uint64
_int = C.c_int
_dbl = C.c_double
_str = C.c_char_p

# name -> (restype, argtypes); mirrors include/lds.h.
SIGNATURES: dict[str, tuple] = {
    "lds_last_error": (_str, []),
    "lds_version": (_str, []),
    "lds_device_count": (_int, []),
    "lds_set_slices": (_int, [_int]),
    "lds_get_slices": (_int, []),
    "lds_kernel_launches": (_u64, []),
    "lds_clear_device_cache": (None, []),
    "lds_last_timings": (_int, [_p, _int]),
    "lds_gw_ldscore": (_int, [_p, _i64, _i64, _i64, _p, _i64, _p, _i64, _int, _int, _int, _u64,
                              _int, _int, _int, _u64, _dbl, _int, _p, _p, _p, _p, _p]),
    "lds_gw_ldscore_bed": (_int, [_str, _str, _p, _i64, _p, _i64, _int, _int, _int, _u64, _int,
                                  _int, _int, _u64, _dbl, _int, _p, _p, _p, _p, _p]),
    "lds_debug_xt_products": (_int, [_p, _i64, _i64, _i64, _p, _i64, _p, _p]),
    "lds_synth_bed": (_int, [_i64, _i64, _u64, _p, _p, _int, _p]),
    "lds_set_stream": (_int, [_p]),
    "lds_debug_xt_products_umma": (_int, [_p, _i64, _i64, _i64, _p, _i64, _p, _p]),
    "lds_set_p2_kernel": (_int, [_int]),
    "lds_win_plan_create": (_int, [_i64, _p, _i64, _p, _i64, _int, _int, _int, _u64, _int, _dbl,
                                   _int, _int, _dbl, _p]),
    "lds_win_ldscore": (_int, [_p, _i64, _i64, _i64, _p, _i64, _p, _i64, _p, _i64, _int, _int,
                               _int, _u64, _int, _int, _int, _u64, _dbl, _int, _int, _int,
                               _p, _p, _p]),
    "lds_win_plan_execute": (_int, [_i64]),
    "lds_win_plan_results": (_int, [_i64, _p, _p, _p, _p]),
    "lds_win_plan_kernel_ms": (_int, [_i64, _p]),
    "lds_win_plan_bin_totals": (_int, [_i64, _p]),
    "lds_win_plan_cv_annot": (_int, [_i64, _p]),
    "lds_win_plan_set_tiling": (_int, [_i64, _int]),
    "lds_win_plan_set_p2_order": (_int, [_i64, _int]),
    "lds_win_plan_set_p2_bins": (_int, [_i64, _int]),
    "lds_win_plan_set_checks": (_int, [_i64, _int]),
    "lds_gw_plan_set_checks": (_int, [_i64, _int]),
    "lds_gw_plan_check": (_int, [_i64, _p, _p, _p, _p, _p]),
    "lds_win_plan_check": (_int, [_i64, _p, _p, _p, _p, _p]),
    "lds_check_vectors": (_int, [_p, _p, _i64, _p, _p]),
    "lds_checked_build": (_int, []),
    "lds_checked_errors": (_int, [_p]),
    "lds_geno_source_product": (_int, [_i64, _i64, _i64, _p, _i64, _p, _i64, _p]),
    "lds_geno_target_product": (_int, [_i64, _i64, _i64, _p, _i64, _p]),
    "lds_global_variant_probes": (_int, [_u64, _u64, _i64, _i64, _i64, _i64, _p]),
    "lds_generalized_component_diagonal": (_int, [_i64, _i64, _i64, _p, _int, _p, _int, _p, _int,
                                                  _p, _p]),
    "lds_generalized_pass2": (_int, [_i64, _p, _int, _int, _int, _int, _p, _p, _p, _dbl, _p, _i64,
                                     _p, _p]),
    "lds_generalized_project": (_int, [_p, _p, _p, _int, _int, _int, _int, _i64, _p, _p, _p]),
    "lds_generalized_pass2_sources": (_int, [_i64, _p, _int, _p, _p, _p, _int, _int, _int, _int,
                                             _p, _p, _p, _dbl, _p, _i64, _p, _p]),
    "lds_win_plan_destroy": (_int, [_i64]),
    "lds_win_plan_set_cv": (_int, [_i64, _p, _int, _int]),
    "lds_win_plan_tiles": (_int, [_i64, _p, _p]),
    "lds_win_plan_cv_outputs": (_int, [_i64, _int, _p, _p, _p, _p]),
    "lds_win_plan_cv_ms": (_int, [_i64, _p]),
    "lds_mlp_param_count": (_i64, [_int, _int]),
    "lds_mlp_forward": (_int, [_p, _int, _int, _p, _i64, _p]),
    "lds_mlp_loss_grad": (_int, [_p, _int, _int, _p, _p, _i64, _p, _p]),
    "lds_mlp_train": (_int, [_p, _int, _int, _p, _p, _i64, _int, _int, C.c_float, _u64, _p]),
    "lds_window_seed": (_u64, [_u64, _i64]),
    "lds_set_wait_limit": (_int, [C.c_longlong]),
    "lds_phase2_guard_counts": (_int, [_p]),
    "lds_get_wait_limit": (C.c_longlong, []),
    "lds_selftest_wait_timeout": (_int, [_p]),
    "lds_phase2_accum_device_noalloc": (_int, [_p, _i64, _i64, _i64, _i64, _i64, _p, _int, _int,
                                               _p, _p, _p, _p, _p, _p, _p, _p]),
    "lds_geno_create": (_int, [_p, _i64, _i64, _i64, _p, _i64, _int, _u64, _int, _p]),
    "lds_geno_destroy": (_int, [_i64]),
    "lds_nn_band": (_int, [_i64, _int, _p, _p]),
    "lds_geno_stats": (_int, [_i64, _p, _p]),
    "lds_geno_window_ld": (_int, [_i64, _i64, _i64, _p, _p, _p, _i64, _dbl, _p]),
    "lds_compute_windowed_ld_chr": (_int, [_str, _str, _int, _int, _p, _p, _i64, _dbl, _int, _p,
                                           _i64, _p, _p, _i64, _int, _int, _u64, _int, _int, _p]),
    "lds_compute_maf_bed": (_int, [_str, _str, _int, _int, _p, _i64, _p]),
    "lds_gxe_create": (_int, [_i64, _i64, _p, _i64, _p, _p, _i64, _p, _p, _p, _p, _int, _p]),
    "lds_gxe_destroy": (_int, [_i64]),
    "lds_gxe_set_checks": (_int, [_i64, _int]),
    "lds_gxe_last_check": (_int, [_i64, _p, _p, _p, _p, _p, _p]),
    "lds_gxe_create_dense": (_int, [_i64, _i64, _p, _i64, _p, _p, _i64, _p, _p, _p, _p, _int,
                                    _p]),
    "lds_gxe_source_block_dense": (_int, [_i64, _p, _i64, _p, _i64, _p, _int, _p, _p, _i64, _int,
                                          _p, _int]),
    "lds_gxe_target_score_block_dense": (_int, [_i64, _p, _i64, _i64, _p, _p, _i64, _p, _p, _p,
                                                _p, _i64, _i64, _int, _int, _int]),
    "lds_gxe_source_block": (_int, [_i64, _i64, _i64, _p, _i64, _p, _int, _p, _p, _i64, _int, _p,
                                    _int]),
    "lds_gxe_project_sources": (_int, [_i64, _p, _i64, _int, _int, _p, _int]),
    "lds_gxe_pair_create": (_int, [_i64, _p, _i64, _p, _i64, _int, _p]),
    "lds_gxe_pair_destroy": (_int, [_i64]),
    "lds_gxe_target_score_block": (_int, [_i64, _i64, _i64, _i64, _p, _p, _i64, _p, _p, _p, _p,
                                          _i64, _i64, _int, _int, _int]),
    "lds_gxe_normalize_scores": (_int, [_p, _p, _p, _p, _i64, _i64, _int, _int]),
    "lds_philox_rademacher": (_int, [_p, _i64, _i64, _p, _int]),
    "lds_block_boundaries": (_int, [_i64, _int, _p, _int, _p, _p]),
    "lds_sym_solve": (_int, [_p, _i64, _int, _dbl, _int, _p, _p, _p, _int]),
    "lds_sym_solve_diag": (_int, [_p, _i64, _int, _dbl, _p, _p, _p, _p, _p, _p, _p, _p]),
    "lds_jackknife_normal_equations": (_int, [_p, _i64, _int, _p, _p, _i64, _dbl, _p, _p, _p, _p,
                                              _int]),
    "lds_gw_plan_create": (_int, [_i64, _p, _i64, _int, _int, _int, _u64, _int, _dbl, _int, _int,
                                  _p]),
    "lds_gw_plan_execute": (_int, [_i64]),
    "lds_gw_plan_results": (_int, [_i64, _p, _p, _p, _p, _p]),
    "lds_gw_plan_kernel_ms": (_int, [_i64, _p]),
    "lds_gw_plan_destroy": (_int, [_i64]),
    "lds_generalized_source_product": (_int, [_i64, _i64, _i64, _p, _i64, _p]),
    "lds_generalized_target_product": (_int, [_i64, _i64, _i64, _p, _i64, _p]),
    "lds_debug_rademacher_block": (_int, [_u64, _int, _int, _int, _int, _p]),
    "lds_geno_create_synthetic": (_int, [_i64, _i64, _u64, _p, _p, _int, _int, _u64, _int, _p]),
    "lds_gw_plan_create_shard": (_int, [_i64, _p, _i64, _int, _int, _int, _u64, _int, _dbl, _int,
                                        _int, _i64, _p]),
    "lds_gw_plan_tiles": (_int, [_i64, _p, _p, _p]),
    "lds_gw_plan_phase1": (_int, [_i64, _int, _p]),
    "lds_gw_plan_phase2": (_int, [_i64, _int, _p]),
    "lds_gw_plan_set_bin_totals": (_int, [_i64, _p]),
    "lds_gw_plan_bin_totals": (_int, [_i64, _p]),
}
for _t in ("f32", "f64"):
    SIGNATURES[f"lds_phase1_compute_Xz_bed_chunk_{_t}"] = (
        _int, [_str, _str, _int, _int, _p, _i64, _int, _p, _i64, _i64, _p, _int, _int, _int, _int,
               _int, _u64, _p, _i64, _i64, _p, _int, _int, _u64, _p, _dbl, _p, _p, _i64, _p, _int])
    SIGNATURES[f"lds_phase2_accum_XtXz_bed_{_t}"] = (
        _int, [_str, _str, _int, _int, _p, _i64, _int, _p, _i64, _int, _p, _i64, _i64, _p, _i64,
               _i64, _int, _int, _int, _u64, _p, _p, _p, _p, _i64])
    SIGNATURES[f"lds_phase1_compute_Xz_bed_chunk_rowmajor_{_t}"] = (
        _int, [_str, _str, _int, _int, _p, _i64, _int, _p, _i64, _i64, _p, _int, _int, _int, _int,
               _int, _u64, _p, _i64, _i64, _int, _int, _u64, _p, _dbl, _p, _p, _i64, _p])
    SIGNATURES[f"lds_phase2_accum_XtXz_bed_mailman_{_t}"] = (
        _int, [_str, _str, _int, _int, _p, _i64, _int, _p, _i64, _int, _p, _i64, _i64, _p, _i64,
               _i64, _int, _int, _u64, _p, _p, _p, _p, _i64])
    SIGNATURES[f"lds_phase2_accum_XtXz_bed_mailman_rowmajor_{_t}"] = (
        _int, [_str, _str, _int, _int, _p, _i64, _int, _p, _i64, _int, _p, _i64, _i64, _p, _i64,
               _i64, _p, _i64, _int, _int, _u64, _p, _p])
    SIGNATURES[f"lds_compute_col_sums_rowmajor_{_t}"] = (_int, [_p, _i64, _i64, _p])
    SIGNATURES[f"lds_project_rowmajor_inplace_and_col_sums_{_t}"] = (
        _int, [_p, _i64, _i64, _p, _p, _i64, _p])
    SIGNATURES[f"lds_project_colmajor_inplace_{_t}"] = (_int, [_p, _i64, _i64, _p, _p, _i64])
    SIGNATURES[f"lds_standardize_dosage_inplace_{_t}"] = (_int, [_p, _i64, _i64, _int, _dbl, _p])
    SIGNATURES[f"lds_precompute_residual_variances_bed_{_t}"] = (
        _int, [_str, _str, _int, _int, _p, _i64, _int, _dbl, _int, _int, _u64, _p, _p, _p, _i64,
               _p, _int, _p, _i64, _i64, _p])
    SIGNATURES[f"lds_phase1_compute_Xz_geno_chunk_{_t}"] = (
        _int, [_p, _i64, _i64, _int, _p, _i64, _i64, _p, _int, _int, _int, _int, _int, _u64, _p,
               _i64, _i64, _p, _p, _p, _i64, _p, _p, _dbl])
    SIGNATURES[f"lds_phase2_accum_XtXz_geno_{_t}"] = (
        _int, [_p, _i64, _i64, _int, _p, _i64, _int, _p, _i64, _i64, _p, _i64, _i64, _p, _p,
               _i64, _int, _p, _p])
    SIGNATURES[f"lds_phase2_compute_XtXz_bed_{_t}"] = (
        _int, [_str, _str, _int, _int, _p, _i64, _int, _p, _i64, _int, _p, _i64, _i64, _p, _i64,
               _i64, _p, _p, _i64, _int, _int, _int, _u64])
    SIGNATURES[f"lds_apply_grm_bed_panel_{_t}"] = (
        _int, [_str, _str, _int, _int, _p, _i64, _int, _p, _i64, _p, _p, _i64, _i64, _p, _p,
               _i64, _int, _int, _u64])
    SIGNATURES[f"lds_apply_grm_bed_panel_mailman_{_t}"] = (
        _int, [_str, _str, _int, _int, _p, _i64, _int, _p, _i64, _p, _p, _i64, _i64, _p, _p,
               _i64, _int, _u64])
    SIGNATURES[f"lds_compute_block_corrections_binary_{_t}"] = (
        _int, [_p, _i64, _i64, _p, _p, _int, _dbl, _p, _p, _p, _p])

_LIB = None


def load() -> C.CDLL:
    """Load liblds.so (once).  Raises RuntimeError if it is not built."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not LIB_PATH.exists():
        raise RuntimeError(
            f"liblds.so not found at {LIB_PATH}; build it with `python -m summit_b200.build` "
            "(there is no CPU fallback)")
    lib = C.CDLL(str(LIB_PATH))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _LIB = lib
    return lib


def check(rc: int) -> None:
    if rc != 0:
        raise RuntimeError(load().lds_last_error().decode(errors="replace"))


def ptr(a):
    return None if a is None else a.ctypes.data_as(_p)


def enc(s) -> bytes:
    return os.fsencode(str(s))
