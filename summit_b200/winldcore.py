"""Drop-in replacement for SUMMIT's native ``winldcore`` module, backed by liblds.so.

``compute_windowed_ld_chr`` and ``compute_maf_bed`` keep the reference's
names, keyword arguments, defaults, array layouts and error messages
(``src/native/winldcore.cpp:964-994``), so ``summit.ldscore.win_ldscore`` can
import this module in place of the native one.  The exact windowed LD scores
are computed from exact int8 tensor-core Gram products of the decoded
genotypes (sm_100a); there is no CPU fallback.
"""
from __future__ import annotations

import numpy as np

from . import _lib
from ._lib import check, enc, ptr
from .gwldcore import _impute, _rows

_verbose = False
_threads = 0


def set_verbose(enabled: bool) -> None:
    global _verbose
    _verbose = bool(enabled)


def set_num_threads(n: int) -> None:
    """Host thread hint (the GPU path has no OpenMP region)."""
    global _threads
    _threads = int(n)


def get_max_threads() -> int:
    return max(1, _threads)


def get_progress_total() -> int:
    return 0


def get_progress_done() -> int:
    return 0


def progress_active() -> bool:
    return False


def compute_windowed_ld_chr(bed_prefix, fam_path, chr_start, chr_end, bp, annot_chr, ld_wind_kb,
                            chunk_size, row_sel=None, C=None, R=None, impute_mode="mean",
                            impute_seed=None, panel_cols=0, cache_mb=-1):
    """Exact windowed LD scores of SNPs [chr_start, chr_end): an m x K
    (column-major) FP64 array, as winldcore.compute_windowed_ld_chr returns."""
    m = int(chr_end) - int(chr_start)
    bp = np.ascontiguousarray(bp, dtype=np.int64)
    annot = np.asfortranarray(annot_chr, dtype=np.float64)
    if annot.ndim != 2:
        raise TypeError("incompatible function arguments: annot_chr must be 2-D")
    if m > 0 and bp.shape[0] != m:
        raise RuntimeError("bp length mismatch in compute_windowed_ld_chr")
    if m > 0 and annot.shape[0] != m:
        raise RuntimeError("annot_chr shape mismatch in compute_windowed_ld_chr")
    rows, nr = _rows(row_sel)
    Cp = Rp = None
    p = 0
    if C is not None and R is not None:
        Cp = np.asfortranarray(C, dtype=np.float64)
        Rp = np.asfortranarray(R, dtype=np.float64)
        p = int(Cp.shape[1])
        if rows is not None:
            n_rows = nr
        else:
            with open(fam_path, "rb") as f:
                n_rows = sum(1 for line in f if line.strip())
        if Cp.shape[0] != n_rows or Rp.shape != (p, n_rows):
            raise RuntimeError("C/R shape mismatch in compute_windowed_ld_chr")
    out = np.empty((max(m, 0), annot.shape[1]), dtype=np.float64, order="F")
    check(_lib.load().lds_compute_windowed_ld_chr(
        enc(bed_prefix), enc(fam_path), int(chr_start), int(chr_end), ptr(bp), ptr(annot),
        annot.shape[1], float(ld_wind_kb), int(chunk_size), ptr(rows), nr, ptr(Cp), ptr(Rp), p,
        _impute(impute_mode), int(impute_seed is not None),
        0 if impute_seed is None else int(impute_seed), int(panel_cols), int(cache_mb), ptr(out)))
    return out


def compute_maf_bed(bed_prefix, fam_path, nsnps, step_size, row_sel=None):
    """Minor allele frequency of the first nsnps SNPs over the selected samples."""
    rows, nr = _rows(row_sel)
    out = np.empty(max(int(nsnps), 0), dtype=np.float64)
    check(_lib.load().lds_compute_maf_bed(enc(bed_prefix), enc(fam_path), int(nsnps),
                                          int(step_size), ptr(rows), nr, ptr(out)))
    return out
