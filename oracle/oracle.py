"""ORACLE — CPU checkers for the genome-wide LD-score hot path (test infrastructure).

Two CPU implementations live here, and only tests/, ``__graft_entry__.smoke()``
and the CPU-baseline leg of ``bench.py`` may use them:

* ``Oracle`` — our FP64 restatement (``oracle/lds_oracle.cpp``), built into
  ``oracle/_build/liblds_oracle.so``;
* ``Reference`` — the reference's own ``gwldcore.cpp``/``genotype.cpp``
  compiled unchanged into ``oracle/_ref/libref_gwld.so`` (``oracle/Makefile``).

``gw_ldscore`` restates the per-V-tile driver of
``src/summit/ldscore/gw_ldscore.py:1753-2222`` (``GenomewideLDScore._compute_ldscore``)
for the case without covariates: balanced V-tiles (``_bounded_vtile_sizes``
:687-697), blocks of ``step_size`` SNPs (:1702-1703), residual variances fused
into the first phase-1 pass (:1776-1787), phase 1 per block (:1959), zeroing of
untouched bins (:2017-2019), phase 2 per block (:2096), division by the probe
count (:2197) and the correlation null ``M_k / N_denom`` (:2220-2222).  It can
drive either CPU implementation, so the restatement is checked against the
reference end to end.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ORACLE_SO = HERE / "_build" / "liblds_oracle.so"
REF_SO = HERE / "_ref" / "libref_gwld.so"
REF_WIN_SO = HERE / "_ref" / "libref_winld.so"

_p = C.c_void_p
_i64 = C.c_int64
_u64 = C.c_uint64
_int = C.c_int
_dbl = C.c_double
_str = C.c_char_p

DIST_CODES = {"rademacher": 0, "gaussian": 1, "normal": 1, "spherical": 2}


def _ptr(a):
    return None if a is None else a.ctypes.data_as(_p)


def bounded_vtile_sizes(nvecs: int, vmax: int, granularity: int = 64) -> list[int]:
    """Probe V-tile partition, gw_ldscore.py:687-697."""
    width = min(nvecs, vmax)
    if width >= granularity:
        width = max(granularity, (width // granularity) * granularity)
    return [min(width, nvecs - s) for s in range(0, nvecs, width)]


def band_counts(geno: np.ndarray, D: int) -> np.ndarray:
    """Integer sums GG, GO, OG, OO of SNP pairs (j, j+d), d = 0..D, from hard calls
    (M x N, missing < 0): the exact counts behind lds_nn_band (numpy, int64)."""
    g = np.where(geno >= 0, geno, 0).astype(np.int64)
    o = (geno >= 0).astype(np.int64)
    m = g.shape[0]
    out = np.zeros((m, D + 1, 4), dtype=np.int64)
    for d in range(D + 1):
        a, b = slice(0, m - d), slice(d, m)
        out[: m - d, d, 0] = (g[a] * g[b]).sum(1)
        out[: m - d, d, 1] = (g[a] * o[b]).sum(1)
        out[: m - d, d, 2] = (o[a] * g[b]).sum(1)
        out[: m - d, d, 3] = (o[a] * o[b]).sum(1)
    return out


def bp_window_bounds(bp: np.ndarray, ld_wind_kb: float) -> tuple[np.ndarray, np.ndarray]:
    """Per SNP j the partner interval [lo_j, hi_j) of |bp_i - bp_j| <= W
    (W = 1000 ld_wind_kb), as winldcore.cpp:434-442 (outside_bp_window) and
    :596-606 (compute_block_left) define the window on sorted positions."""
    bp = np.asarray(bp, dtype=np.int64)
    w = float(ld_wind_kb) * 1000.0
    lo = np.searchsorted(bp.astype(np.float64), bp - w, side="left")
    hi = np.searchsorted(bp.astype(np.float64), bp + w, side="right")
    return lo.astype(np.int64), hi.astype(np.int64)


def windowed_ld_exact(X: np.ndarray, annot: np.ndarray, lo: np.ndarray, hi: np.ndarray,
                      restandardize: bool, corr_dim: int | None) -> np.ndarray:
    """Exact windowed LD scores (FP64, dense; small inputs only).

    X: N x m standardized genotypes.  With ``restandardize`` each column is
    recentred and rescaled to unit variance over the N rows (ddof 0), as
    restandardize_cols_inplace (winldcore.cpp:215-267) does for mean
    imputation; r = X^T X / N (accum_self_panel / accum_cross_panels,
    :480-594); with ``corr_dim`` the unbiased r^2 - (1 - r^2)/(corr_dim - 1)
    (:409-432), else plain r^2; pairs outside [lo_j, hi_j) are zeroed after
    that (:434-478); LD = (f(r) o mask) annot."""
    X = np.array(X, dtype=np.float64, order="F", copy=True)
    n, m = X.shape
    if restandardize:
        for j in range(m):
            col = X[:, j]
            s, ss = col.sum(), (col * col).sum()
            mean = s / n
            v = ss - s * s / n
            if -1e-12 < v < 0.0:
                v = 0.0
            inv = 1.0
            if v > 0.0 and np.isfinite(v):
                var = v / n
                if var > 0.0 and np.isfinite(var):
                    inv = 1.0 / np.sqrt(var)
            X[:, j] = (col - mean) * inv
    r = (X.T @ X) / n
    f = r * r
    if corr_dim is not None:
        f = f - (1.0 - f) / float(corr_dim - 1)
    idx = np.arange(m)
    mask = (idx[None, :] >= lo[:, None]) & (idx[None, :] < hi[:, None])
    return np.where(mask, f, 0.0) @ np.asarray(annot, dtype=np.float64)


def compute_blocks(nsnps: int, step: int) -> list[tuple[int, int]]:
    """SNP blocks, gw_ldscore.py:1702-1703."""
    return [(s, min(nsnps, s + step)) for s in range(0, nsnps, step)]


class Oracle:
    """ctypes view of oracle/_build/liblds_oracle.so (our FP64 restatement)."""

    def __init__(self, path: Path = ORACLE_SO):
        if not path.exists():
            raise RuntimeError(f"oracle library missing: {path} (run `make -C oracle`)")
        L = C.CDLL(str(path))
        L.orc_last_error.restype = _str
        L.orc_standardize_block.argtypes = [_p, _i64, _i64, _p, _i64, _int, _int, _int, _int,
                                            _u64, _p, _p, _p]
        L.orc_make_probes.argtypes = [_u64, _int, _int, _int, _int, _int, _int, _p]
        L.orc_phase1_block.argtypes = [_p, _i64, _int, _p, _int, _p, _p, _int, _p, _p, _int]
        L.orc_phase2_block.argtypes = [_p, _i64, _int, _int, _p, _int, _p, _i64, _p, _int, _int,
                                       _p, _p, _dbl, _int]
        L.orc_inv_resvar_block.argtypes = [_p, _i64, _int, _dbl, _p]
        L.orc_int_products.argtypes = [_p, _i64, _i64, _int, _p, _i64, _p, _p]
        L.orc_synth_bed.argtypes = [_i64, _i64, _u64, _p, _p, _int, _p]
        self.lib = L

    def synth_bed_rows(self, n: int, m: int, seed: int, missing: bool = True) -> np.ndarray:
        """The synthetic generator of summit_b200/bedfile.py in C (same bytes)."""
        from summit_b200.bedfile import allele_freqs, hwe_thresholds

        t0, t1 = hwe_thresholds(allele_freqs(seed, m))
        out = np.empty((m, (n + 3) // 4), dtype=np.uint8)
        self.lib.orc_synth_bed(n, m, seed, _ptr(np.ascontiguousarray(t0)),
                               _ptr(np.ascontiguousarray(t1)), int(missing), _ptr(out))
        return out

    def standardize(self, bed_rows: np.ndarray, n_total: int, blk_start: int, blk_end: int,
                    rows=None, ddof=1, impute="mean", impute_seed=0):
        bed_rows = np.ascontiguousarray(bed_rows, dtype=np.uint8)
        rows_a = None if rows is None else np.ascontiguousarray(rows, dtype=np.int64)
        n = n_total if rows_a is None else rows_a.size
        L = blk_end - blk_start
        geno = np.empty((n, L), dtype=np.float64, order="F")
        mean = np.empty(L)
        inv = np.empty(L)
        self.lib.orc_standardize_block(_ptr(bed_rows), bed_rows.shape[1], n_total, _ptr(rows_a),
                                       n, blk_start, blk_end, ddof, int(impute == "hwe"),
                                       impute_seed, _ptr(geno), _ptr(mean), _ptr(inv))
        return geno, mean, inv

    def band_products(self, bed_rows, n_total, D, rows=None, ddof=1, impute="mean", impute_seed=0):
        """x_j . x_{j+d} for d = 0..D (0 past the last SNP) from the standardized
        genotypes of ``standardize`` (FP64)."""
        m = bed_rows.shape[0]
        X = self.standardize(bed_rows, n_total, 0, m, rows, ddof, impute, impute_seed)[0]
        xx = np.zeros((m, D + 1))
        for d in range(D + 1):
            xx[: m - d, d] = np.einsum("ij,ij->j", X[:, : m - d], X[:, d:])
        return xx

    def probes(self, root, blk_start, v_start, L, V, dist="rademacher", as_float=False):
        Z = np.empty((L, V), dtype=np.float64, order="F")
        self.lib.orc_make_probes(root, blk_start, v_start, L, V, DIST_CODES[dist],
                                 int(as_float), _ptr(Z))
        return Z

    def phase1_block(self, geno, annot, inv, Z, Xz, bin_init=None, as_float=False):
        N, L = geno.shape
        K = annot.shape[1]
        V = Z.shape[1]
        self.lib.orc_phase1_block(_ptr(geno), N, L, _ptr(np.ascontiguousarray(annot, np.float64)),
                                  K, _ptr(np.ascontiguousarray(inv, np.float64)), _ptr(Z), V,
                                  _ptr(Xz), _ptr(bin_init), int(as_float))

    def phase2_block(self, geno, blk_start, inv, V, Xz, meansq, N_denom, mc_agg=None,
                     mc_per_snp=None, extreme=1e10, drop_extreme=True):
        N, L = geno.shape
        rc = self.lib.orc_phase2_block(_ptr(geno), N, L, blk_start,
                                       _ptr(np.ascontiguousarray(inv, np.float64)), V, _ptr(Xz),
                                       Xz.shape[1], _ptr(meansq), meansq.shape[1], N_denom,
                                       _ptr(mc_agg), _ptr(mc_per_snp), extreme, int(drop_extreme))
        if rc:
            raise RuntimeError(self.lib.orc_last_error().decode())

    def inv_resvar(self, geno, eps=1e-10):
        N, L = geno.shape
        out = np.empty(L)
        self.lib.orc_inv_resvar_block(_ptr(geno), N, L, eps, _ptr(out))
        return out

    def int_products(self, bed_rows, n, y_q):
        """Exact int64 G^T y and O^T y for int8 columns y_q (N x Q, F-order)."""
        bed_rows = np.ascontiguousarray(bed_rows, dtype=np.uint8)
        y = np.asfortranarray(y_q, dtype=np.int8)
        L = bed_rows.shape[0]
        Q = y.shape[1]
        out = np.empty((L, Q), dtype=np.int64)
        obs = np.empty((L, Q), dtype=np.int64)
        self.lib.orc_int_products(_ptr(bed_rows), bed_rows.shape[1], n, L, _ptr(y), Q,
                                  _ptr(out), _ptr(obs))
        return out, obs

    # ------------------------------------------------------------------
    def gw_ldscore(self, bed_rows, n, annot, nvecs, step, seed, dist="rademacher",
                   vtile=None, ddof=1, impute="mean", impute_seed=0, as_float=False,
                   with_mc=False, rows=None, eps=1e-10, snp0=None):
        """Whole genome-wide estimator on our restatement (FP64 arithmetic).

        ``snp0`` (not None) runs the estimator on SNPs [snp0, snp0 + len(annot)) of the
        full image ``bed_rows`` (blocks and probe seeds counted from snp0, HWE
        imputation seeded by the SNP's index in the image) — one window of a
        windowed estimate.  Returns a dict with ``ldscore`` (M x K),
        ``meansq_accum``, ``inv`` and, if requested, the MC fourth-moment sums.
        """
        m = bed_rows.shape[0] if snp0 is None else len(annot)
        base = 0 if snp0 is None else int(snp0)
        annot = np.ascontiguousarray(annot, dtype=np.float64)
        K = annot.shape[1]
        nsel = n if rows is None else len(rows)
        blocks = compute_blocks(m, step)
        vt = bounded_vtile_sizes(nvecs, vtile or nvecs)
        std = [self.standardize(bed_rows, n, base + s, base + e, rows, ddof, impute, impute_seed)[0]
               for (s, e) in blocks]
        inv = np.concatenate([self.inv_resvar(g, eps) for g in std])
        if as_float:
            inv = inv.astype(np.float32).astype(np.float64)
        meansq = np.zeros((m, K))
        mc_agg = np.zeros(K) if with_mc else None
        mc_snp = np.zeros((m, K)) if with_mc else None
        N_denom = nsel - ddof + 1
        v0 = 0
        for V in vt:
            Xz = np.empty((nsel, K * V), order="F")
            init = np.zeros(K, dtype=np.uint8)
            for (s, e), g in zip(blocks, std):
                Z = self.probes(seed, s, v0, e - s, V, dist, as_float)
                self.phase1_block(g, annot[s:e], inv[s:e], Z, Xz, init, as_float)
            for k in np.flatnonzero(init == 0):
                Xz[:, k * V:(k + 1) * V] = 0.0
            for (s, e), g in zip(blocks, std):
                self.phase2_block(g, s, inv[s:e], V, Xz, meansq, N_denom, mc_agg, mc_snp)
            v0 += V
        ld = meansq / float(nvecs) - (annot.sum(axis=0) / float(nsel - ddof))[None, :]
        return {"ldscore": ld, "meansq_accum": meansq, "inv": inv,
                "mc_aggregate_sumsq": mc_agg, "mc_per_snp_sumsq": mc_snp}


class Reference:
    """ctypes view of the reference's own gwldcore.cpp, compiled unchanged."""

    def __init__(self, path: Path = REF_SO):
        if not path.exists():
            raise RuntimeError(f"reference library missing: {path} (run `make -C oracle ref`)")
        L = C.CDLL(str(path))
        L.ref_last_error.restype = _str
        L.ref_blas_config.restype = _str
        for t in ("f32", "f64"):
            getattr(L, f"ref_phase1_bed_{t}").argtypes = [
                _str, _str, _int, _int, _p, _i64, _int, _p, _i64, _i64, _p, _int, _int, _int,
                _str, _int, _u64, _p, _i64, _p, _str, _int, _u64, _p]
            getattr(L, f"ref_phase2_bed_{t}").argtypes = [
                _str, _str, _int, _int, _p, _i64, _int, _p, _i64, _int, _p, _i64, _i64, _p, _i64,
                _int, _str, _int, _u64, _p, _p]
            getattr(L, f"ref_phase2_geno_{t}").argtypes = [
                _p, _i64, _i64, _int, _p, _int, _p, _i64, _p, _i64, _int, _p, _p]
            getattr(L, f"ref_phase1_geno_{t}").argtypes = [
                _p, _i64, _i64, _int, _p, _i64, _p, _int, _int, _int, _str, _int, _u64, _p, _p]
            getattr(L, f"ref_resvar_bed_{t}").argtypes = [
                _str, _str, _int, _int, _p, _i64, _int, _dbl, _str, _int, _u64, _p]
            getattr(L, f"ref_phase1_bed_rowmajor_{t}").argtypes = [
                _str, _str, _int, _int, _p, _i64, _int, _p, _i64, _i64, _p, _int, _int, _int,
                _str, _int, _u64, _p, _i64, _str, _int, _u64]
            getattr(L, f"ref_col_sums_rowmajor_{t}").argtypes = [_p, _i64, _i64, _p]
            getattr(L, f"ref_project_rowmajor_{t}").argtypes = [_p, _i64, _i64, _p, _p, _i64, _p]
            getattr(L, f"ref_resvar_bed_cov_{t}").argtypes = [
                _str, _str, _int, _int, _p, _i64, _int, _dbl, _str, _int, _u64, _p, _p, _i64, _i64,
                _p, _p]
            getattr(L, f"ref_phase1_bed_cov_{t}").argtypes = [
                _str, _str, _int, _int, _p, _i64, _int, _p, _i64, _i64, _int, _int, _str, _u64, _p,
                _i64, _str, _p, _p, _i64, _p, _p]
            getattr(L, f"ref_project_colmajor_{t}").argtypes = [_p, _i64, _i64, _p, _p, _i64]
            getattr(L, f"ref_standardize_dosage_{t}").argtypes = [_p, _i64, _i64, _int, _dbl, _p]
            getattr(L, f"ref_phase2_mailman_rowmajor_{t}").argtypes = [
                _str, _str, _int, _int, _p, _i64, _int, _p, _i64, _int, _p, _i64, _i64, _p, _i64,
                _p, _int, _int, _u64, _p, _p]
            getattr(L, f"ref_phase1_geno_cov_{t}").argtypes = [
                _p, _i64, _i64, _int, _p, _i64, _p, _int, _int, _str, _u64, _p, _p, _p, _p, _i64,
                _p, _p]
            getattr(L, f"ref_phase2_geno_cov_{t}").argtypes = [
                _p, _i64, _i64, _int, _p, _int, _p, _i64, _p, _i64, _p, _p, _i64, _int, _p, _p]
            getattr(L, f"ref_phase2_bed_cov_{t}").argtypes = [
                _str, _str, _int, _int, _p, _i64, _int, _p, _i64, _int, _p, _i64, _i64, _p, _i64,
                _int, _str, _p, _p, _i64, _int, _p, _p]
            getattr(L, f"ref_phase1_bed_projright_{t}").argtypes = [
                _str, _str, _int, _int, _int, _p, _i64, _i64, _p, _int, _int, _str, _u64, _p, _i64,
                _p, _str, _p, _p, _i64]
            getattr(L, f"ref_phase2_legacy_{t}").argtypes = [
                _str, _str, _int, _int, _int, _p, _i64, _int, _p, _i64, _i64, _p, _i64, _int, _str,
                _p, _p, _i64]
            getattr(L, f"ref_apply_grm_{t}").argtypes = [
                _str, _str, _int, _int, _int, _p, _p, _p, _i64, _i64, _p, _p, _i64, _str, _int,
                _u64, _int]
            getattr(L, f"ref_resvar_mu22_{t}").argtypes = [
                _str, _str, _int, _int, _int, _str, _p, _i64, _p, _p, _i64, _i64, _p, _p]
            getattr(L, f"ref_block_corrections_{t}").argtypes = [
                _p, _i64, _i64, _p, _p, _int, _dbl, _p]
        L.ref_mailman_mean_stats.argtypes = [_p, _i64, _int, _i64, _int, _int, _p, _i64, _int, _p,
                                             _p, _p]
        L.ref_set_num_threads.argtypes = [_int]
        L.ref_set_omp_threads.argtypes = [_int]
        L.ref_set_blas_threads.argtypes = [_int]
        self.lib = L
        self.threads = 0

    def _chk(self, rc):
        if rc:
            raise RuntimeError(self.lib.ref_last_error().decode())

    def set_threads(self, n: int):
        self.threads = int(n)
        self.lib.ref_set_num_threads(int(n))

    def _phase_threads(self, phase: int):
        """OpenMP/BLAS split of the reference driver (gw_ldscore.py:1765-1771)."""
        if self.threads <= 0:
            return
        if phase == 1:
            self.lib.ref_set_omp_threads(self.threads)
            self.lib.ref_set_blas_threads(1)
        else:
            self.lib.ref_set_omp_threads(1)
            self.lib.ref_set_blas_threads(self.threads)

    def blas_config(self) -> str:
        return self.lib.ref_blas_config().decode()

    def clear_caches(self):
        self.lib.ref_clear_caches()

    @staticmethod
    def _t(dtype):
        return "f32" if np.dtype(dtype) == np.float32 else "f64"

    def phase1_bed(self, prefix, blk_start, blk_end, annot_blk, inv_right, v_start, v_count,
                   kmax_hint, rand_dist, seed, Xz, bin_init_mask=None, rows=None, ddof=1,
                   impute_mode="mean", impute_seed=None, inv_out=None):
        dt = Xz.dtype
        t = self._t(dt)
        annot_blk = np.ascontiguousarray(annot_blk, dtype=dt)
        inv_right = np.ascontiguousarray(inv_right, dtype=dt)
        rows_a = None if rows is None else np.ascontiguousarray(rows, dtype=np.int64)
        fn = getattr(self.lib, f"ref_phase1_bed_{t}")
        self._chk(fn(f"{prefix}.bed".removesuffix(".bed").encode(), f"{prefix}.fam".encode(),
                     blk_start, blk_end, _ptr(rows_a), 0 if rows_a is None else rows_a.size, ddof,
                     _ptr(annot_blk), annot_blk.shape[0], annot_blk.shape[1], _ptr(inv_right),
                     v_start, v_count, kmax_hint, rand_dist.encode(), int(seed is not None),
                     0 if seed is None else seed, _ptr(Xz), Xz.shape[0], _ptr(bin_init_mask),
                     impute_mode.encode(), int(impute_seed is not None),
                     0 if impute_seed is None else impute_seed, _ptr(inv_out)))

    def phase2_bed(self, prefix, blk_start, blk_end, inv_left, tile_nvecs, Xz, meansq,
                   N_denom, rows=None, ddof=1, impute_mode="mean", impute_seed=None,
                   mc_agg=None, mc_per_snp=None):
        t = self._t(Xz.dtype)
        inv_left = np.ascontiguousarray(inv_left, dtype=Xz.dtype)
        rows_a = None if rows is None else np.ascontiguousarray(rows, dtype=np.int64)
        fn = getattr(self.lib, f"ref_phase2_bed_{t}")
        self._chk(fn(str(prefix).encode(), f"{prefix}.fam".encode(), blk_start, blk_end,
                     _ptr(rows_a), 0 if rows_a is None else rows_a.size, ddof, _ptr(inv_left),
                     inv_left.size, tile_nvecs, _ptr(Xz), Xz.shape[0], Xz.shape[1], _ptr(meansq),
                     meansq.shape[0], N_denom, impute_mode.encode(), int(impute_seed is not None),
                     0 if impute_seed is None else impute_seed, _ptr(mc_agg), _ptr(mc_per_snp)))

    def phase2_geno(self, geno, blk_start, inv_left, tile_nvecs, Xz, meansq, N_denom,
                    mc_agg=None, mc_per_snp=None):
        t = self._t(Xz.dtype)
        geno = np.asfortranarray(geno, dtype=Xz.dtype)
        inv_left = np.ascontiguousarray(inv_left, dtype=Xz.dtype)
        fn = getattr(self.lib, f"ref_phase2_geno_{t}")
        self._chk(fn(_ptr(geno), geno.shape[0], geno.shape[1], blk_start, _ptr(inv_left),
                     tile_nvecs, _ptr(Xz), Xz.shape[1], _ptr(meansq), meansq.shape[0], N_denom,
                     _ptr(mc_agg), _ptr(mc_per_snp)))

    def phase1_bed_rowmajor(self, prefix, blk_start, blk_end, annot_blk, inv_right, v_start,
                            v_count, kmax_hint, rand_dist, seed, Xz, rows=None, ddof=1,
                            impute_mode="hwe", impute_seed=None):
        t = self._t(Xz.dtype)
        annot_blk = np.ascontiguousarray(annot_blk, dtype=Xz.dtype)
        inv_right = np.ascontiguousarray(inv_right, dtype=Xz.dtype)
        rows_a = None if rows is None else np.ascontiguousarray(rows, dtype=np.int64)
        fn = getattr(self.lib, f"ref_phase1_bed_rowmajor_{t}")
        self._chk(fn(str(prefix).encode(), f"{prefix}.fam".encode(), blk_start, blk_end,
                     _ptr(rows_a), 0 if rows_a is None else rows_a.size, ddof, _ptr(annot_blk),
                     annot_blk.shape[0], annot_blk.shape[1], _ptr(inv_right), v_start, v_count,
                     kmax_hint, rand_dist.encode(), int(seed is not None),
                     0 if seed is None else seed, _ptr(Xz), Xz.shape[0], impute_mode.encode(),
                     int(impute_seed is not None), 0 if impute_seed is None else impute_seed))

    def col_sums_rowmajor(self, Xz):
        out = np.empty(Xz.shape[1])
        self._chk(getattr(self.lib, f"ref_col_sums_rowmajor_{self._t(Xz.dtype)}")(
            _ptr(Xz), Xz.shape[0], Xz.shape[1], _ptr(out)))
        return out

    def phase2_mailman_rowmajor(self, prefix, blk_start, blk_end, inv_left, tile_nvecs, Xz,
                                meansq, sum_Xz, N_denom, rows=None, ddof=1, impute_seed=None,
                                mc_agg=None, mc_per_snp=None):
        t = self._t(Xz.dtype)
        inv_left = np.ascontiguousarray(inv_left, dtype=Xz.dtype)
        rows_a = None if rows is None else np.ascontiguousarray(rows, dtype=np.int64)
        sum_Xz = np.ascontiguousarray(sum_Xz, dtype=np.float64)
        fn = getattr(self.lib, f"ref_phase2_mailman_rowmajor_{t}")
        self._chk(fn(str(prefix).encode(), f"{prefix}.fam".encode(), blk_start, blk_end,
                     _ptr(rows_a), 0 if rows_a is None else rows_a.size, ddof, _ptr(inv_left),
                     inv_left.size, tile_nvecs, _ptr(Xz), Xz.shape[0], Xz.shape[1], _ptr(meansq),
                     meansq.shape[0], _ptr(sum_Xz), N_denom, int(impute_seed is not None),
                     0 if impute_seed is None else impute_seed, _ptr(mc_agg), _ptr(mc_per_snp)))

    def resvar_bed_cov(self, prefix, nsnps, step, C, R, dtype=np.float64, ddof=1, eps=1e-10,
                       impute_mode="mean", snp_var=None):
        t = self._t(dtype)
        Cf = np.asfortranarray(C, dtype=dtype)
        Rf = np.asfortranarray(R, dtype=dtype)
        out = np.empty(nsnps, dtype=dtype)
        self._chk(getattr(self.lib, f"ref_resvar_bed_cov_{t}")(
            str(prefix).encode(), f"{prefix}.fam".encode(), nsnps, step, None, 0, ddof, eps,
            impute_mode.encode(), 0, 0, _ptr(Cf), _ptr(Rf), Cf.shape[0], Cf.shape[1],
            _ptr(snp_var), _ptr(out)))
        return out

    def phase1_bed_cov(self, prefix, blk_start, blk_end, annot_blk, v_start, v_count, seed, Xz,
                       C, R, gram=None, ddof=1, impute_mode="mean"):
        t = self._t(Xz.dtype)
        dt = Xz.dtype
        ann = np.ascontiguousarray(annot_blk, dtype=dt)
        Cf = np.asfortranarray(C, dtype=dt)
        Rf = np.asfortranarray(R, dtype=dt)
        G = None if gram is None else np.ascontiguousarray(gram, dtype=dt)
        inv = np.empty(ann.shape[0], dtype=dt)
        self._chk(getattr(self.lib, f"ref_phase1_bed_cov_{t}")(
            str(prefix).encode(), f"{prefix}.fam".encode(), blk_start, blk_end, None, 0, ddof,
            _ptr(ann), ann.shape[0], ann.shape[1], v_start, v_count, b"rademacher", seed,
            _ptr(Xz), Xz.shape[0], impute_mode.encode(), _ptr(Cf), _ptr(Rf), Cf.shape[1],
            _ptr(G), _ptr(inv)))
        return inv

    # -- dense blocks, covariates inside the phases, GRM, mu22, corrections --
    @staticmethod
    def _cr(C, R, dt):
        if C is None or R is None:
            return None, None, 0
        Cf = np.asfortranarray(C, dtype=dt)
        return Cf, np.asfortranarray(R, dtype=dt), Cf.shape[1]

    def phase1_geno_cov(self, geno, blk_start, annot, inv_right, v_start, v_count, seed, Xz,
                        bin_init=None, C=None, R=None, gram=None, inv_out=None,
                        rand_dist="rademacher"):
        dt = Xz.dtype
        ann = np.ascontiguousarray(annot, dtype=dt)
        Cf, Rf, p = self._cr(C, R, dt)
        G = None if gram is None else np.ascontiguousarray(gram, dtype=dt)
        inv = None if inv_right is None else np.ascontiguousarray(inv_right, dtype=dt)
        self._chk(getattr(self.lib, f"ref_phase1_geno_cov_{self._t(dt)}")(
            _ptr(geno), geno.shape[0], geno.shape[1], blk_start, _ptr(ann), ann.shape[1],
            _ptr(inv), v_start, v_count, rand_dist.encode(), seed, _ptr(Xz), _ptr(bin_init),
            _ptr(Cf), _ptr(Rf), p, _ptr(G), _ptr(inv_out)))

    def phase2_geno_cov(self, geno, blk_start, inv_left, tile_nvecs, Xz, meansq, N_denom,
                        C=None, R=None, mc_agg=None, mc_per_snp=None):
        dt = meansq.dtype
        Cf, Rf, p = self._cr(C, R, dt)
        inv = np.ascontiguousarray(inv_left, dtype=dt)
        self._chk(getattr(self.lib, f"ref_phase2_geno_cov_{self._t(dt)}")(
            _ptr(geno), geno.shape[0], geno.shape[1], blk_start, _ptr(inv), tile_nvecs, _ptr(Xz),
            Xz.shape[1], _ptr(meansq), meansq.shape[0], _ptr(Cf), _ptr(Rf), p, N_denom,
            _ptr(mc_agg), _ptr(mc_per_snp)))

    def phase2_bed_cov(self, prefix, blk_start, blk_end, inv_left, tile_nvecs, Xz, meansq,
                       N_denom, C, R, mailman=False, impute_mode="mean", ddof=1, mc_agg=None,
                       mc_per_snp=None):
        dt = meansq.dtype
        Cf, Rf, p = self._cr(C, R, dt)
        inv = np.ascontiguousarray(inv_left, dtype=dt)
        self._chk(getattr(self.lib, f"ref_phase2_bed_cov_{self._t(dt)}")(
            str(prefix).encode(), f"{prefix}.fam".encode(), blk_start, blk_end, None, 0, ddof,
            _ptr(inv), inv.size, tile_nvecs, _ptr(Xz), Xz.shape[0], Xz.shape[1], _ptr(meansq),
            meansq.shape[0], N_denom, impute_mode.encode(), _ptr(Cf), _ptr(Rf), p, int(mailman),
            _ptr(mc_agg), _ptr(mc_per_snp)))

    def phase1_bed_projright(self, prefix, blk_start, blk_end, annot, inv_right, v_start,
                             v_count, seed, Xz, C, R, bin_init=None, impute_mode="mean", ddof=1):
        dt = Xz.dtype
        ann = np.ascontiguousarray(annot, dtype=dt)
        inv = np.ascontiguousarray(inv_right, dtype=dt)
        Cf, Rf, p = self._cr(C, R, dt)
        self._chk(getattr(self.lib, f"ref_phase1_bed_projright_{self._t(dt)}")(
            str(prefix).encode(), f"{prefix}.fam".encode(), blk_start, blk_end, ddof, _ptr(ann),
            ann.shape[0], ann.shape[1], _ptr(inv), v_start, v_count, b"rademacher", seed,
            _ptr(Xz), Xz.shape[0], _ptr(bin_init), impute_mode.encode(), _ptr(Cf), _ptr(Rf), p))

    def phase2_legacy(self, prefix, blk_start, blk_end, inv_left, nvecs, Xz, meansq, N_denom,
                      C=None, R=None, impute_mode="mean", ddof=1):
        dt = meansq.dtype
        Cf, Rf, p = self._cr(C, R, dt)
        inv = np.ascontiguousarray(inv_left, dtype=dt)
        self._chk(getattr(self.lib, f"ref_phase2_legacy_{self._t(dt)}")(
            str(prefix).encode(), f"{prefix}.fam".encode(), blk_start, blk_end, ddof, _ptr(inv),
            inv.size, nvecs, _ptr(Xz), Xz.shape[0], Xz.shape[1], _ptr(meansq), meansq.shape[0],
            N_denom, impute_mode.encode(), _ptr(Cf), _ptr(Rf), p))

    def apply_grm(self, prefix, nsnps, step, inv_all, panel_in, C=None, R=None,
                  impute_mode="mean", impute_seed=None, mailman=False, ddof=1):
        dt = panel_in.dtype
        Cf, Rf, p = self._cr(C, R, dt)
        pin = np.asfortranarray(panel_in)
        out = np.zeros(pin.shape, dtype=dt, order="F")
        inv = np.ascontiguousarray(inv_all, dtype=dt)
        self._chk(getattr(self.lib, f"ref_apply_grm_{self._t(dt)}")(
            str(prefix).encode(), f"{prefix}.fam".encode(), nsnps, step, ddof, _ptr(inv),
            _ptr(pin), _ptr(out), pin.shape[0], pin.shape[1], _ptr(Cf), _ptr(Rf), p,
            impute_mode.encode(), int(impute_seed is not None),
            0 if impute_seed is None else impute_seed, int(mailman)))
        return out

    def resvar_mu22(self, prefix, nsnps, step, annot, C=None, R=None, dtype=np.float64,
                    impute_mode="mean", ddof=1):
        t = self._t(dtype)
        ann = np.ascontiguousarray(annot, dtype=dtype)
        Cf, Rf, p = self._cr(C, R, dtype)
        inv = np.empty(nsnps, dtype=dtype)
        mu22 = np.empty((ann.shape[1], ann.shape[1]))
        N = 0 if Cf is None else Cf.shape[0]
        self._chk(getattr(self.lib, f"ref_resvar_mu22_{t}")(
            str(prefix).encode(), f"{prefix}.fam".encode(), nsnps, step, ddof,
            impute_mode.encode(), _ptr(ann), ann.shape[1], _ptr(Cf), _ptr(Rf), N, p, _ptr(inv),
            _ptr(mu22)))
        return inv, mu22

    def mailman_mean_stats(self, bed_path, n_total, start, stop, rows=None, ddof=1):
        """Mean, inverse scale and observed count of the Mailman mean pack."""
        bed = np.fromfile(str(bed_path), dtype=np.uint8)
        L = stop - start
        mean, inv, obs = np.empty(L), np.empty(L), np.empty(L, dtype=np.int32)
        rows_a = None if rows is None else np.ascontiguousarray(rows, dtype=np.int64)
        self._chk(self.lib.ref_mailman_mean_stats(
            _ptr(bed), bed.size, n_total, (n_total + 3) // 4, start, stop, _ptr(rows_a),
            0 if rows_a is None else rows_a.size, ddof, _ptr(mean), _ptr(inv), _ptr(obs)))
        return mean, inv, obs

    def block_corrections(self, meansq_raw, mu22, annot, N, d):
        m = np.ascontiguousarray(meansq_raw, dtype=np.float64)
        u = np.ascontiguousarray(mu22, dtype=np.float64)
        a = np.ascontiguousarray(annot)
        out = np.empty((4, m.shape[1], m.shape[1]))
        self._chk(getattr(self.lib, f"ref_block_corrections_{self._t(a.dtype)}")(
            _ptr(m), m.shape[0], m.shape[1], _ptr(u), _ptr(a), int(N), float(d), _ptr(out)))
        return tuple(out)

    def project_rowmajor(self, Xz, C=None, R=None):
        t = self._t(Xz.dtype)
        Cf = None if C is None else np.asfortranarray(C, dtype=Xz.dtype)
        Rf = None if R is None else np.asfortranarray(R, dtype=Xz.dtype)
        sums = np.empty(Xz.shape[1])
        self._chk(getattr(self.lib, f"ref_project_rowmajor_{t}")(
            _ptr(Xz), Xz.shape[0], Xz.shape[1], _ptr(Cf), _ptr(Rf),
            0 if Cf is None else Cf.shape[1], _ptr(sums)))
        return sums

    def project_colmajor(self, Xz, C=None, R=None):
        t = self._t(Xz.dtype)
        Cf = None if C is None else np.asfortranarray(C, dtype=Xz.dtype)
        Rf = None if R is None else np.asfortranarray(R, dtype=Xz.dtype)
        self._chk(getattr(self.lib, f"ref_project_colmajor_{t}")(
            _ptr(Xz), Xz.shape[0], Xz.shape[1], _ptr(Cf), _ptr(Rf),
            0 if Cf is None else Cf.shape[1]))

    def standardize_dosage(self, G, ddof=1, missing_value=-9.0):
        n = np.zeros(1, dtype=np.int64)
        self._chk(getattr(self.lib, f"ref_standardize_dosage_{self._t(G.dtype)}")(
            _ptr(G), G.shape[0], G.shape[1], int(ddof), float(missing_value), _ptr(n)))
        return int(n[0])

    def resvar_bed(self, prefix, nsnps, step, dtype=np.float64, rows=None, ddof=1, eps=1e-10,
                   impute_mode="mean", impute_seed=None):
        t = self._t(dtype)
        out = np.empty(nsnps, dtype=dtype)
        rows_a = None if rows is None else np.ascontiguousarray(rows, dtype=np.int64)
        fn = getattr(self.lib, f"ref_resvar_bed_{t}")
        self._chk(fn(str(prefix).encode(), f"{prefix}.fam".encode(), nsnps, step, _ptr(rows_a),
                     0 if rows_a is None else rows_a.size, ddof, eps, impute_mode.encode(),
                     int(impute_seed is not None), 0 if impute_seed is None else impute_seed,
                     _ptr(out)))
        return out

    def gw_ldscore(self, prefix, n, m, annot, nvecs, step, seed, dist="rademacher", vtile=None,
                   ddof=1, impute="mean", impute_seed=0, dtype=np.float64, with_mc=False,
                   rows=None, eps=1e-10):
        """The reference's per-block native calls in the order of
        GenomewideLDScore._compute_ldscore (gw_ldscore.py:1753-2222)."""
        annot = np.ascontiguousarray(annot, dtype=dtype)
        K = annot.shape[1]
        nsel = n if rows is None else len(rows)
        blocks = compute_blocks(m, step)
        vt = bounded_vtile_sizes(nvecs, vtile or nvecs)
        inv = np.empty(m, dtype=dtype)
        meansq = np.zeros((m, K), dtype=dtype)
        mc_agg = np.zeros(K) if with_mc else None
        mc_snp = np.zeros((m, K)) if with_mc else None
        N_denom = nsel - ddof + 1
        kmax = [int((annot[s:e] != 0).sum(axis=0).max()) for (s, e) in blocks]
        Xz_chunk = np.empty((nsel, K * max(vt)), dtype=dtype, order="F")
        init = np.empty(K, dtype=np.uint8)
        # The phase-1 CSR cache is keyed by array addresses; the driver clears
        # it around every run (gw_ldscore.py:1775, :2151).
        self.clear_caches()
        v0 = 0
        for ti, V in enumerate(vt):
            fuse = ti == 0
            Xz = Xz_chunk[:, :K * V]
            init.fill(0)
            self._phase_threads(1)
            for bi, (s, e) in enumerate(blocks):
                if kmax[bi] == 0 and not fuse:
                    continue
                self.phase1_bed(prefix, s, e, annot[s:e], inv[s:e], v0, V, kmax[bi], dist, seed,
                                Xz, init, rows, ddof, impute, impute_seed,
                                inv_out=inv[s:e] if fuse else None)
            for k in np.flatnonzero(init == 0):
                Xz[:, k * V:(k + 1) * V] = 0
            self._phase_threads(2)
            for (s, e) in blocks:
                self.phase2_bed(prefix, s, e, inv[s:e], V, Xz, meansq, N_denom, rows, ddof,
                                impute, impute_seed, mc_agg, mc_snp)
            v0 += V
        self.clear_caches()
        ms = (meansq / float(nvecs)).astype(dtype)
        ld = ms - (annot.sum(axis=0, dtype=np.float64) / float(nsel - ddof)).astype(dtype)[None, :]
        return {"ldscore": ld.astype(np.float64), "meansq_accum": meansq, "inv": inv,
                "mc_aggregate_sumsq": mc_agg, "mc_per_snp_sumsq": mc_snp}


class ReferenceWindowed:
    """ctypes view of the reference's own winldcore.cpp, compiled unchanged."""

    def __init__(self, path: Path = REF_WIN_SO):
        if not path.exists():
            raise RuntimeError(f"reference library missing: {path} (run `make -C oracle ref`)")
        L = C.CDLL(str(path))
        L.refw_last_error.restype = _str
        L.refw_set_num_threads.argtypes = [_int]
        L.refw_compute_windowed_ld_chr.argtypes = [
            _str, _str, _int, _int, _p, _p, _i64, _dbl, _int, _p, _i64, _p, _p, _i64, _i64,
            _str, _int, _u64, _int, _int, _p]
        L.refw_compute_maf_bed.argtypes = [_str, _str, _int, _int, _p, _i64, _p]
        self.lib = L

    def _chk(self, rc):
        if rc:
            raise RuntimeError(self.lib.refw_last_error().decode())

    def set_threads(self, n: int):
        self.lib.refw_set_num_threads(int(n))

    def compute_windowed_ld_chr(self, prefix, chr_start, chr_end, bp, annot, ld_wind_kb,
                                chunk_size, row_sel=None, C=None, R=None, impute_mode="mean",
                                impute_seed=None, panel_cols=0, cache_mb=-1):
        m = chr_end - chr_start
        bp = np.ascontiguousarray(bp, dtype=np.int64)
        annot = np.asfortranarray(annot, dtype=np.float64)
        rows = None if row_sel is None else np.ascontiguousarray(row_sel, dtype=np.int64)
        Cf = None if C is None else np.asfortranarray(C, dtype=np.float64)
        Rf = None if R is None else np.asfortranarray(R, dtype=np.float64)
        out = np.empty((m, annot.shape[1]), dtype=np.float64, order="F")
        self._chk(self.lib.refw_compute_windowed_ld_chr(
            str(prefix).encode(), f"{prefix}.fam".encode(), chr_start, chr_end, _ptr(bp),
            _ptr(annot), annot.shape[1], float(ld_wind_kb), int(chunk_size), _ptr(rows),
            0 if rows is None else rows.size, _ptr(Cf), _ptr(Rf),
            0 if Cf is None else Cf.shape[0], 0 if Cf is None else Cf.shape[1],
            impute_mode.encode(), int(impute_seed is not None),
            0 if impute_seed is None else int(impute_seed), int(panel_cols), int(cache_mb),
            _ptr(out)))
        return out

    def compute_maf_bed(self, prefix, nsnps, step_size, row_sel=None):
        rows = None if row_sel is None else np.ascontiguousarray(row_sel, dtype=np.int64)
        out = np.empty(nsnps)
        self._chk(self.lib.refw_compute_maf_bed(str(prefix).encode(), f"{prefix}.fam".encode(),
                                                nsnps, step_size, _ptr(rows),
                                                0 if rows is None else rows.size, _ptr(out)))
        return out


REF_GXE_SO = HERE / "_ref" / "libref_gxe.so"


class ReferenceGxe:
    """ctypes view of the reference's own gxeldcore.cpp (MultiEnvironmentKernel,
    protected right pair, NumPy-Philox probes), compiled unchanged."""

    def __init__(self, path: Path = REF_GXE_SO):
        if not path.exists():
            raise RuntimeError(f"reference library missing: {path} (run `make -C oracle ref`)")
        L = C.CDLL(str(path))
        L.refg_last_error.restype = _str
        L.refg_kernel_create.argtypes = [_i64, _i64, _p, _i64, _p, _p, _i64, _p, _p, _p, _i64, _p,
                                         _p, _i64, _p, _p, _int, _int, _int, C.POINTER(_p)]
        L.refg_kernel_destroy.argtypes = [_p]
        L.refg_source_block.argtypes = [_p, _p, _i64, _i64, _p, _i64, _p, _i64, _p, _i64, _p, _p,
                                        _i64, _int, _int]
        L.refg_project_sources.argtypes = [_p, _p, _i64, _i64, _int, _int, _p]
        L.refg_prepare_pair.argtypes = [_p, _i64, _i64, _p, _i64, _int, C.POINTER(_p)]
        L.refg_pair_destroy.argtypes = [_p]
        L.refg_target_score_block.argtypes = [_p, _p, _i64, _i64, _p, _p, _p, _i64, _p, _p, _p, _p,
                                              _i64, _i64, _int, _int, _int, _int]
        L.refg_normalize_scores.argtypes = [_p, _p, _p, _p, _p, _i64, _i64, _int]
        L.refg_philox_rademacher.argtypes = [_p, _i64, _int, _int, _p]
        L.refg_generalized_products.argtypes = [_p, _i64, _int, _i64, _int, _int, _int, _int, _p,
                                                _p, _p, _p]
        self.lib = L

    def _chk(self, rc):
        if rc:
            raise RuntimeError(self.lib.refg_last_error().decode())

    def kernel(self, environments, feature_basis, power_indices, power_offsets, ranks,
               gram_values, gram_offsets, e2_gram_values, common_basis, directions, ddof,
               annotation_bins, threads=1):
        return _RefGxeKernel(self, environments, feature_basis, power_indices, power_offsets,
                             ranks, gram_values, gram_offsets, e2_gram_values, common_basis,
                             directions, ddof, annotation_bins, threads)

    def generalized_products(self, bed_path, n_total, start, stop, rhs_src, rhs_tgt, ddof=1):
        """The reference's packed_source_product / packed_target_product
        (generalized_gxe_variant.inc:1749-1988) on the mean-imputed Mailman pack
        of SNPs [start, stop): returns (N x cols source, L x cols target)."""
        bed = np.fromfile(str(bed_path), dtype=np.uint8)
        L = stop - start
        cols = rhs_src.shape[1]
        rs = np.asfortranarray(rhs_src, dtype=np.float64)
        rt = np.asfortranarray(rhs_tgt, dtype=np.float64)
        assert rs.shape == (L, cols) and rt.shape == (n_total, cols)
        src = np.empty((n_total, cols), order="F")
        tgt = np.empty((L, cols), order="F")
        self._chk(self.lib.refg_generalized_products(
            _ptr(bed), bed.size, n_total, (n_total + 3) // 4, start, stop, ddof, cols, _ptr(rs),
            _ptr(src), _ptr(rt), _ptr(tgt)))
        return src, tgt

    def philox_rademacher(self, keys, rows, threads=1):
        keys = np.ascontiguousarray(keys, dtype=np.uint64)
        out = np.empty((rows, keys.shape[0]), dtype=np.float64, order="F")
        self._chk(self.lib.refg_philox_rademacher(_ptr(keys), keys.shape[0], int(rows),
                                                   int(threads), _ptr(out)))
        return out


class _RefGxeKernel:
    def __init__(self, ref, env, fb, pidx, poff, ranks, gv, goff, e2, common, dirs, ddof, bins,
                 threads):
        self.ref = ref
        F = lambda a: np.asfortranarray(a, dtype=np.float64)
        self.keep = [F(env), F(fb), np.ascontiguousarray(pidx, np.int64),
                     np.ascontiguousarray(poff, np.int64), np.ascontiguousarray(ranks, np.int32),
                     np.ascontiguousarray(gv, np.float64), np.ascontiguousarray(goff, np.int64),
                     np.ascontiguousarray(e2, np.float64), F(common), F(dirs)]
        env, fb, pidx, poff, ranks, gv, goff, e2, common, dirs = self.keep
        self.N, self.E = env.shape
        h = _p()
        ref._chk(ref.lib.refg_kernel_create(
            self.N, self.E, _ptr(env), fb.shape[1], _ptr(fb), _ptr(pidx), pidx.size, _ptr(poff),
            _ptr(ranks), _ptr(gv), gv.size, _ptr(goff), _ptr(e2), common.shape[1], _ptr(common),
            _ptr(dirs), int(ddof), int(bins), int(threads), C.byref(h)))
        self.h = h

    def source_block(self, target, genotype, probes, annotation, scale_x, scale_w,
                     environment_start, annotation_is_sqrt=False):
        F = lambda a: np.asfortranarray(a, dtype=np.float64)
        g, z, a, sx, sw = F(genotype), F(probes), F(annotation), F(scale_x), F(scale_w)
        self.ref._chk(self.ref.lib.refg_source_block(
            self.h, _ptr(target), target.shape[0], target.shape[1], _ptr(g), g.shape[1], _ptr(z),
            z.shape[1], _ptr(a), a.shape[1], _ptr(sx), _ptr(sw), sx.shape[1],
            int(environment_start), int(bool(annotation_is_sqrt))))

    def project_sources(self, panel, columns_per_environment, environment_start):
        tile = panel.shape[1] // (2 * columns_per_environment)
        leak = np.empty(max(tile, 1))
        self.ref._chk(self.ref.lib.refg_project_sources(
            self.h, _ptr(panel), panel.shape[0], panel.shape[1], int(columns_per_environment),
            int(environment_start), _ptr(leak)))
        return leak[:tile]

    def pair(self, right, row_weights, threads=1):
        right = np.asfortranarray(right, dtype=np.float64)
        w = np.asfortranarray(row_weights, dtype=np.float64)
        h = _p()
        self.ref._chk(self.ref.lib.refg_prepare_pair(_ptr(right), right.shape[0], right.shape[1],
                                                     _ptr(w), w.shape[1], int(threads), C.byref(h)))
        return h

    def target_score_block(self, genotype, pair, scale_x, scale_w, accs, block_start,
                           total_variants, probe_count, environment_start):
        F = lambda a: np.asfortranarray(a, dtype=np.float64)
        g, sx, sw = F(genotype), F(scale_x), F(scale_w)
        xx, xw, wx, ww = accs
        self.ref._chk(self.ref.lib.refg_target_score_block(
            self.h, _ptr(g), g.shape[0], g.shape[1], pair, _ptr(sx), _ptr(sw), sx.shape[1],
            _ptr(xx), _ptr(xw), _ptr(wx), _ptr(ww), xx.shape[0], xx.shape[1], int(block_start),
            int(total_variants), int(probe_count), int(environment_start)))

    def normalize_scores(self, accs, probe_count):
        xx, xw, wx, ww = accs
        self.ref._chk(self.ref.lib.refg_normalize_scores(
            self.h, _ptr(xx), _ptr(xw), _ptr(wx), _ptr(ww), xx.shape[0], xx.shape[1],
            int(probe_count)))

    def __del__(self):
        try:
            self.ref.lib.refg_kernel_destroy(self.h)
        except Exception:
            pass
