"""Resident genome-wide LD-score estimates (device genotype image + reusable plan).

``GwSession`` wraps the handle/plan entry points of liblds.so: the BED image
is uploaded and prepared once; ``plan()`` builds every kernel input of one
estimate (residual variances, annotation CSR lists, the reference's per-block
probe streams); ``execute()`` enqueues the estimate's kernels asynchronously
on the library stream; ``results()`` waits and finalizes.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import check, ptr
from .gwldcore import _dist, _impute, _rows


class GwPlan:
    def __init__(self, session: "GwSession", handle: int, M: int, K: int, with_mc: bool):
        self.session = session
        self.handle = handle
        self.M, self.K, self.with_mc = M, K, with_mc

    def execute(self) -> None:
        check(_lib.load().lds_gw_plan_execute(self.handle))

    def results(self) -> dict:
        M, K = self.M, self.K
        ld = np.empty((M, K))
        ms = np.empty((M, K))
        inv = np.empty(M)
        mca = np.empty(K) if self.with_mc else None
        mcp = np.empty((M, K)) if self.with_mc else None
        check(_lib.load().lds_gw_plan_results(self.handle, ptr(ld), ptr(ms), ptr(inv), ptr(mca),
                                              ptr(mcp)))
        return {"ldscore": ld, "meansq_accum": ms, "inv": inv, "mc_aggregate_sumsq": mca,
                "mc_per_snp_sumsq": mcp}

    def kernel_ms(self) -> dict:
        """Mean CUDA-event time per kernel kind over the executes since the last call."""
        buf = np.zeros(4)
        check(_lib.load().lds_gw_plan_kernel_ms(self.handle, ptr(buf)))
        return {"weights": buf[0], "phase1": buf[1], "digits": buf[2], "phase2": buf[3]}

    def set_checks(self, on: bool = True) -> None:
        """Exact integrity checks of the phase-2 products (as WinPlan.set_checks);
        call before the first execute."""
        check(_lib.load().lds_gw_plan_set_checks(self.handle, int(bool(on))))

    def check_products(self) -> dict:
        """Checksums of the last estimate (as WinPlan.check_products)."""
        n = np.zeros(1, dtype=np.int64)
        f = np.zeros(1, dtype=np.int64)
        ms = np.zeros(1)
        lhs = np.zeros((self.M, 2), dtype=np.uint64)
        rhs = np.zeros((self.M, 2), dtype=np.uint64)
        check(_lib.load().lds_gw_plan_check(self.handle, ptr(lhs), ptr(rhs), ptr(n), ptr(f),
                                            ptr(ms)))
        return {"mismatches": int(n[0]), "first_snp": int(f[0]), "check_ms": float(ms[0]),
                "lhs": lhs, "rhs": rhs}

    # -- the two halves of an estimate, for callers that exchange the sketch --
    def tiles(self) -> tuple[list[int], int]:
        """Probe counts of the V-tiles and the sketch's row count N_pad."""
        n = C.c_int(0)
        rows = C.c_int64(0)
        lib = _lib.load()
        check(lib.lds_gw_plan_tiles(self.handle, C.byref(n), None, C.byref(rows)))
        sizes = np.zeros(max(n.value, 1), dtype=np.int32)
        check(lib.lds_gw_plan_tiles(self.handle, None, ptr(sizes), None))
        return [int(v) for v in sizes[:n.value]], int(rows.value)

    def phase1(self, tile: int, sketch_ptr: int) -> None:
        """Enqueue phase 1 of V-tile ``tile`` into the device buffer at
        ``sketch_ptr`` (N_pad x K*V FP64, column-major)."""
        check(_lib.load().lds_gw_plan_phase1(self.handle, int(tile), C.c_void_p(int(sketch_ptr))))

    def phase2(self, tile: int, sketch_ptr: int) -> None:
        """Enqueue phase 2 of V-tile ``tile`` from the (all-reduced) sketch."""
        check(_lib.load().lds_gw_plan_phase2(self.handle, int(tile), C.c_void_p(int(sketch_ptr))))

    def bin_totals(self) -> np.ndarray:
        out = np.empty(self.K)
        check(_lib.load().lds_gw_plan_bin_totals(self.handle, ptr(out)))
        return out

    def set_bin_totals(self, Mk) -> None:
        Mk = np.ascontiguousarray(Mk, dtype=np.float64)
        if Mk.shape != (self.K,):
            raise ValueError("bin totals must have one value per annotation bin")
        check(_lib.load().lds_gw_plan_set_bin_totals(self.handle, ptr(Mk)))

    def close(self) -> None:
        if self.handle:
            _lib.load().lds_gw_plan_destroy(self.handle)
            self.handle = 0

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class GwSession:
    def __init__(self, bed_rows: np.ndarray, n_total: int, impute_mode: str = "mean",
                 impute_seed: int = 0, ddof: int = 1, row_sel=None):
        bed_rows = np.ascontiguousarray(bed_rows, dtype=np.uint8)
        self.M, self.row_bytes = bed_rows.shape
        self.n_total = int(n_total)
        rows, nr = _rows(row_sel)
        self.N = self.n_total if rows is None else nr
        h = C.c_int64(0)
        check(_lib.load().lds_geno_create(ptr(bed_rows), self.row_bytes, self.n_total, self.M,
                                          ptr(rows), nr, _impute(impute_mode), int(impute_seed),
                                          int(ddof), C.byref(h)))
        self.handle = h.value

    @classmethod
    def synthetic(cls, n: int, m: int, seed: int, missing: bool = True, impute_mode: str = "mean",
                  impute_seed: int = 0, ddof: int = 1) -> "GwSession":
        """Image of the seeded synthetic genotypes (gwldcore.synth_bed_rows'
        bytes) generated on the device, with no host copy of the BED rows."""
        from .bedfile import allele_freqs, hwe_thresholds

        t0, t1 = hwe_thresholds(allele_freqs(seed, m))
        self = cls.__new__(cls)
        self.M, self.row_bytes = int(m), (int(n) + 3) // 4
        self.n_total = self.N = int(n)
        h = C.c_int64(0)
        check(_lib.load().lds_geno_create_synthetic(
            int(n), int(m), int(seed), ptr(np.ascontiguousarray(t0, dtype=np.int64)),
            ptr(np.ascontiguousarray(t1, dtype=np.int64)), int(missing), _impute(impute_mode),
            int(impute_seed), int(ddof), C.byref(h)))
        self.handle = h.value
        return self

    def plan(self, annot, nvecs: int, step_size: int, seed: int, rand_dist: str = "rademacher",
             vtile: int | None = None, eps: float = 1e-10, as_float: bool = False,
             with_mc: bool = False) -> GwPlan:
        annot = np.ascontiguousarray(annot, dtype=np.float64)
        if annot.shape[0] != self.M:
            raise ValueError("annot must have one row per SNP")
        h = C.c_int64(0)
        check(_lib.load().lds_gw_plan_create(self.handle, ptr(annot), annot.shape[1], int(nvecs),
                                             int(step_size), int(vtile or 0), int(seed),
                                             _dist(rand_dist), float(eps), int(as_float),
                                             int(with_mc), C.byref(h)))
        return GwPlan(self, h.value, self.M, annot.shape[1], with_mc)

    def shard_plan(self, annot, nvecs: int, step_size: int, seed: int, snp_offset: int,
                   rand_dist: str = "rademacher", vtile: int | None = None, eps: float = 1e-10,
                   as_float: bool = False, with_mc: bool = False) -> GwPlan:
        """``plan`` for an image that holds SNPs [snp_offset, snp_offset + M) of
        the fileset (one SNP shard); snp_offset is a multiple of step_size."""
        annot = np.ascontiguousarray(annot, dtype=np.float64)
        if annot.shape[0] != self.M:
            raise ValueError("annot must have one row per SNP")
        h = C.c_int64(0)
        check(_lib.load().lds_gw_plan_create_shard(
            self.handle, ptr(annot), annot.shape[1], int(nvecs), int(step_size), int(vtile or 0),
            int(seed), _dist(rand_dist), float(eps), int(as_float), int(with_mc),
            int(snp_offset), C.byref(h)))
        return GwPlan(self, h.value, self.M, annot.shape[1], with_mc)

    def stats(self) -> dict:
        """Per-SNP mean (2 x allele frequency) and inverse sd of the standardization."""
        mean, sdinv = np.empty(self.M), np.empty(self.M)
        check(_lib.load().lds_geno_stats(self.handle, ptr(mean), ptr(sdinv)))
        return {"mean": mean, "sdinv": sdinv}

    def nn_band(self, D: int = 8, with_counts: bool = False):
        """Exact products x_j . x_{j+d}, d = 0..D, of the standardized genotypes
        (M x (D+1)); with ``with_counts`` also the integer sums GG, GO, OG, OO
        (M x (D+1) x 4)."""
        xx = np.empty((self.M, D + 1))
        cnt = np.empty((self.M, D + 1, 4), dtype=np.int32) if with_counts else None
        check(_lib.load().lds_nn_band(self.handle, int(D), ptr(xx), ptr(cnt)))
        return (xx, cnt) if with_counts else xx

    def block(self, start: int, stop: int):
        """SNPs [start, stop) of this image as a genotype block argument of the
        GxE kernel (summit_b200.gxeldcore)."""
        from .gxeldcore import GenotypeBlock

        return GenotypeBlock(self, start, stop)

    def window_ld(self, lo, hi, annot, corr_dim: float | None = None, row0: int = 0,
                  row1: int | None = None) -> np.ndarray:
        """Exact windowed LD scores of SNPs [row0, row1): row j sums f(r_ij) annot[i]
        over i in [lo[j - row0], hi[j - row0]), f = r^2, or with ``corr_dim`` the
        unbiased r^2 - (1 - r^2)/(corr_dim - 1).  annot has one row per SNP of the
        range; returns (row1 - row0) x K."""
        row1 = self.M if row1 is None else int(row1)
        m = row1 - int(row0)
        lo = np.ascontiguousarray(lo, dtype=np.int64)
        hi = np.ascontiguousarray(hi, dtype=np.int64)
        annot = np.ascontiguousarray(annot, dtype=np.float64)
        if annot.ndim == 1:
            annot = annot[:, None]
        if lo.shape != (m,) or hi.shape != (m,) or annot.shape[0] != m:
            raise ValueError("lo, hi and annot must have one row per SNP of [row0, row1)")
        out = np.empty((m, annot.shape[1]))
        check(_lib.load().lds_geno_window_ld(self.handle, int(row0), row1, ptr(lo), ptr(hi),
                                             ptr(annot), annot.shape[1],
                                             float(corr_dim or 0.0), ptr(out)))
        return out

    def partition_ld_expectation(self, annot, window_starts) -> np.ndarray:
        """Exact expectation of the windowed stochastic estimator (WinPlan) on
        this image: per SNP j of window w, sum_{i in w} r_ij^2 annot[i] minus the
        correlation null M_k(w) / (N - 1)."""
        ws = np.ascontiguousarray(window_starts, dtype=np.int64)
        annot = np.ascontiguousarray(annot, dtype=np.float64)
        win = np.repeat(np.arange(ws.size - 1), np.diff(ws))
        lo, hi = ws[win], ws[win + 1]
        ld = self.window_ld(lo, hi, annot)
        mkw = np.zeros((ws.size - 1, annot.shape[1]))
        np.add.at(mkw, win, annot)
        return ld - mkw[win] / float(self.N - 1)

    def close(self) -> None:
        if self.handle:
            _lib.load().lds_geno_destroy(self.handle)
            self.handle = 0

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class WinPlan:
    """Windowed + partitioned stochastic LD scores on a resident genotype image.

    Windows partition the SNPs (``window_starts`` = W+1 increasing offsets from 0
    to M).  Window w uses probe root ``window_seed(seed, w)`` and SNP blocks counted
    from its start, so its scores equal the genome-wide estimate on its SNPs.
    The first ``execute()`` captures the whole estimate in a CUDA graph.
    """

    def __init__(self, session: "GwSession", annot, window_starts, nvecs: int, step_size: int,
                 seed: int, rand_dist: str = "rademacher", vtile: int | None = None,
                 eps: float = 1e-10, as_float: bool = False, with_mc: bool = False,
                 batch_gb: float = 8.0):
        annot = np.ascontiguousarray(annot, dtype=np.float64)
        ws = np.ascontiguousarray(window_starts, dtype=np.int64)
        self.M, self.K = annot.shape
        self.W = ws.size - 1
        self.with_mc = with_mc
        h = C.c_int64(0)
        check(_lib.load().lds_win_plan_create(session.handle, ptr(annot), self.K, ptr(ws),
                                              ws.size - 1, int(nvecs), int(step_size),
                                              int(vtile or 0), int(seed), _dist(rand_dist),
                                              float(eps), int(as_float), int(with_mc),
                                              float(batch_gb), C.byref(h)))
        self.handle = h.value

    def execute(self) -> None:
        check(_lib.load().lds_win_plan_execute(self.handle))

    def results(self, meansq: bool = True) -> dict:
        """LD scores (M x K); with ``meansq`` also the raw accumulators and the
        inverse residual sds (and the MC sums of a with_mc plan)."""
        M, K = self.M, self.K
        ld = np.empty((M, K))
        ms = np.empty((M, K)) if meansq else None
        inv = np.empty(M) if meansq else None
        mcp = np.empty((M, K)) if (self.with_mc and meansq) else None
        check(_lib.load().lds_win_plan_results(self.handle, ptr(ld), ptr(ms), ptr(inv), ptr(mcp)))
        return {"ldscore": ld, "meansq_accum": ms, "inv": inv, "mc_per_snp_sumsq": mcp}

    def kernel_ms(self) -> dict:
        buf = np.zeros(4)
        check(_lib.load().lds_win_plan_kernel_ms(self.handle, ptr(buf)))
        return {"weights": buf[0], "phase1": buf[1], "digits": buf[2], "phase2": buf[3]}

    # ---- control-variate outputs (see lds_win_plan_set_cv) ----
    def set_tiling(self, p1_sb_per_cta: int = 0) -> None:
        """Phase-1 super-bins per CTA (0: default); call before the first
        execute."""
        check(_lib.load().lds_win_plan_set_tiling(self.handle, int(p1_sb_per_cta)))

    def set_p2_order(self, bin_chunk: int = 4) -> None:
        """Phase-2 CTA order: chunks of about bin_chunk bins per window (whole
        bin groups, at least one; 0: grid order); call before the first
        execute."""
        check(_lib.load().lds_win_plan_set_p2_order(self.handle, int(bin_chunk)))

    def set_p2_bins(self, bins_per_cta: int = 0) -> None:
        """Bins per phase-2 CTA (0: the fewest 256-column MMA groups per SNP
        tile); call before the first execute."""
        check(_lib.load().lds_win_plan_set_p2_bins(self.handle, int(bins_per_cta)))

    def set_checks(self, on: bool = True) -> None:
        """Exact integrity checks of the phase-2 products on every estimate
        (checksums from the tensor-core epilogue against a CUDA-core
        recomputation); call before the first execute."""
        check(_lib.load().lds_win_plan_set_checks(self.handle, int(bool(on))))

    def check_products(self) -> dict:
        """Checksums of the last estimate: {"mismatches", "first_snp",
        "check_ms", "lhs", "rhs"} (lhs / rhs: M x 2 uint64, columns G and O).
        A mismatch means some tensor-core product of that SNP was wrong."""
        n = np.zeros(1, dtype=np.int64)
        f = np.zeros(1, dtype=np.int64)
        ms = np.zeros(1)
        lhs = np.zeros((self.M, 2), dtype=np.uint64)
        rhs = np.zeros((self.M, 2), dtype=np.uint64)
        check(_lib.load().lds_win_plan_check(self.handle, ptr(lhs), ptr(rhs), ptr(n), ptr(f),
                                             ptr(ms)))
        return {"mismatches": int(n[0]), "first_snp": int(f[0]), "check_ms": float(ms[0]),
                "lhs": lhs, "rhs": rhs}

    def cv_annot_view(self):
        """Read-only torch view (cuda, float64, M x K) of the annotation matrix the
        plan uploaded in set_cv; valid while the plan lives."""
        import torch

        p = C.c_void_p(0)
        check(_lib.load().lds_win_plan_cv_annot(self.handle, C.byref(p)))

        class _View:  # __cuda_array_interface__ v3 of the plan's buffer
            __cuda_array_interface__ = {"shape": (self.M, self.K), "typestr": "<f8",
                                        "data": (int(p.value), False), "version": 3,
                                        "strides": None}

        return torch.as_tensor(_View(), device="cuda")

    def bin_totals(self) -> np.ndarray:
        """Per-window annotation totals M_{w,k} (W x K, summed in SNP order)."""
        out = np.empty((self.W, self.K))
        check(_lib.load().lds_win_plan_bin_totals(self.handle, ptr(out)))
        return out

    def set_cv(self, annot, split_tiles: bool = True, band: int = 8) -> None:
        annot = np.ascontiguousarray(annot, dtype=np.float64)
        check(_lib.load().lds_win_plan_set_cv(self.handle, ptr(annot), int(split_tiles), int(band)))
        self.split, self.band = bool(split_tiles), int(band)

    def tiles(self) -> list[int]:
        n = C.c_int(0)
        sizes = np.zeros(4096, dtype=np.int32)
        check(_lib.load().lds_win_plan_tiles(self.handle, C.byref(n), ptr(sizes)))
        return [int(x) for x in sizes[: n.value]]

    def cv_outputs(self) -> dict:
        """Host copies: meansq per probe slice (two halves with split_tiles), near-field
        sums C per slice, mu, xx."""
        T = 2 if getattr(self, "split", False) else 1
        M, K = self.M, self.K
        out = {"meansq": np.empty((T, M, K)), "C": None, "mu": None, "xx": None}
        if getattr(self, "band", 0):
            out["C"] = np.empty((T, M, K))
            out["mu"] = np.empty((M, K))
            out["xx"] = np.empty((M, self.band + 1))
        check(_lib.load().lds_win_plan_cv_outputs(self.handle, 0, ptr(out["meansq"]), ptr(out["C"]),
                                                  ptr(out["mu"]), ptr(out["xx"])))
        return out

    def cv_outputs_device(self, meansq, C_tiles=None, mu=None, xx=None) -> None:
        """Copy the outputs into caller-owned device buffers (integer addresses,
        e.g. torch tensors' data_ptr())."""
        vp = lambda a: None if a is None else C.c_void_p(int(a))
        check(_lib.load().lds_win_plan_cv_outputs(self.handle, 1, vp(meansq), vp(C_tiles), vp(mu),
                                                  vp(xx)))

    def cv_ms(self) -> float:
        x = C.c_double(0.0)
        check(_lib.load().lds_win_plan_cv_ms(self.handle, C.byref(x)))
        return x.value

    def close(self) -> None:
        if self.handle:
            _lib.load().lds_win_plan_destroy(self.handle)
            self.handle = 0

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def windowed_ldscore(bed_rows, n_total: int, annot, window_starts, nvecs: int, step_size: int,
                     seed: int, rand_dist: str = "rademacher", vtile: int | None = None,
                     ddof: int = 1, impute_mode: str = "mean", impute_seed: int = 0,
                     eps: float = 1e-10, as_float: bool = False, row_sel=None, chunks: int = 8,
                     meansq: bool = False, tiling: dict | None = None) -> dict:
    """Windowed + partitioned LD scores in one call from host BED rows.

    Same estimate as ``WinPlan(GwSession(bed_rows, ...), ...)`` (bit for bit),
    with the upload streamed in ``chunks`` window-aligned pieces: the next
    piece's upload and set-up overlap the current piece's kernels.  Pass
    ``bed_rows`` in pinned memory (e.g. a ``pin_memory=True`` torch tensor's
    ``.numpy()``) for full-rate uploads.  Returns ``ldscore`` (M x K) and, with
    ``meansq``, ``meansq_accum`` and ``inv``.  ``tiling`` (``p1_sb_per_cta``,
    e.g. an autotuner record's config) sets the chunks' tiling.
    """
    tiling = tiling or {}
    bed_rows = np.ascontiguousarray(bed_rows, dtype=np.uint8)
    M, row_bytes = bed_rows.shape
    annot = np.ascontiguousarray(annot, dtype=np.float64)
    ws = np.ascontiguousarray(window_starts, dtype=np.int64)
    if annot.ndim != 2 or annot.shape[0] != M:
        raise ValueError("annot must be (M, K) with M = bed_rows.shape[0]")
    K = annot.shape[1]
    ld = np.empty((M, K))
    ms = np.empty((M, K)) if meansq else None
    inv = np.empty(M) if meansq else None
    rows, nr = _rows(row_sel)
    check(_lib.load().lds_win_ldscore(ptr(bed_rows), row_bytes, int(n_total), M, ptr(rows), nr,
                                      ptr(annot), K, ptr(ws), ws.size - 1, int(nvecs),
                                      int(step_size), int(vtile or 0), int(seed), _dist(rand_dist),
                                      int(ddof), _impute(impute_mode), int(impute_seed),
                                      float(eps), int(as_float), int(chunks),
                                      int(tiling.get("p1_sb_per_cta", 0)),
                                      ptr(ld), ptr(ms), ptr(inv)))
    return {"ldscore": ld, "meansq_accum": ms, "inv": inv}


def window_seed(seed: int, w: int) -> int:
    """Probe root seed of window w (same function as the library's)."""
    return int(_lib.load().lds_window_seed(int(seed), int(w)))


def set_stream(stream_ptr: int | None) -> None:
    """Launch library kernels on an external CUDA stream (e.g. torch.cuda.Stream.cuda_stream).

    0 / None restores the library's own stream, so the legacy default stream
    (torch's default stream, handle 0) cannot be selected: use a created stream."""
    check(_lib.load().lds_set_stream(None if not stream_ptr else C.c_void_p(stream_ptr)))
