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

    def results(self) -> dict:
        M, K = self.M, self.K
        ld = np.empty((M, K))
        ms = np.empty((M, K))
        inv = np.empty(M)
        mcp = np.empty((M, K)) if self.with_mc else None
        check(_lib.load().lds_win_plan_results(self.handle, ptr(ld), ptr(ms), ptr(inv), ptr(mcp)))
        return {"ldscore": ld, "meansq_accum": ms, "inv": inv, "mc_per_snp_sumsq": mcp}

    def kernel_ms(self) -> dict:
        buf = np.zeros(4)
        check(_lib.load().lds_win_plan_kernel_ms(self.handle, ptr(buf)))
        return {"weights": buf[0], "phase1": buf[1], "digits": buf[2], "phase2": buf[3]}

    def close(self) -> None:
        if self.handle:
            _lib.load().lds_win_plan_destroy(self.handle)
            self.handle = 0

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def window_seed(seed: int, w: int) -> int:
    """Probe root seed of window w (same function as the library's)."""
    return int(_lib.load().lds_window_seed(int(seed), int(w)))


def set_stream(stream_ptr: int | None) -> None:
    """Launch library kernels on an external CUDA stream (e.g. torch.cuda.Stream.cuda_stream)."""
    check(_lib.load().lds_set_stream(None if not stream_ptr else C.c_void_p(stream_ptr)))
