"""Whole-genome SUMMIT-GxE reference products on one resident genotype image.

The reference builds its multi-environment references block by block from the
host (``generate_multi_environment_references``, gxe_multi.py:6509, calling
MultiEnvironmentKernel.source_block / project_sources / target_score_block /
normalize_scores).  ``GxeReference.run`` performs the same sequence for all
SNPs with every panel resident on the device (liblds's C ABI with device
pointers): source over all SNPs, projection of the source panel, the sealed
[S, phi o S] pair, the target scores, and the division by the probe count.
torch only provides device memory.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import check
from .gxeldcore import MultiEnvironmentKernel


def _dp(t):
    return C.c_void_p(int(t.data_ptr()))


class GxeReference:
    def __init__(self, session, environments, feature_basis, power_indices, power_offsets, ranks,
                 gram_values, gram_offsets, e2_gram_values, common_basis, directions,
                 annotation_bins: int = 1, ddof: int = 1, product_checks: bool = False):
        self.session = session
        self.kernel = MultiEnvironmentKernel(environments, feature_basis, power_indices,
                                             power_offsets, ranks, gram_values, gram_offsets,
                                             e2_gram_values, common_basis, directions, ddof,
                                             annotation_bins, 1)
        self.h = self.kernel._ctx(session)
        if product_checks:
            # exact checksums of the target's tensor-core products, compared
            # on the host after every target call (a mismatch raises)
            check(_lib.load().lds_gxe_set_checks(self.h, 1))
        self.E = self.kernel._E
        self.K = int(annotation_bins)
        self.env = np.asfortranarray(environments, dtype=np.float64)
        self.timings = {}

    def run(self, probes, annotation, scale_x, scale_w, environment_start: int = 0,
            tile: int | None = None) -> dict:
        """probes (M x B), annotation (M x K), scale_x / scale_w (M x tile):
        torch CUDA tensors in column-major storage (shape (cols, M) row-major
        tensors transposed, i.e. ``t.T`` of a contiguous (cols, M) tensor).
        Returns the four normalized score accumulators ((E M) x K, torch) and
        the projection leakages."""
        import torch

        lib = _lib.load()
        sess = self.session
        M, N, K = sess.M, sess.N, self.K
        T = self.E - environment_start if tile is None else int(tile)
        B = probes.shape[1]
        cols = T * 2 * K * B
        dev = probes.device
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(5)]
        panel = torch.zeros((cols, N), dtype=torch.float64, device=dev)  # N x cols, column-major
        w = torch.from_numpy(self.env[:, environment_start:environment_start + T].T.copy()).to(dev)
        accs = torch.zeros((4, self.E * M, K), dtype=torch.float64, device=dev)
        leak = np.zeros(T)
        torch.cuda.synchronize()
        ev[0].record()
        check(lib.lds_gxe_source_block(self.h, 0, M, _dp(probes), B, _dp(annotation), 0,
                                       _dp(scale_x), _dp(scale_w), T, environment_start,
                                       _dp(panel), 1))
        ev[1].record()
        check(lib.lds_gxe_project_sources(self.h, _dp(panel), cols, K * B, environment_start,
                                          leak.ctypes.data_as(C.c_void_p), 1))
        ev[2].record()
        pair = C.c_int64(0)
        check(lib.lds_gxe_pair_create(self.h, _dp(panel), cols, _dp(w), T, 1, C.byref(pair)))
        del panel
        ev[3].record()
        try:
            check(lib.lds_gxe_target_score_block(
                self.h, 0, M, pair.value, _dp(scale_x), _dp(scale_w), T, _dp(accs[0]),
                _dp(accs[1]), _dp(accs[2]), _dp(accs[3]), 0, M, B, environment_start, 1))
            check(lib.lds_gxe_normalize_scores(_dp(accs[0]), _dp(accs[1]), _dp(accs[2]),
                                               _dp(accs[3]), self.E * M, K, B, 1))
        finally:
            lib.lds_gxe_pair_destroy(pair.value)
        ev[4].record()
        torch.cuda.synchronize()
        names = ["source", "project", "pair", "target"]
        self.timings = {n: ev[i].elapsed_time(ev[i + 1]) for i, n in enumerate(names)}
        self.timings["total"] = ev[0].elapsed_time(ev[4])
        return {"accum_xx": accs[0], "accum_xw": accs[1], "accum_wx": accs[2],
                "accum_ww": accs[3], "leakages": leak, "timings": dict(self.timings)}

    def last_check(self, vectors: bool = False) -> dict:
        """The last target call's product check: rows checked, mismatching
        SNPs and the first of them, and with ``vectors`` the per-SNP checksum
        pairs (rows x 2 each: tensor-core epilogue, CUDA-core recomputation)."""
        lib = _lib.load()
        first_row, rows, bad, first = (C.c_int64(0) for _ in range(4))
        check(lib.lds_gxe_last_check(self.h, None, None, C.byref(first_row), C.byref(rows),
                                     C.byref(bad), C.byref(first)))
        out = {"first_row": first_row.value, "rows": rows.value, "mismatches": bad.value,
               "first_snp": first.value}
        if vectors:
            lhs = np.zeros((rows.value, 2), dtype=np.uint64)
            rhs = np.zeros((rows.value, 2), dtype=np.uint64)
            check(lib.lds_gxe_last_check(self.h, lhs.ctypes.data_as(C.c_void_p),
                                         rhs.ctypes.data_as(C.c_void_p), None, None, None, None))
            out["lhs"], out["rhs"] = lhs, rhs
        return out

    def close(self):
        self.kernel = None


def synthetic_design(n: int, E: int, seed: int = 0, n_cov: int = 1, categorical: int = 0):
    """Self-consistent kernel inputs: environments (E - categorical continuous
    N(0,1) with pairwise correlation 0.2, then ``categorical`` level-coded
    exposures with 3, 5, ... levels, each standardized), a common basis of the
    intercept and ``n_cov`` covariates, unit directions of the environments
    orthogonal to it, and per environment the fixed-effect basis [U, d_e]
    (feature power ranges all point at it; Grams are identities)."""
    rng = np.random.default_rng(seed)
    Ec = E - categorical
    cov = np.full((Ec, Ec), 0.2) + 0.8 * np.eye(Ec)
    envs = [rng.multivariate_normal(np.zeros(Ec), cov, size=n)] if Ec else []
    for c in range(categorical):
        levels = 3 + 2 * c
        x = rng.integers(0, levels, size=n).astype(np.float64)
        envs.append(((x - x.mean()) / x.std())[:, None])
    env = np.asfortranarray(np.hstack(envs))
    Xc = np.column_stack([np.ones(n)] + [rng.normal(size=n) for _ in range(n_cov)])
    U = np.linalg.qr(Xc)[0]
    D = env - U @ (U.T @ env)
    D /= np.linalg.norm(D, axis=0)
    r = U.shape[1]
    feature_basis = np.asfortranarray(np.hstack([U, D]))
    rank = r + 1
    pidx, poff = [], [0]
    for e in range(E):
        cols = list(range(r)) + [r + e]
        for _ in range(4):
            pidx += cols
            poff.append(len(pidx))
    gram = np.concatenate([np.eye(rank).ravel() for _ in range(E)])
    goff = np.arange(E + 1, dtype=np.int64) * rank * rank
    fixed = [np.hstack([U, D[:, [e]]]) for e in range(E)]
    return {"environments": env, "feature_basis": feature_basis,
            "power_indices": np.asarray(pidx, np.int64), "power_offsets": np.asarray(poff, np.int64),
            "ranks": np.full(E, rank, np.int32), "gram_values": gram, "gram_offsets": goff,
            "e2_gram_values": gram.copy(), "common_basis": np.asfortranarray(U),
            "directions": np.asfortranarray(D), "fixed_bases": fixed}
