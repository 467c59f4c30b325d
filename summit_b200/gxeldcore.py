"""Drop-in replacement for the SUMMIT-GxE products of SUMMIT's native
``gxeldcore`` module, backed by liblds.so.

``MultiEnvironmentKernel`` keeps the reference's constructor arguments, method
names, argument order, array layouts (column-major panels and genotype-side
arrays, row-major ``(E * total_variants) x K`` score accumulators) and error
messages (``src/native/gxeldcore.cpp:16420-16474``).  ``source_block`` and
``target_score_block`` take the ``genotype`` argument in either of two forms:

* the reference's own: a dense N x L FP64 block of standardized genotypes (the
  reference's driver passes ``np.asfortranarray(genotype, dtype=np.float64)``,
  ``gxe_multi.py:3066-3230``), multiplied as FP64 GEMMs on the device; or
* a block of a resident genotype image (``GwSession.block(start, stop)``),
  multiplied on the int8 tensor cores straight from the packed codes - the
  role the reference's packed-genotype variants give a MailmanPackedBlock.  Its
  standardization is the image's (mean imputation, its ddof), which is what the
  reference's driver decodes into its dense blocks.

``prepare_protected_row_weighted_pair`` and ``numpy_philox_rademacher_block``
mirror the module functions of the same names.  There is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import check, ptr


class GenotypeBlock:
    """SNPs [start, stop) of a resident genotype image (GwSession)."""

    def __init__(self, session, start: int, stop: int):
        if not (0 <= start < stop <= session.M):
            raise ValueError("genotype block outside the image")
        self.session, self.start, self.stop = session, int(start), int(stop)

    @property
    def shape(self):
        return (self.session.N, self.stop - self.start)


class ProtectedRightPair:
    """Immutable [right, row_weight o right] target operand (snapshot of the
    inputs; sealed on the device at its first use)."""

    def __init__(self, right, row_weights):
        self._right = np.array(right, dtype=np.float64, order="F", copy=True)
        self._weights = np.array(row_weights, dtype=np.float64, order="F", copy=True)
        self._handles = {}

    @property
    def rows(self) -> int:
        return int(self._right.shape[0])

    @property
    def columns(self) -> int:
        return int(self._right.shape[1])

    def _handle(self, gxe: int) -> int:
        h = self._handles.get(gxe)
        if h is None:
            out = C.c_int64(0)
            check(_lib.load().lds_gxe_pair_create(gxe, ptr(self._right), self.columns,
                                                  ptr(self._weights), self._weights.shape[1], 0,
                                                  C.byref(out)))
            h = self._handles[gxe] = out.value
        return h

    def __del__(self):
        try:
            for h in self._handles.values():
                _lib.load().lds_gxe_pair_destroy(h)
        except Exception:
            pass


def prepare_protected_row_weighted_pair(right, row_weights, threads):
    right = np.asarray(right)
    row_weights = np.asarray(row_weights)
    if (right.ndim != 2 or row_weights.ndim != 2 or right.shape[0] != row_weights.shape[0]
            or row_weights.shape[1] <= 0 or right.shape[1] % row_weights.shape[1] != 0):
        raise RuntimeError("Protected GxE right-pair inputs have incompatible dimensions")
    return ProtectedRightPair(right, row_weights)


def numpy_philox_rademacher_block(keys, rows, threads):
    """Rows x P (column-major) +-1 probes of NumPy's Philox streams with the
    given keys (P x 2 uint64), as Generator(Philox).integers(0, 2) yields them."""
    keys = np.ascontiguousarray(keys, dtype=np.uint64)
    if keys.ndim != 2 or keys.shape[1] != 2:
        raise RuntimeError("Native Philox Rademacher inputs are invalid")
    out = np.empty((int(rows), keys.shape[0]), dtype=np.float64, order="F")
    check(_lib.load().lds_philox_rademacher(ptr(keys), keys.shape[0], int(rows), ptr(out), 0))
    return out


def _f64f(a, name):
    a = np.asarray(a)
    if a.dtype != np.float64:
        raise TypeError(f"incompatible function arguments: {name} must be float64")
    return np.asfortranarray(a)


def _rw(a, order, name):
    if not isinstance(a, np.ndarray) or a.dtype != np.float64 or not a.flags.writeable:
        raise TypeError(f"incompatible function arguments: {name} must be a writable float64 array")
    if not (a.flags.f_contiguous if order == "F" else a.flags.c_contiguous):
        raise TypeError(f"incompatible function arguments: {name} has the wrong memory order")
    return a


class MultiEnvironmentKernel:
    def __init__(self, environments, feature_basis, feature_power_indices,
                 feature_power_offsets, feature_ranks, feature_gram_values, feature_gram_offsets,
                 feature_e2_gram_values, common_basis, directions, ddof, annotation_bins, threads):
        env = _f64f(environments, "environments")
        fb = _f64f(feature_basis, "feature_basis")
        cb = _f64f(common_basis, "common_basis")
        dr = _f64f(directions, "directions")
        n, E = env.shape
        if (n <= 2 or E <= 0 or fb.shape[1] <= 0 or ddof < 0 or ddof >= n or annotation_bins <= 0
                or fb.shape[0] != n or cb.shape[0] != n or dr.shape != (n, E)):
            raise RuntimeError("Multi-environment native kernel inputs have incompatible dimensions")
        pidx = np.ascontiguousarray(feature_power_indices, dtype=np.int64)
        poff = np.ascontiguousarray(feature_power_offsets, dtype=np.int64)
        ranks = np.ascontiguousarray(feature_ranks, dtype=np.int32)
        goff = np.ascontiguousarray(feature_gram_offsets, dtype=np.int64)
        gv = np.asarray(feature_gram_values, dtype=np.float64)
        e2 = np.asarray(feature_e2_gram_values, dtype=np.float64)
        if (ranks.shape != (E,) or poff.shape != (4 * E + 1,) or goff.shape != (E + 1,)
                or gv.shape != e2.shape):
            raise RuntimeError("Multi-environment native feature metadata has incompatible dimensions")
        if poff[0] != 0 or poff[-1] != pidx.size or goff[0] != 0 or goff[-1] != gv.size:
            raise RuntimeError("Multi-environment native feature offsets do not span their buffers")
        for name, a in (("environment", env), ("feature basis", fb), ("common basis", cb),
                        ("direction", dr)):
            if not np.all(np.isfinite(a)):
                raise RuntimeError(f"Multi-environment native {name} contains NaN or infinity")
        self._env, self._fb, self._cb, self._dr = env, fb, cb, dr
        self._pidx, self._poff, self._ranks = pidx, poff, ranks
        self._rows, self._E, self._bins, self._ddof = n, E, int(annotation_bins), int(ddof)
        self._threads = int(threads)
        self._handles = {}  # genotype-image handle -> GxE context handle

    def info(self) -> dict:
        return {"schema": "summit.multi_environment_native_kernel.v1", "schema_version": 1,
                "rows": self._rows, "environment_count": self._E,
                "annotation_bins": self._bins, "feature_basis_columns": self._fb.shape[1],
                "common_basis_rank": self._cb.shape[1], "ddof": self._ddof,
                "threads": self._threads, "backend": "liblds sm_100a"}

    def _ctx(self, session) -> int:
        h = self._handles.get(session.handle)
        if h is None:
            if session.N != self._rows:
                raise RuntimeError("Multi-environment native source genotype rows do not match")
            out = C.c_int64(0)
            check(_lib.load().lds_gxe_create(
                session.handle, self._E, ptr(self._env), self._cb.shape[1],
                ptr(self._cb) if self._cb.shape[1] else None, ptr(self._dr), self._fb.shape[1],
                ptr(self._fb), ptr(self._pidx), ptr(self._poff), ptr(self._ranks), self._bins,
                C.byref(out)))
            h = self._handles[session.handle] = out.value
        return h

    def _dense_ctx(self) -> int:
        h = self._handles.get("dense")
        if h is None:
            out = C.c_int64(0)
            check(_lib.load().lds_gxe_create_dense(
                self._rows, self._E, ptr(self._env), self._cb.shape[1],
                ptr(self._cb) if self._cb.shape[1] else None, ptr(self._dr), self._fb.shape[1],
                ptr(self._fb), ptr(self._pidx), ptr(self._poff), ptr(self._ranks), self._bins,
                C.byref(out)))
            h = self._handles["dense"] = out.value
        return h

    def _dense(self, genotype):
        """The reference's dense genotype argument (N x L, float64), or None
        for a resident-image block."""
        if isinstance(genotype, GenotypeBlock):
            return None
        if not isinstance(genotype, np.ndarray) or genotype.dtype != np.float64 \
                or genotype.ndim != 2:
            raise TypeError("incompatible function arguments: genotype must be a float64 "
                            "(N, L) array or a resident-image block (GwSession.block)")
        if genotype.shape[0] != self._rows:
            raise RuntimeError("Multi-environment native source genotype rows do not match")
        return np.asfortranarray(genotype)

    def source_block(self, target, genotype, probes, annotation, scale_x, scale_w,
                     environment_start, annotation_is_sqrt=False) -> int:
        dense = self._dense(genotype)
        L = dense.shape[1] if dense is not None else genotype.stop - genotype.start
        target = _rw(target, "F", "target")
        z = _f64f(probes, "probes")
        a = _f64f(annotation, "annotation")
        sx, sw = _f64f(scale_x, "scale_x"), _f64f(scale_w, "scale_w")
        B, T = z.shape[1], sx.shape[1]
        if (B <= 0 or T <= 0 or environment_start < 0 or environment_start + T > self._E
                or z.shape[0] != L or a.shape != (L, self._bins) or sx.shape[0] != L
                or sw.shape != sx.shape):
            raise RuntimeError("Multi-environment native source inputs have incompatible dimensions")
        if target.shape != (self._rows, 2 * T * self._bins * B):
            raise RuntimeError("Multi-environment native packed source target is mis-sized")
        if dense is not None:
            check(_lib.load().lds_gxe_source_block_dense(
                self._dense_ctx(), ptr(dense), L, ptr(z), B, ptr(a), int(bool(annotation_is_sqrt)),
                ptr(sx), ptr(sw), T, int(environment_start), ptr(target), 0))
            return 0
        check(_lib.load().lds_gxe_source_block(
            self._ctx(genotype.session), genotype.start, genotype.stop, ptr(z), B, ptr(a),
            int(bool(annotation_is_sqrt)), ptr(sx), ptr(sw), T, int(environment_start),
            ptr(target), 0))
        return 0

    def project_sources(self, panel, columns_per_environment, environment_start):
        panel = _rw(panel, "F", "panel")
        if panel.shape[0] != self._rows:
            raise RuntimeError("Multi-environment native projection panel is mis-sized")
        h = next(iter(self._handles.values())) if self._handles else self._dense_ctx()
        tile = panel.shape[1] // (2 * max(int(columns_per_environment), 1))
        leak = np.empty(max(tile, 1))
        check(_lib.load().lds_gxe_project_sources(h, ptr(panel), panel.shape[1],
                                                  int(columns_per_environment),
                                                  int(environment_start), ptr(leak), 0))
        return leak[:tile]

    def target_score_block(self, genotype, right_pair, scale_x, scale_w, accum_xx, accum_xw,
                           accum_wx, accum_ww, block_start, total_variants, probe_count,
                           environment_start) -> int:
        dense = self._dense(genotype)
        L = dense.shape[1] if dense is not None else genotype.stop - genotype.start
        sx, sw = _f64f(scale_x, "scale_x"), _f64f(scale_w, "scale_w")
        accs = [_rw(x, "C", n) for x, n in ((accum_xx, "accum_xx"), (accum_xw, "accum_xw"),
                                             (accum_wx, "accum_wx"), (accum_ww, "accum_ww"))]
        T = sx.shape[1]
        if (block_start < 0 or total_variants <= 0 or block_start + L > total_variants
                or probe_count <= 0 or T <= 0 or environment_start < 0
                or environment_start + T > self._E or sx.shape[0] != L or sw.shape != sx.shape):
            raise RuntimeError("Multi-environment native target scale/block metadata is invalid")
        if not isinstance(right_pair, ProtectedRightPair) or right_pair.rows != self._rows or \
                right_pair.columns != T * 2 * self._bins * probe_count:
            raise RuntimeError("Multi-environment native target pair is incompatible with the tile")
        for x in accs:
            if x.shape != (self._E * total_variants, self._bins):
                raise RuntimeError("Multi-environment native score accumulator is mis-sized")
        if dense is not None:
            h = self._dense_ctx()
            check(_lib.load().lds_gxe_target_score_block_dense(
                h, ptr(dense), L, right_pair._handle(h), ptr(sx), ptr(sw), T, ptr(accs[0]),
                ptr(accs[1]), ptr(accs[2]), ptr(accs[3]), int(block_start), int(total_variants),
                int(probe_count), int(environment_start), 0))
            return 0
        h = self._ctx(genotype.session)
        check(_lib.load().lds_gxe_target_score_block(
            h, genotype.start, genotype.stop, right_pair._handle(h), ptr(sx), ptr(sw), T,
            ptr(accs[0]), ptr(accs[1]), ptr(accs[2]), ptr(accs[3]), int(block_start),
            int(total_variants), int(probe_count), int(environment_start), 0))
        return 0

    def normalize_scores(self, accum_xx, accum_xw, accum_wx, accum_ww, probe_count) -> None:
        if probe_count <= 0:
            raise RuntimeError("Multi-environment native score normalization requires probes")
        accs = [_rw(x, "C", "accum") for x in (accum_xx, accum_xw, accum_wx, accum_ww)]
        rows, cols = accs[0].shape
        if rows <= 0 or rows % self._E != 0 or cols != self._bins:
            raise RuntimeError("Multi-environment native score normalization shape is invalid")
        if any(x.shape != accs[0].shape for x in accs[1:]):
            raise RuntimeError("Multi-environment native score accumulators disagree")
        check(_lib.load().lds_gxe_normalize_scores(ptr(accs[0]), ptr(accs[1]), ptr(accs[2]),
                                                   ptr(accs[3]), rows, cols, int(probe_count), 0))

    def __del__(self):
        try:
            for h in self._handles.values():
                _lib.load().lds_gxe_destroy(h)
        except Exception:
            pass


# ---------------------------------------------------------------------------
# Generalized per-SNP GxE products (GeneralizedGxELDScoreDirectContext::
# packed_source_product / packed_target_product, generalized_gxe_variant.inc:
# 1749-1988): mean-imputed genotypes scaled by the Mailman mean pack's
# sqrt((N - ddof) / M2_j), with the reference's sign convention.
# ---------------------------------------------------------------------------
def generalized_source_product(genotype: GenotypeBlock, rhs) -> np.ndarray:
    """-X' rhs: rhs (L x columns) -> N x columns (column-major)."""
    rhs = np.asfortranarray(rhs, dtype=np.float64)
    L = genotype.stop - genotype.start
    if rhs.ndim != 2 or rhs.shape[0] != L or rhs.shape[1] <= 0:
        raise RuntimeError("Generalized packed source product is mis-sized")
    out = np.empty((genotype.session.N, rhs.shape[1]), order="F")
    check(_lib.load().lds_generalized_source_product(
        genotype.session.handle, genotype.start, genotype.stop, ptr(rhs), rhs.shape[1], ptr(out)))
    return out


def generalized_target_product(genotype: GenotypeBlock, rhs) -> np.ndarray:
    """-X'^T rhs: rhs (N x columns) -> L x columns (column-major)."""
    rhs = np.asfortranarray(rhs, dtype=np.float64)
    if rhs.ndim != 2 or rhs.shape[0] != genotype.session.N or rhs.shape[1] <= 0:
        raise RuntimeError("Generalized packed target product is mis-sized")
    out = np.empty((genotype.stop - genotype.start, rhs.shape[1]), order="F")
    check(_lib.load().lds_generalized_target_product(
        genotype.session.handle, genotype.start, genotype.stop, ptr(rhs), rhs.shape[1], ptr(out)))
    return out
