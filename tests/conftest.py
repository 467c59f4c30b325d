"""Shared fixtures.  GPU tests are marked ``gpu``; everything else runs on CPU."""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and liblds.so")


@pytest.fixture(scope="session")
def oracle():
    from oracle.oracle import Oracle

    return Oracle()


@pytest.fixture(scope="session")
def reference():
    from oracle.oracle import REF_SO, Reference

    if not REF_SO.exists():
        pytest.skip("reference checker oracle/_ref/libref_gwld.so not built (make -C oracle ref)")
    return Reference()


@pytest.fixture(scope="session")
def small_bed(tmp_path_factory):
    """Synthetic BED fileset: 333 samples x 410 SNPs with 1% missing."""
    from summit_b200 import bedfile

    n, m = 333, 410
    geno = bedfile.synth_genotypes(n, m, seed=424242)
    prefix = bedfile.write_plink(tmp_path_factory.mktemp("bed") / "small", geno)
    return {"prefix": prefix, "n": n, "m": m, "geno": geno, "rows": bedfile.pack_bed_rows(geno)}


def rel_err(a, b) -> float:
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def assert_rel_elementwise(got, ref, rtol: float, what: str = "", atol_frac: float = 1e-12):
    """Per-element relative bound |got - ref| <= rtol |ref| + atol_frac max|ref|.

    The absolute floor only covers exact zeros (monomorphic or all-missing
    SNPs, whose sums of squares are 0 on both sides) and values within
    rounding of zero; every other element is held to the relative bound."""
    got = np.asarray(got, dtype=np.float64)
    ref = np.asarray(ref, dtype=np.float64)
    assert got.shape == ref.shape, (got.shape, ref.shape)
    assert np.isfinite(got).all() == np.isfinite(ref).all(), f"{what}: finiteness differs"
    scale = float(np.max(np.abs(ref))) if ref.size else 0.0
    bound = rtol * np.abs(ref) + atol_frac * scale
    err = np.abs(got - ref)
    bad = np.flatnonzero(err > bound)
    if bad.size:
        i = bad[np.argmax((err / np.maximum(np.abs(ref), 1e-300)).ravel()[bad])]
        raise AssertionError(
            f"{what}: {bad.size} of {ref.size} elements beyond {rtol:g} relative; worst at flat "
            f"index {i}: got {got.ravel()[i]!r}, ref {ref.ravel()[i]!r}")


def max_rel_elementwise(got, ref) -> float:
    """max |got - ref| / |ref| over the elements with ref != 0."""
    got = np.asarray(got, dtype=np.float64)
    ref = np.asarray(ref, dtype=np.float64)
    nz = ref != 0
    if not nz.any():
        return 0.0
    return float(np.max(np.abs(got[nz] - ref[nz]) / np.abs(ref[nz])))


def dropin_gw_ldscore(mod, prefix, n, m, annot, nvecs, step, seed, dist, impute, dtype, vtile,
                      impute_seed=4):
    """The native call sequence of GenomewideLDScore._compute_ldscore
    (gw_ldscore.py:1753-2222, no covariates) against module `mod` (the
    drop-in per-block functions)."""
    from oracle.oracle import bounded_vtile_sizes, compute_blocks

    annot = np.ascontiguousarray(annot, dtype=dtype)
    K = annot.shape[1]
    blocks = compute_blocks(m, step)
    vt = bounded_vtile_sizes(nvecs, vtile)
    inv = np.empty(m, dtype=dtype)
    meansq = np.zeros((m, K), dtype=dtype)
    mc_agg = np.zeros(K)
    mc_snp = np.zeros((m, K))
    kmax = [int((annot[s:e] != 0).sum(axis=0).max()) for (s, e) in blocks]
    v0 = 0
    for ti, V in enumerate(vt):
        Xz = np.empty((n, K * V), dtype=dtype, order="F")
        init = np.zeros(K, dtype=np.uint8)
        for bi, (s, e) in enumerate(blocks):
            mod.phase1_compute_Xz_bed_chunk(
                bed_prefix=prefix, fam_path=prefix + ".fam", blk_start=s, blk_end=e,
                row_sel=None, ddof=1, annot_blk=annot[s:e], inv_right=inv[s:e], v_start=v0,
                v_count=V, kmax_hint=kmax[bi], rand_dist=dist, seed=seed, Xz2d_chunk=Xz,
                bin_init_mask=init, impute_mode=impute, impute_seed=impute_seed,
                inv_out=inv[s:e] if ti == 0 else None)
        for k in np.flatnonzero(init == 0):
            Xz[:, k * V:(k + 1) * V] = 0
        for (s, e) in blocks:
            mod.phase2_accum_XtXz_bed(
                bed_prefix=prefix, fam_path=prefix + ".fam", blk_start=s, blk_end=e, row_sel=None,
                ddof=1, inv_left=inv[s:e], tile_nvecs=V, Xz2d=Xz, meansq_accum=meansq,
                mc_aggregate_sumsq=mc_agg, mc_per_snp_sumsq=mc_snp, C=None, R=None, N_denom=n,
                impute_mode=impute, impute_seed=impute_seed)
        v0 += V
    return {"meansq": meansq, "inv": inv, "mc_agg": mc_agg, "mc_snp": mc_snp}
