"""GPU test of lds_phase2_accum_device_noalloc, the phase-2 entry point that
allocates no device memory.

Callers that cannot allocate during this step (graph capture, memory owned by
another framework's pool, allocator-free services) pass their own device
buffers; the library's scratch is a fixed file-scope device array.  This test
plays such a caller: its buffers come from torch, and the entry point's
accumulated LD-score sums are checked against the regular per-block entry
(lds_phase2_accum_XtXz_bed_f64) on the same genotypes, sketch and scales, on
two calls in a row with different sketches (the shared scratch keeps the
previous call's contents, which must not leak into the next result).

The file name sorts last so that a run stopping at the first failure has run
every other test before this one.
"""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

RTOL = 1e-12


def _device_rows(geno: np.ndarray, row_bytes: int) -> np.ndarray:
    """Packed rows in the library's device layout (samples >= n coded 01)."""
    m, n = geno.shape
    codes = np.where(geno < 0, 1, np.array([0, 2, 3], np.uint8)[np.clip(geno, 0, 2)]).astype(np.uint8)
    full = np.ones((m, row_bytes * 4), dtype=np.uint8)
    full[:, :n] = codes
    q = full.reshape(m, row_bytes, 4)
    return (q[:, :, 0] | (q[:, :, 1] << 2) | (q[:, :, 2] << 4) | (q[:, :, 3] << 6)).astype(np.uint8)


def _mean_sdinv(geno: np.ndarray):
    """Per-SNP mean and inverse sd over observed calls, ddof = 1 (mean imputation)."""
    obs = geno >= 0
    g = np.where(obs, geno, 0).astype(np.float64)
    nobs = obs.sum(axis=1).astype(np.float64)
    s = g.sum(axis=1)
    ss = (g * g).sum(axis=1)
    mu = np.where(nobs > 0, s / np.maximum(nobs, 1), 0.0)
    m2 = ss - s * s / np.maximum(nobs, 1)
    m2[(m2 < 0) & (m2 > -1e-12)] = 0.0
    var = np.where((nobs - 1 > 0) & (m2 > 0), m2 / np.maximum(nobs - 1, 1), 0.0)
    sdinv = np.where(var > 0, 1.0 / np.sqrt(np.where(var > 0, var, 1.0)), 1.0)
    return mu, sdinv


def test_noalloc_phase2_matches_regular_entry_on_two_calls(tmp_path):
    import torch

    from summit_b200 import _lib, bedfile, gwldcore

    lib = _lib.load()
    rng = np.random.default_rng(2024)
    n, m, K, V = 333, 410, 2, 24
    geno = bedfile.synth_genotypes(n, m, seed=77)
    prefix = bedfile.write_plink(tmp_path / "noalloc", geno)
    n_pad = ((n + 255) // 256) * 256
    row_bytes = n_pad // 4
    mu, sdinv = _mean_sdinv(geno)
    inv = rng.uniform(0.5, 1.5, size=m)
    denom = float(n - 1)
    left = inv * inv / (denom * denom)

    dev = torch.device("cuda", 0)
    d_codes = torch.from_numpy(_device_rows(geno, row_bytes)).to(dev)
    d_mu = torch.from_numpy(mu).to(dev)
    d_sd = torch.from_numpy(sdinv).to(dev)
    d_left = torch.from_numpy(left).to(dev)

    for call in range(2):
        Y = rng.standard_normal((K * V, n_pad))
        Y[:, n:] = 0.0
        xz = np.asfortranarray(Y[:, :n].T)
        ms_ref = np.zeros((m, K))
        mc_ref = np.zeros((m, K))
        gwldcore.phase2_accum_XtXz_bed(
            bed_prefix=prefix, fam_path=prefix + ".fam", blk_start=0, blk_end=m, ddof=1,
            inv_left=inv, tile_nvecs=V, Xz2d=xz, meansq_accum=ms_ref, N_denom=n,
            impute_mode="mean", mc_per_snp_sumsq=mc_ref)

        d_Y = torch.from_numpy(np.ascontiguousarray(Y)).to(dev)
        d_acc = torch.zeros((m, K), dtype=torch.float64, device=dev)
        d_mc = torch.zeros((m, K), dtype=torch.float64, device=dev)
        rc = lib.lds_phase2_accum_device_noalloc(
            d_codes.data_ptr(), row_bytes, n, m, 0, m, d_Y.data_ptr(), K, V, d_mu.data_ptr(),
            d_sd.data_ptr(), d_left.data_ptr(), d_acc.data_ptr(), d_mc.data_ptr(), None)
        assert rc == 0, lib.lds_last_error().decode()
        torch.cuda.synchronize()
        acc = d_acc.cpu().numpy()
        mc = d_mc.cpu().numpy()
        scale = np.max(np.abs(ms_ref))
        assert np.max(np.abs(acc - ms_ref)) <= RTOL * scale, f"call {call}: LD sums differ"
        assert np.max(np.abs(mc - mc_ref)) <= RTOL * np.max(np.abs(mc_ref)), f"call {call}: MC sums differ"


def test_noalloc_rejects_sizes_beyond_its_scratch():
    import torch

    from summit_b200 import _lib

    lib = _lib.load()
    dev = torch.device("cuda", 0)
    n, row_bytes, K, V = 200_000, 50_048, 8, 64  # ~102 MB of digits > 16 MiB
    d_codes = torch.zeros(row_bytes * 4, dtype=torch.uint8, device=dev)
    dummy = torch.zeros(8, dtype=torch.float64, device=dev)
    rc = lib.lds_phase2_accum_device_noalloc(
        d_codes.data_ptr(), row_bytes, n, 4, 0, 4, dummy.data_ptr(), K, V, dummy.data_ptr(),
        dummy.data_ptr(), dummy.data_ptr(), dummy.data_ptr(), None, None)
    assert rc == -1
    assert "scratch" in lib.lds_last_error().decode()
