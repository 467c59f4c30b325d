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
            d_sd.data_ptr(), d_left.data_ptr(), d_acc.data_ptr(), d_mc.data_ptr(), None, None,
            None)
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
        dummy.data_ptr(), dummy.data_ptr(), dummy.data_ptr(), None, None, None, None)
    assert rc == -1
    assert "scratch" in lib.lds_last_error().decode()


def test_noalloc_subrange_without_mc_and_status_words(tmp_path):
    """Rows [j0, j1) strictly inside the image, no fourth-moment output, and
    the asynchronous form that reports the kernel's status and guard counts
    into caller-owned device words.  The output block holds (j1 - j0) x K
    values; a guard band after it must stay untouched."""
    import torch

    from summit_b200 import _lib, bedfile, gwldcore

    lib = _lib.load()
    rng = np.random.default_rng(99)
    n, m, K, V = 401, 520, 3, 17
    j0, j1 = 130, 389  # neither a tile multiple
    geno = bedfile.synth_genotypes(n, m, seed=5150)
    prefix = bedfile.write_plink(tmp_path / "noalloc_sub", geno)
    n_pad = ((n + 255) // 256) * 256
    row_bytes = n_pad // 4
    mu, sdinv = _mean_sdinv(geno)
    inv = rng.uniform(0.5, 1.5, size=m)
    left = inv * inv / float(n - 1) ** 2

    Y = rng.standard_normal((K * V, n_pad))
    Y[:, n:] = 0.0
    ms_ref = np.zeros((m, K))
    gwldcore.phase2_accum_XtXz_bed(
        bed_prefix=prefix, fam_path=prefix + ".fam", blk_start=0, blk_end=m, ddof=1,
        inv_left=inv, tile_nvecs=V, Xz2d=np.asfortranarray(Y[:, :n].T), meansq_accum=ms_ref,
        N_denom=n, impute_mode="mean")

    dev = torch.device("cuda", 0)
    d_codes = torch.from_numpy(_device_rows(geno, row_bytes)).to(dev)
    d_mu = torch.from_numpy(mu).to(dev)
    d_sd = torch.from_numpy(sdinv).to(dev)
    d_left = torch.from_numpy(left).to(dev)
    d_Y = torch.from_numpy(np.ascontiguousarray(Y)).to(dev)
    rows = j1 - j0
    band = 64
    d_acc = torch.full((rows * K + band,), 7.0, dtype=torch.float64, device=dev)
    d_acc[: rows * K] = 0.0
    d_status = torch.full((1,), 12345, dtype=torch.int32, device=dev)
    d_guards = torch.full((2,), 99, dtype=torch.int64, device=dev)
    rc = lib.lds_phase2_accum_device_noalloc(
        d_codes.data_ptr(), row_bytes, n, m, j0, j1, d_Y.data_ptr(), K, V, d_mu.data_ptr(),
        d_sd.data_ptr(), d_left.data_ptr(), d_acc.data_ptr(), None, d_status.data_ptr(),
        d_guards.data_ptr(), None)
    assert rc == 0, lib.lds_last_error().decode()
    torch.cuda.synchronize()
    acc = d_acc.cpu().numpy()
    assert int(d_status.item()) == 0
    assert d_guards.cpu().tolist() == [0, 0]
    np.testing.assert_array_equal(acc[rows * K:], 7.0)  # nothing written past the block
    got = acc[: rows * K].reshape(rows, K)
    ref = ms_ref[j0:j1]
    assert np.all(np.abs(got - ref) <= RTOL * np.abs(ref) + 1e-300)


def test_noalloc_reports_dropped_nonfinite_updates(tmp_path):
    """A non-finite sketch column makes every update of its bin non-finite;
    both entries drop them, and the no-allocation entry reports the count
    (one per SNP row of the bin) in the caller's guard words."""
    import torch

    from summit_b200 import _lib, bedfile, gwldcore

    lib = _lib.load()
    rng = np.random.default_rng(7)
    n, m, K, V = 300, 200, 2, 8
    geno = bedfile.synth_genotypes(n, m, seed=404)
    prefix = bedfile.write_plink(tmp_path / "noalloc_nan", geno)
    n_pad = ((n + 255) // 256) * 256
    row_bytes = n_pad // 4
    mu, sdinv = _mean_sdinv(geno)
    inv = np.ones(m)
    left = inv / float(n - 1) ** 2
    Y = rng.standard_normal((K * V, n_pad))
    Y[:, n:] = 0.0
    Y[V + 3, 17] = np.nan  # bin 1, probe 3
    ms_ref = np.zeros((m, K))
    gwldcore.phase2_accum_XtXz_bed(
        bed_prefix=prefix, fam_path=prefix + ".fam", blk_start=0, blk_end=m, ddof=1,
        inv_left=inv, tile_nvecs=V, Xz2d=np.asfortranarray(Y[:, :n].T), meansq_accum=ms_ref,
        N_denom=n, impute_mode="mean")
    dev = torch.device("cuda", 0)
    d_acc = torch.zeros((m, K), dtype=torch.float64, device=dev)
    d_status = torch.zeros(1, dtype=torch.int32, device=dev)
    d_guards = torch.zeros(2, dtype=torch.int64, device=dev)
    args = [torch.from_numpy(x).to(dev) for x in (_device_rows(geno, row_bytes), mu, sdinv, left,
                                                   np.ascontiguousarray(Y))]
    rc = lib.lds_phase2_accum_device_noalloc(
        args[0].data_ptr(), row_bytes, n, m, 0, m, args[4].data_ptr(), K, V, args[1].data_ptr(),
        args[2].data_ptr(), args[3].data_ptr(), d_acc.data_ptr(), None, d_status.data_ptr(),
        d_guards.data_ptr(), None)
    assert rc == 0, lib.lds_last_error().decode()
    torch.cuda.synchronize()
    assert int(d_status.item()) == 0
    assert d_guards.cpu().tolist() == [m, 0]
    acc = d_acc.cpu().numpy()
    np.testing.assert_array_equal(acc[:, 1], 0.0)
    np.testing.assert_array_equal(ms_ref[:, 1], 0.0)
    assert np.all(np.abs(acc[:, 0] - ms_ref[:, 0]) <= RTOL * np.abs(ms_ref[:, 0]) + 1e-300)
