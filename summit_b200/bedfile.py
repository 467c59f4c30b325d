"""PLINK BED/BIM/FAM writing and the seeded synthetic genotype generator.

The BED layout follows the PLINK 1 SNP-major format the reference reads
(``src/native/common/genotype.cpp:350-410``: magic ``6C 1B 01``; each SNP is a
row of ``ceil(N/4)`` bytes, sample ``i`` in bits ``2*(i%4)`` of byte ``i//4``).
Two-bit codes decode as the reference does (``genotype.cpp:135-140``):
``00 -> 0``, ``10 -> 1``, ``11 -> 2``, ``01 -> missing``.

The synthetic generator is defined with integer arithmetic only, so the numpy
version here and the CUDA version in ``csrc/lds_synth.cu`` produce identical
bytes.  Per SNP ``j`` and sample ``i``:

* allele frequency ``p_j = 0.05 + 0.45 * U(hash(seed, 1, 0, j))``;
* innovation ``e_ij`` = centred sum of the four 16-bit fields of
  ``hash(seed, 2, i, j)`` (Irwin-Hall, sd ``SD_E``);
* latent AR(1): ``u_i0 = e_i0``, ``u_ij = (58982 u_i,j-1 + 28567 e_ij) >> 16``
  (rho = 0.9, sqrt(1-rho^2) in Q16, stationary sd = ``SD_E``);
* hard call by thresholding at the Gaussian quantiles of the HWE
  Binomial(2, p_j) cell probabilities ``(1-p)^2`` and ``1-p^2``;
* missing completely at random with probability 1% from ``hash(seed, 3, i, j)``.
"""
from __future__ import annotations

import os
from pathlib import Path

import numpy as np

MASK64 = np.uint64(0xFFFFFFFFFFFFFFFF)
_GOLD = np.uint64(0x9E3779B97F4A7C15)
_M1 = np.uint64(0xBF58476D1CE4E5B9)
_M2 = np.uint64(0x94D049BB133111EB)

#: sd of the centred sum of four U{0..65535} variables.
SD_E = float(np.sqrt(4.0 * (65536.0 ** 2 - 1.0) / 12.0))
RHO_Q16 = 58982
INNOV_Q16 = 28567
#: missing when the top 32 bits of the stream-3 draw fall below this (1%).
MISS_THRESH = 42949673

CODE_OF_VALUE = np.array([0b00, 0b10, 0b11], dtype=np.uint8)
MISSING_CODE = 0b01


def mix64(x):
    """splitmix64 finaliser on uint64 numpy values (wrapping arithmetic)."""
    with np.errstate(over="ignore"):
        x = np.asarray(x, dtype=np.uint64) + _GOLD
        x = (x ^ (x >> np.uint64(30))) * _M1
        x = (x ^ (x >> np.uint64(27))) * _M2
        return x ^ (x >> np.uint64(31))


def stream_key(seed: int, stream: int) -> np.uint64:
    return mix64(np.uint64(seed & 0xFFFFFFFFFFFFFFFF) ^ mix64(np.uint64(stream)))


def draw(key, i, j):
    """Counter-based 64-bit draw for sample ``i`` and SNP ``j`` (both < 2**32)."""
    i = np.asarray(i, dtype=np.uint64)
    j = np.asarray(j, dtype=np.uint64)
    return mix64(np.uint64(key) ^ mix64((j << np.uint64(32)) | i))


def allele_freqs(seed: int, m: int, j0: int = 0) -> np.ndarray:
    r = draw(stream_key(seed, 1), 0, np.arange(j0, j0 + m, dtype=np.uint64))
    u = (r >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)
    return 0.05 + 0.45 * u


def hwe_thresholds(p: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    """Integer latent thresholds (t0, t1) for HWE cells (1-p)^2 and 1-p^2."""
    from scipy.special import ndtri

    t0 = np.rint(ndtri((1.0 - p) ** 2) * SD_E).astype(np.int64)
    t1 = np.rint(ndtri(1.0 - p * p) * SD_E).astype(np.int64)
    return t0, t1


def synth_genotypes(n: int, m: int, seed: int, missing: bool = True) -> np.ndarray:
    """Return an (m, n) int8 matrix of hard calls 0/1/2, -9 for missing."""
    p = allele_freqs(seed, m)
    t0, t1 = hwe_thresholds(p)
    k2 = stream_key(seed, 2)
    k3 = stream_key(seed, 3)
    i = np.arange(n, dtype=np.uint64)
    out = np.empty((m, n), dtype=np.int8)
    u = None
    for j in range(m):
        r = draw(k2, i, j)
        e = ((r & np.uint64(0xFFFF)).astype(np.int64)
             + ((r >> np.uint64(16)) & np.uint64(0xFFFF)).astype(np.int64)
             + ((r >> np.uint64(32)) & np.uint64(0xFFFF)).astype(np.int64)
             + (r >> np.uint64(48)).astype(np.int64) - 131070)
        u = e if u is None else (RHO_Q16 * u + INNOV_Q16 * e) >> 16
        g = np.where(u < t0[j], 0, np.where(u < t1[j], 1, 2)).astype(np.int8)
        if missing:
            miss = (draw(k3, i, j) >> np.uint64(32)) < np.uint64(MISS_THRESH)
            g[miss] = -9
        out[j] = g
    return out


def pack_bed_rows(geno: np.ndarray) -> np.ndarray:
    """Pack an (m, n) 0/1/2/-9 matrix into (m, ceil(n/4)) BED bytes.

    Padding bits of the last byte are written as ``00`` like PLINK does.
    """
    geno = np.asarray(geno)
    m, n = geno.shape
    codes = np.where(geno < 0, MISSING_CODE, CODE_OF_VALUE[np.clip(geno, 0, 2)]).astype(np.uint8)
    nb = (n + 3) // 4
    padded = np.zeros((m, nb * 4), dtype=np.uint8)
    padded[:, :n] = codes
    q = padded.reshape(m, nb, 4)
    return (q[:, :, 0] | (q[:, :, 1] << 2) | (q[:, :, 2] << 4) | (q[:, :, 3] << 6)).astype(np.uint8)


def unpack_bed_rows(rows: np.ndarray, n: int) -> np.ndarray:
    """Inverse of :func:`pack_bed_rows` (returns 0/1/2/-9 int8, shape (m, n))."""
    rows = np.asarray(rows, dtype=np.uint8)
    m = rows.shape[0]
    codes = np.stack([(rows >> (2 * t)) & 3 for t in range(4)], axis=-1).reshape(m, -1)[:, :n]
    lut = np.array([0, -9, 1, 2], dtype=np.int8)
    return lut[codes]


def write_plink(prefix: str | os.PathLike, geno: np.ndarray | None = None,
                packed: np.ndarray | None = None, n: int | None = None,
                bp: np.ndarray | None = None, chrom: np.ndarray | None = None) -> str:
    """Write ``prefix.bed/.bim/.fam`` and return the prefix as a string."""
    prefix = str(prefix)
    if packed is None:
        packed = pack_bed_rows(geno)
        n = geno.shape[1]
    m = packed.shape[0]
    with open(prefix + ".bed", "wb") as f:
        f.write(bytes([0x6C, 0x1B, 0x01]))
        f.write(np.ascontiguousarray(packed, dtype=np.uint8).tobytes())
    if bp is None:
        bp = np.arange(1, m + 1, dtype=np.int64) * 100
    if chrom is None:
        chrom = np.ones(m, dtype=np.int64)
    with open(prefix + ".bim", "w") as f:
        for j in range(m):
            f.write(f"{int(chrom[j])}\trs{j}\t0\t{int(bp[j])}\tA\tG\n")
    with open(prefix + ".fam", "w") as f:
        for i in range(int(n)):
            f.write(f"f{i} i{i} 0 0 0 -9\n")
    return prefix


def read_bed_packed(prefix: str | os.PathLike, n: int, m: int) -> np.ndarray:
    data = np.fromfile(str(prefix) + ".bed", dtype=np.uint8)
    if data.size < 3 or data[0] != 0x6C or data[1] != 0x1B or data[2] != 0x01:
        raise ValueError("Invalid BED magic/mode (expected 6C 1B 01)")
    nb = (n + 3) // 4
    return data[3:3 + nb * m].reshape(m, nb)


def count_lines(path: str | os.PathLike) -> int:
    n = 0
    with open(path) as f:
        for line in f:
            if line.startswith("#"):
                continue
            n += 1
    return n


def synth_plink(prefix: str | os.PathLike, n: int, m: int, seed: int,
                missing: bool = True) -> str:
    """Generate and write a synthetic BED fileset; returns the prefix."""
    Path(prefix).parent.mkdir(parents=True, exist_ok=True)
    return write_plink(prefix, synth_genotypes(n, m, seed, missing=missing))
