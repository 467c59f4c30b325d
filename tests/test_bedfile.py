"""CPU: BED writer and the integer-exact synthetic generator."""
from __future__ import annotations

import numpy as np

from summit_b200 import bedfile


def test_pack_unpack_roundtrip_and_file(tmp_path):
    g = bedfile.synth_genotypes(37, 11, seed=2)
    packed = bedfile.pack_bed_rows(g)
    assert packed.shape == (11, 10)
    np.testing.assert_array_equal(bedfile.unpack_bed_rows(packed, 37), g)
    prefix = bedfile.write_plink(tmp_path / "rt", g)
    np.testing.assert_array_equal(bedfile.read_bed_packed(prefix, 37, 11), packed)
    assert bedfile.count_lines(prefix + ".fam") == 37
    assert bedfile.count_lines(prefix + ".bim") == 11
    raw = open(prefix + ".bed", "rb").read(3)
    assert raw == bytes([0x6C, 0x1B, 0x01])


def test_bed_codes_follow_plink_mapping():
    g = np.array([[0, 1, 2, -9]], dtype=np.int8)
    assert bedfile.pack_bed_rows(g)[0, 0] == (0b00 | 0b10 << 2 | 0b11 << 4 | 0b01 << 6)


def test_generator_statistics():
    g = bedfile.synth_genotypes(2000, 300, seed=11)
    miss = (g < 0).mean()
    assert 0.008 < miss < 0.012
    p = bedfile.allele_freqs(11, 300)
    assert p.min() >= 0.05 and p.max() <= 0.5
    gm = np.where(g < 0, np.nan, g)
    assert np.corrcoef(np.nanmean(gm, 1) / 2, p)[0, 1] > 0.99
    x = np.nan_to_num(gm - np.nanmean(gm, 1, keepdims=True))
    c = np.corrcoef(x)
    adj = np.mean([c[j, j + 1] for j in range(299)])
    far = np.mean([abs(c[j, j + 50]) for j in range(249)])
    assert adj > 0.5 and far < 0.05


def test_c_generator_matches_numpy(oracle):
    a = oracle.synth_bed_rows(1001, 40, seed=99)
    b = bedfile.pack_bed_rows(bedfile.synth_genotypes(1001, 40, seed=99))
    np.testing.assert_array_equal(a, b)
