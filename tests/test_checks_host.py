"""Host comparison of phase-2 product checksums (lds_check_vectors): pure host
code, so it runs without a GPU.  Mismatches are planted in the host arrays."""
import numpy as np

from summit_b200 import _lib
from summit_b200._lib import check, ptr


def _verify(lhs, rhs):
    bad, first = np.zeros(1, np.int64), np.zeros(1, np.int64)
    check(_lib.load().lds_check_vectors(ptr(lhs), ptr(rhs), lhs.shape[0], ptr(bad), ptr(first)))
    return int(bad[0]), int(first[0])


def test_check_vectors_counts_differing_snps():
    rng = np.random.default_rng(1)
    lhs = rng.integers(0, 2**63, size=(1000, 2), dtype=np.uint64)
    rhs = lhs.copy()
    assert _verify(lhs, rhs) == (0, -1)
    rhs[17, 0] += np.uint64(1)
    assert _verify(lhs, rhs) == (1, 17)
    rhs[17, 1] ^= np.uint64(1 << 63)  # same SNP: still one
    rhs[900, 1] ^= np.uint64(4)
    assert _verify(lhs, rhs) == (2, 17)
    assert _verify(lhs[:0], rhs[:0]) == (0, -1)
