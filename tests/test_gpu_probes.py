"""GPU: Rademacher probe streams generated on the device are the host's
std::mt19937_64 streams bit for bit (make_seed, gwldcore.cpp:452-458, draws in
column order, gwldcore.cpp:1702-1706), checked against the oracle's host
generator for blocks shorter and longer than one 312-word twist."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("root,blk,v0,L,V", [
    (11, 0, 0, 1, 1), (11, 97, 16, 97, 40), (2**63 + 5, 1000, 0, 1000, 50),
    (0, 312, 64, 313, 7), (123456789, 0, 3, 5, 400)])
def test_device_rademacher_matches_host(oracle, root, blk, v0, L, V):
    from summit_b200 import _lib

    got = np.empty((V, L))  # column-major L x V
    _lib.check(_lib.load().lds_debug_rademacher_block(root, blk, v0, L, V, _lib.ptr(got)))
    want = oracle.probes(root, blk, v0, L, V, "rademacher")
    np.testing.assert_array_equal(got.T, want)
