"""GPU: bounded waits.  Every mbarrier wait of the tensor-core kernels gives
up after a run-time limit and records an error status instead of hanging
the GPU.  The self-test kernel waits on a barrier that nothing arrives at
(no copy or MMA in flight), so the only way out is the limit; the context
must stay usable afterwards."""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu


def test_short_wait_limit_runs_out_and_the_kernel_reports_it(small_bed, oracle):
    from summit_b200 import _lib, gwldcore

    lib = _lib.load()
    default = lib.lds_get_wait_limit()
    assert default == 1 << 25
    assert lib.lds_set_wait_limit(2000) == 0, lib.lds_last_error().decode()
    try:
        assert lib.lds_get_wait_limit() == 2000
        st = ctypes.c_uint(0)
        assert lib.lds_selftest_wait_timeout(ctypes.byref(st)) == 0, lib.lds_last_error().decode()
        assert st.value == 1, f"the bounded wait did not run out (status {st.value})"
    finally:
        assert lib.lds_set_wait_limit(default) == 0
    # the device context is intact: an estimate still runs and is right
    n, m, rows = small_bed["n"], small_bed["m"], small_bed["rows"]
    annot = np.ones((m, 1))
    out = gwldcore.gw_ldscore(rows, n, annot, 16, 64, 5)
    ora = oracle.gw_ldscore(rows, n, annot, 16, 64, 5)
    assert rel_err(out["ldscore"], ora["ldscore"]) < 1e-6


def test_invalid_wait_limit_is_rejected():
    from summit_b200 import _lib

    lib = _lib.load()
    assert lib.lds_set_wait_limit(0) == -1
    assert "wait limit" in lib.lds_last_error().decode()
