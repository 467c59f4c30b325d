"""CPU: the C-ABI library loads, exports every function include/lds.h
declares, and the Python shim validates arguments like the nanobind module
(no compute calls: no GPU here)."""
from __future__ import annotations

import ctypes
import re
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]


def _declared() -> set[str]:
    text = (ROOT / "include" / "lds.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return set(re.findall(r"\b(lds_[a-z0-9_]+)\s*\(", text))


def test_library_exports_every_declared_symbol():
    from summit_b200 import _lib

    lib = ctypes.CDLL(str(_lib.LIB_PATH))
    declared = _declared()
    assert len(declared) >= 25
    missing = [s for s in sorted(declared) if not hasattr(lib, s)]
    assert not missing, f"declared but not exported: {missing}"
    # the Python binding table covers every declared entry
    assert declared <= set(_lib.SIGNATURES), sorted(declared - set(_lib.SIGNATURES))


def test_library_reports_version_and_no_device_without_gpu():
    from summit_b200 import _lib

    lib = _lib.load()
    assert b"sm_100a" in lib.lds_version()
    assert lib.lds_device_count() >= 0


def test_shim_argument_validation_matches_nanobind_rules():
    from summit_b200 import gwldcore

    xz = np.zeros((4, 2), dtype=np.float64)  # C order: not F-contiguous -> rejected
    with pytest.raises(TypeError):
        gwldcore.phase1_compute_Xz_bed_chunk("x", "x.fam", 0, 1, annot_blk=np.ones((1, 2)),
                                             inv_right=np.ones(1), v_start=0, v_count=1,
                                             kmax_hint=1, Xz2d_chunk=xz)
    with pytest.raises(TypeError):
        gwldcore.phase2_accum_XtXz_bed("x", "x.fam", 0, 1, inv_left=np.ones(1), tile_nvecs=1,
                                       Xz2d=np.zeros((4, 1)), meansq_accum=np.zeros((1, 1), np.int32))
    with pytest.raises(TypeError):
        gwldcore.phase2_accum_XtXz_bed("x", "x.fam", 0, 1, inv_left=np.ones(1), tile_nvecs=1)
    with pytest.raises(RuntimeError, match="impute_mode"):
        gwldcore._impute("median")
    assert gwldcore._dist("rademacher") == 0 and gwldcore._dist("normal") == 1
    assert gwldcore._dist("spherical") == 2


def test_wait_limit_argument_check_without_gpu():
    from summit_b200 import _lib

    lib = _lib.load()
    assert lib.lds_set_wait_limit(0) == -1
    assert "wait limit" in lib.lds_last_error().decode()
    assert lib.lds_get_wait_limit() == 1 << 25


def test_checked_build_reports_itself_and_exports_every_symbol():
    """The bounds-checked build (liblds_checked.so) and the ordinary one say
    which they are; the checked one exports the same entries."""
    from summit_b200 import _lib

    plain = ctypes.CDLL(str(_lib.PKG / "liblds.so"))
    plain.lds_checked_build.restype = ctypes.c_int
    assert plain.lds_checked_build() == 0
    path = _lib.PKG / "liblds_checked.so"
    if not path.exists():
        pytest.skip("bounds-checked build not built (python -m summit_b200.build --checked)")
    checked = ctypes.CDLL(str(path))
    checked.lds_checked_build.restype = ctypes.c_int
    assert checked.lds_checked_build() == 1
    missing = [s for s in sorted(_declared()) if not hasattr(checked, s)]
    assert not missing, f"declared but not exported by the checked build: {missing}"
