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
