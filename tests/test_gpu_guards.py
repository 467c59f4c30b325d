"""GPU: the phase-2 guards against the reference's own compiled gwldcore.cpp.

The reference drops non-finite LD-score updates, and finite updates above
SUMMIT_P2_EXTREME_LD_WARN times the bin's probe count unless
SUMMIT_P2_DROP_EXTREME=0, and prints both counts per call
(gwldcore.cpp:295-417, "[phase2-watch] ... nonfinite_dropped=N extreme=M").
Both libraries read the environment once per process, so each setting runs
in a fresh child process that calls the reference and liblds on the same
genotypes, sketch and scales, and reports the sums and the counts (ours
through lds_phase2_guard_counts).
"""
from __future__ import annotations

import json
import os
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

from conftest import assert_rel_elementwise

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parents[1]

CHILD = r"""
import ctypes, json, os, re, sys, tempfile
import numpy as np
sys.path.insert(0, sys.argv[1])
from oracle.oracle import Reference
from summit_b200 import _lib, bedfile, gwldcore

nan = sys.argv[2] == "1"
n, m, K, V = 200, 90, 2, 6
geno = bedfile.synth_genotypes(n, m, seed=8)
geno[5] = 1          # monomorphic: its update is exactly 0, never extreme
td = tempfile.mkdtemp()
prefix = bedfile.write_plink(td + "/g", geno)
rng = np.random.default_rng(3)
Xz = np.asfortranarray(rng.standard_normal((n, K * V)))
if nan:
    Xz[7, V + 2] = np.nan   # bin 1 becomes non-finite for every SNP
inv = np.ones(m)

ref = Reference()
ms_ref = np.zeros((m, K))
log = tempfile.TemporaryFile()
saved = os.dup(2)
os.dup2(log.fileno(), 2)
try:
    ref.phase2_bed(prefix, 0, m, inv, V, Xz, ms_ref, n)
finally:
    os.dup2(saved, 2)
log.seek(0)
text = log.read().decode()
hit = re.search(r"nonfinite_dropped=(\d+) extreme=(\d+)", text)
ms = np.zeros((m, K))
gwldcore.phase2_accum_XtXz_bed(bed_prefix=prefix, fam_path=prefix + ".fam", blk_start=0,
                               blk_end=m, ddof=1, inv_left=inv, tile_nvecs=V, Xz2d=Xz,
                               meansq_accum=ms, N_denom=n, impute_mode="mean")
counts = (ctypes.c_uint64 * 2)()
assert _lib.load().lds_phase2_guard_counts(counts) == 0
print(json.dumps({"ref_counts": [int(hit.group(1)), int(hit.group(2))] if hit else None,
                  "ours_counts": [int(counts[0]), int(counts[1])],
                  "ref": ms_ref.tolist(), "ours": ms.tolist()}))
"""


def _run(env_extra: dict, nan: bool) -> dict:
    env = dict(os.environ)
    for k in ("SUMMIT_P2_EXTREME_LD_WARN", "SUMMIT_P2_ABS_LD_MAX", "SUMMIT_P2_DROP_EXTREME"):
        env.pop(k, None)
    env.update(env_extra)
    out = subprocess.run([sys.executable, "-c", CHILD, str(ROOT), "1" if nan else "0"], env=env,
                         capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-3000:]
    return json.loads(out.stdout.strip().splitlines()[-1])


@pytest.fixture(scope="module")
def _have_reference():
    from oracle.oracle import REF_SO

    if not REF_SO.exists():
        pytest.skip("reference checker oracle/_ref/libref_gwld.so not built")


@pytest.mark.parametrize(
    "name,env,nan,expect",
    [
        ("nonfinite", {}, True, [90, 0]),
        ("extreme_dropped", {"SUMMIT_P2_EXTREME_LD_WARN": "1e-30"}, False, [0, 2 * 89]),
        ("extreme_kept", {"SUMMIT_P2_EXTREME_LD_WARN": "1e-30", "SUMMIT_P2_DROP_EXTREME": "0"},
         False, [0, 2 * 89]),
        ("defaults", {}, False, [0, 0]),
    ],
)
def test_guard_counts_and_sums_match_reference(_have_reference, name, env, nan, expect):
    r = _run(env, nan)
    assert r["ref_counts"] is not None, "the reference printed no guard line"
    # expected counts: one per (SNP, bin) update judged; the monomorphic SNP's
    # update is exactly 0 and never extreme, but its products with a NaN
    # column are NaN in both libraries
    assert r["ref_counts"] == expect, r["ref_counts"]
    assert r["ours_counts"] == r["ref_counts"], (name, r["ours_counts"], r["ref_counts"])
    ref, ours = np.asarray(r["ref"]), np.asarray(r["ours"])
    assert_rel_elementwise(ours, ref, 1e-6, name)
