"""Generate the golden fixtures of tests/golden/ by running the reference's own
native code (gwldcore.cpp + genotype.cpp compiled unchanged into
oracle/_ref/libref_gwld.so by oracle/Makefile).

    make -C oracle ref && python tests/golden/make_golden.py

Fixtures:
* hardcalls_gw.npz — the 7 x 12 hard-call matrix of the reference's
  tests/test_pgen_gwld.py:139-151 (incl. missing, monomorphic and all-missing
  SNPs), genome-wide LD scores for mean and HWE imputation, Rademacher probes,
  float64 path, plus the residual variances.
* synth_gw.npz — a 97 x 131 synthetic fileset (bedfile.py generator, seed 5),
  two annotation bins, Gaussian and spherical probes, with MC fourth moments.
* hardcalls_winld.npz — exact windowed LD scores of the same hard calls from
  the reference's winldcore.cpp (oracle/_ref/libref_winld.so): mean and HWE
  imputation, 0.15 kb and 1 Mb windows over positions 100 bp apart, two
  annotation columns.
"""
from __future__ import annotations

import sys
import tempfile
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle.oracle import Reference, ReferenceWindowed  # noqa: E402
from summit_b200 import bedfile  # noqa: E402

HERE = Path(__file__).resolve().parent


def hardcalls() -> np.ndarray:
    """Variant x sample hard calls (A1 counts), -9 = missing (test_pgen_gwld.py:139-151)."""
    return np.asarray(
        [
            [0, 1, 2, 0, 1, 2, 0, 1, 2, 0, 1, 2],
            [2, 1, 0, 2, 1, 0, 2, 1, 0, 2, 1, 0],
            [0, -9, 1, 2, -9, 0, 1, 2, 0, 1, -9, 2],
            [0] * 12,
            [2] * 12,
            [-9] * 12,
            [0, 0, 0, 1, 1, 1, 2, 2, 2, -9, 0, 2],
        ],
        dtype=np.int8,
    )


def main() -> None:
    ref = Reference()
    ref.set_threads(1)
    out = {}
    with tempfile.TemporaryDirectory() as td:
        g = hardcalls()
        prefix = bedfile.write_plink(Path(td) / "hc", g)
        m, n = g.shape
        annot = np.ones((m, 1))
        for impute in ("mean", "hwe"):
            r = ref.gw_ldscore(prefix, n, m, annot, nvecs=64, step=3, seed=991,
                               dist="rademacher", impute=impute, impute_seed=17,
                               with_mc=True)
            out[f"{impute}_ldscore"] = r["ldscore"]
            out[f"{impute}_meansq"] = r["meansq_accum"]
            out[f"{impute}_inv"] = r["inv"]
            out[f"{impute}_mc"] = r["mc_per_snp_sumsq"]
        out["packed"] = bedfile.pack_bed_rows(g)
        np.savez(HERE / "hardcalls_gw.npz", **out)

        out = {}
        n, m = 97, 131
        g = bedfile.synth_genotypes(n, m, seed=5)
        prefix = bedfile.write_plink(Path(td) / "sy", g)
        annot = np.ones((m, 2))
        annot[::3, 1] = 0.0
        for dist in ("gaussian", "spherical"):
            r = ref.gw_ldscore(prefix, n, m, annot, nvecs=24, step=40, seed=31, dist=dist,
                               vtile=16, impute="mean", with_mc=True)
            out[f"{dist}_ldscore"] = r["ldscore"]
            out[f"{dist}_meansq"] = r["meansq_accum"]
            out[f"{dist}_mc"] = r["mc_per_snp_sumsq"]
            out[f"{dist}_mc_agg"] = r["mc_aggregate_sumsq"]
        out["packed"] = bedfile.pack_bed_rows(g)
        out["annot"] = annot
        np.savez(HERE / "synth_gw.npz", **out)

        refw = ReferenceWindowed()
        refw.set_threads(1)
        out = {}
        g = hardcalls()
        prefix = bedfile.write_plink(Path(td) / "hcw", g)
        m, n = g.shape
        bp = np.arange(1, m + 1, dtype=np.int64) * 100
        annot = np.column_stack([np.ones(m), np.arange(m) % 2 == 0]).astype(np.float64)
        for impute in ("mean", "hwe"):
            for kb in (0.15, 1000.0):
                key = f"{impute}_{'narrow' if kb < 1 else 'wide'}"
                out[key] = refw.compute_windowed_ld_chr(prefix, 0, m, bp, annot, kb, 4,
                                                        impute_mode=impute, impute_seed=17)
        out["packed"] = bedfile.pack_bed_rows(g)
        out["bp"] = bp
        out["annot"] = annot
        np.savez(HERE / "hardcalls_winld.npz", **out)
    print("wrote", sorted(p.name for p in HERE.glob("*.npz")))


if __name__ == "__main__":
    main()
