"""Golden output files written by the reference's own Python code.

The reference's genome-wide driver module cannot be imported here (it needs
bed_reader and its native modules), so this script takes the writer and MC
functions (write_gw_ldscore_table, write_gw_annotation_masses,
_mc_variance_from_probe_sums, _integrated_mc_variance_from_probe_sums,
_column_rms_chunked) and the driver's MC-diagnostic block (the statements
between ``write_gw_ldscore_table(...)`` and ``masses = self.nsnps_bin`` in
GenomewideLDScore._compute_ldscore) verbatim from src/summit/ldscore/
gw_ldscore.py of the tree named by SUMMIT_REFERENCE_DIR and runs them on fixed
synthetic inputs.  The inputs and the files they produce are saved under
tests/golden/gw_outputs/.

    SUMMIT_REFERENCE_DIR=<SUMMIT checkout> python tests/golden/make_golden_outputs.py
"""
from __future__ import annotations

import ast
import gzip
import os
import shutil
import tempfile
import textwrap
import types
from pathlib import Path

import numpy as np
import pandas as pd

HERE = Path(__file__).resolve().parent
OUT = HERE / "gw_outputs"

FUNCS = ("write_gw_ldscore_table", "write_gw_annotation_masses", "_mc_variance_from_probe_sums",
         "_integrated_mc_variance_from_probe_sums", "_column_rms_chunked")


def inputs():
    rng = np.random.default_rng(20261204)
    m, K, B = 37, 3, 12
    # per-probe terms Y_v >= 0 give consistent first / second sums
    Y = rng.gamma(2.0, 0.7, size=(m, K, B))
    Y[5] = 0.0  # a monomorphic SNP: every term zero
    meansq = Y.sum(2)
    mc_snp = (Y * Y).sum(2)
    mc_agg = mc_snp.sum(0)
    masses = np.array([37.0, 11.0, 20.5])
    n_denom = 499.0
    ld = meansq / B - masses[None, :] / n_denom
    snpdf = pd.DataFrame({"CHR": np.ones(m, dtype=np.int64),
                          "SNP": [f"rs{j}" for j in range(m)],
                          "BP": 100 * np.arange(1, m + 1)})
    return dict(meansq=meansq, mc_snp=mc_snp, mc_agg=mc_agg, masses=masses, n_denom=n_denom,
                ld=ld, B=B, snpdf=snpdf, l2cols=["L2_0", "base", "L2_2"], seed=991)


def reference_namespace(src: str) -> dict:
    tree = ast.parse(src)
    ns = {"np": np, "pd": pd, "gzip": gzip}
    for node in tree.body:
        if isinstance(node, ast.FunctionDef) and node.name in FUNCS:
            exec(compile(ast.Module([node], []), "gw_ldscore.py", "exec"), ns)
    missing = [f for f in FUNCS if f not in ns]
    if missing:
        raise SystemExit(f"reference functions not found: {missing}")
    return ns


def mc_block(src: str) -> str:
    start = src.index("        write_gw_ldscore_table(self.outpath, self.snpdf, scores_df")
    start = src.index("\n", start) + 1
    stop = src.index("        masses = self.nsnps_bin if self.annot_mass is None", start)
    return textwrap.dedent(src[start:stop])


def main() -> None:
    ref = os.environ.get("SUMMIT_REFERENCE_DIR")
    if not ref:
        raise SystemExit("set SUMMIT_REFERENCE_DIR to the SUMMIT source tree")
    src = (Path(ref) / "src" / "summit" / "ldscore" / "gw_ldscore.py").read_text()
    ns = reference_namespace(src)
    d = inputs()
    if OUT.exists():
        shutil.rmtree(OUT)
    OUT.mkdir()
    np.savez(OUT / "inputs.npz", meansq=d["meansq"], mc_snp=d["mc_snp"], mc_agg=d["mc_agg"],
             masses=d["masses"], n_denom=d["n_denom"], ld=d["ld"], B=d["B"], seed=d["seed"])
    with tempfile.TemporaryDirectory() as td:
        out = str(Path(td) / "ref")
        scores = pd.DataFrame(d["ld"], columns=d["l2cols"])
        ns["write_gw_ldscore_table"](out, d["snpdf"], scores)
        ns["write_gw_annotation_masses"](out, d["masses"])
        # the driver's MC block, run on a stand-in for the estimator object
        integrated, agg_info = ns["_integrated_mc_variance_from_probe_sums"](
            d["meansq"], d["mc_agg"], d["B"], return_info=True)
        var, snp_info = ns["_mc_variance_from_probe_sums"](
            d["meansq"], d["mc_snp"].copy(), d["B"], return_info=True)
        self = types.SimpleNamespace(
            outpath=out, gwldscore=d["ld"], nsnps=d["ld"].shape[0], snpdf=d["snpdf"],
            nbins=d["ld"].shape[1],
            l2cols=d["l2cols"], nsnps_bin=d["masses"], nvecs=d["B"], root_seed=d["seed"],
            rand_dist="rademacher", dtype=np.float64, estimate_mc_noise=True,
            write_ld_mc_var=True, ld_mc_variance=var,
            _ld_mc_integrated_variance=integrated,
            _ld_mc_numerical_info={"aggregate": agg_info, "per_snp": snp_info},
            log=types.SimpleNamespace(_log=lambda *a, **k: None))
        env = dict(ns, self=self, N_denom=d["n_denom"])
        exec(compile(mc_block(src), "gw_ldscore.py", "exec"), env)
        for suffix in (".gw.ldscore.gz", ".gw.M", ".gw.mc.tsv", ".gw.mcvar.gz"):
            shutil.copy(out + suffix, OUT / ("ref" + suffix))
    print("wrote", sorted(p.name for p in OUT.iterdir()))


if __name__ == "__main__":
    main()
