"""CPU: the genome-wide output files (.gw.ldscore.gz, .gw.M, .gw.mc.tsv,
.gw.mcvar.gz) written by summit_b200.outputs are identical, text for text, to
the files the reference's own writer and MC-diagnostic code produce from the
same inputs (tests/golden/make_golden_outputs.py)."""
from __future__ import annotations

import gzip
from pathlib import Path

import numpy as np
import pandas as pd

GOLD = Path(__file__).resolve().parent / "golden" / "gw_outputs"


def _text(path: Path) -> str:
    if path.suffix == ".gz":
        with gzip.open(path, "rt") as f:
            return f.read()
    return path.read_text()


def test_outputs_match_reference_files(tmp_path):
    from summit_b200.outputs import write_gw_outputs

    d = np.load(GOLD / "inputs.npz")
    m = d["ld"].shape[0]
    snpdf = pd.DataFrame({"CHR": np.ones(m, dtype=np.int64), "SNP": [f"rs{j}" for j in range(m)],
                          "BP": 100 * np.arange(1, m + 1)})
    result = {"ldscore": d["ld"], "meansq_accum": d["meansq"], "mc_aggregate_sumsq": d["mc_agg"],
              "mc_per_snp_sumsq": d["mc_snp"]}
    out = str(tmp_path / "ours")
    paths = write_gw_outputs(out, result, snpdf=snpdf, l2cols=["L2_0", "base", "L2_2"],
                             masses=d["masses"], nvecs=int(d["B"]), seed=int(d["seed"]),
                             n_denom=float(d["n_denom"]), write_mc_var=True)
    assert set(paths) == {"ldscore", "M", "mc", "mcvar"}
    for suffix in (".gw.ldscore.gz", ".gw.M", ".gw.mc.tsv", ".gw.mcvar.gz"):
        assert _text(Path(out + suffix)) == _text(GOLD / ("ref" + suffix)), suffix


def test_outputs_without_snp_list_or_mc(tmp_path):
    from summit_b200.outputs import write_gw_outputs

    ld = np.arange(12, dtype=np.float64).reshape(4, 3) / 7.0
    paths = write_gw_outputs(str(tmp_path / "x"), {"ldscore": ld}, masses=[4, 2, 1])
    assert set(paths) == {"ldscore", "M"}
    t = pd.read_csv(paths["ldscore"], sep="\t")
    assert list(t.columns) == ["CHR", "SNP", "BP", "L2_0", "L2_1", "L2_2"]
    assert t[["CHR", "SNP", "BP"]].isna().all().all()
    np.testing.assert_allclose(t[["L2_0", "L2_1", "L2_2"]].to_numpy(), ld, atol=5e-7)
    assert Path(paths["M"]).read_text() == "4\t2\t1\n"
