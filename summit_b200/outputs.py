"""The reference's genome-wide output files, written from this library's results.

SUMMIT's genome-wide driver writes (gw_ldscore.py:1186-1208, :2230-2338):

* ``<out>.gw.ldscore.gz`` - CHR, SNP, BP, optionally V, one column per
  annotation and optionally LD_REL_<annotation>; tab-separated, six decimals,
  gzip level 6;
* ``<out>.gw.M`` - the annotation masses on one tab-separated line, ``%.10g``;
* ``<out>.gw.mc.tsv`` - the annotation-level Monte-Carlo noise diagnostic
  (integrated MC variance of the probe mean, RMS MC SE, numerical status);
* ``<out>.gw.mcvar.gz`` - optional per-SNP MC variances, SEs and 95 % intervals.

``write_gw_outputs`` produces all of them from the dict that
``gwldcore.gw_ldscore`` / ``session.windowed_ldscore`` return (LD scores,
``meansq_accum`` and the fourth-moment sums), so a user of the one-call GPU
entries gets the files the reference's downstream readers consume.  The MC
arithmetic follows _mc_variance_from_probe_sums and
_integrated_mc_variance_from_probe_sums (gw_ldscore.py:874-996): per SNP and
annotation, Y_v = the probe-v term of the LD-score sum, first sum S1 =
meansq_accum = sum_v Y_v, second sum S2 = sum_v Y_v^2 (the fourth-moment sums),
and var = (S2 - S1^2 / B) / (B (B - 1)) with the reference's round-off rule.
"""
from __future__ import annotations

import gzip
from pathlib import Path

import numpy as np
import pandas as pd

Z95 = 1.959963984540054


def write_gw_ldscore_table(outpath, snpdf: pd.DataFrame, scores_df: pd.DataFrame, *,
                           snp_var=None, ld_rel=None) -> str:
    """``<outpath>.gw.ldscore.gz``: the SNP columns, V (when given), one column
    per annotation and LD_REL_<annotation> (when given)."""
    cols = [snpdf.reset_index(drop=True)]
    if snp_var is not None:
        cols.append(pd.DataFrame({"V": np.asarray(snp_var)}))
    cols.append(scores_df.reset_index(drop=True))
    if ld_rel is not None:
        cols.append(pd.DataFrame(np.asarray(ld_rel),
                                 columns=[f"LD_REL_{c}" for c in scores_df.columns]))
    table = pd.concat(cols, axis=1)
    path = f"{outpath}.gw.ldscore.gz"
    table.to_csv(path, sep="\t", index=False, float_format="%.6f",
                 compression={"method": "gzip", "compresslevel": 6})
    return path


def write_gw_annotation_masses(outpath, masses) -> str:
    """``<outpath>.gw.M``: one tab-separated line of masses, ``%.10g`` each."""
    path = f"{outpath}.gw.M"
    Path(path).write_text("\t".join(format(float(x), ".10g") for x in masses) + "\n")
    return path


def _clip_centered(centered, second, correction, eps):
    """The reference's round-off rule: a centered second moment that is
    negative within 512 eps of the larger term is clipped to 0, one further
    below (or non-finite) is a numerical failure (NaN)."""
    scale = np.maximum(np.maximum(np.abs(second), np.abs(correction)), 1.0)
    tol = 512.0 * eps * scale
    finite = np.isfinite(centered) & np.isfinite(tol)
    tiny = finite & (centered < 0.0) & (centered >= -tol)
    bad = ~finite | (centered < -tol)
    centered = centered.copy()
    centered[tiny] = 0.0
    centered[bad] = np.nan
    return centered, tiny, bad


def mc_variance(probe_sum, probe_sumsq, nvecs: int, eps: float | None = None):
    """Per-SNP MC variance of the probe mean: (S2 - S1^2/B) / (B (B-1)).
    Returns (variance M x K, round-off clip counts K, failure counts K)."""
    s1 = np.asarray(probe_sum, dtype=np.float64)
    s2 = np.asarray(probe_sumsq, dtype=np.float64)
    if s1.shape != s2.shape or s1.ndim != 2:
        raise ValueError("probe_sum and probe_sumsq must be two-dimensional with equal shapes")
    if nvecs < 2:
        return (np.full(s1.shape, np.nan), np.zeros(s1.shape[1], np.int64),
                np.full(s1.shape[1], s1.shape[0], np.int64))
    if eps is None:
        dt = np.asarray(probe_sum).dtype
        eps = np.finfo(dt if np.issubdtype(dt, np.floating) else np.float64).eps
    corr = s1 * s1 / float(nvecs)
    cen, tiny, bad = _clip_centered(s2 - corr, s2, corr, eps)
    return (cen / float(nvecs * (nvecs - 1)), tiny.sum(0).astype(np.int64),
            bad.sum(0).astype(np.int64))


def integrated_mc_variance(probe_sum, aggregate_sumsq, nvecs: int, eps: float | None = None):
    """Sum over SNPs of the per-SNP MC variances from the per-SNP first sums
    and the aggregate second sums (K): returns (variance K, clip flags K,
    failure flags K)."""
    s1 = np.asarray(probe_sum)
    s2 = np.asarray(aggregate_sumsq, dtype=np.float64)
    if s1.ndim != 2 or s2.shape != (s1.shape[1],):
        raise ValueError("aggregate MC sufficient-statistic shapes are inconsistent")
    if nvecs < 2:
        return (np.full(s2.shape, np.nan), np.zeros(s2.shape, np.int64),
                np.ones(s2.shape, np.int64))
    if eps is None:
        eps = np.finfo(s1.dtype if np.issubdtype(s1.dtype, np.floating) else np.float64).eps
    sq = np.einsum("ij,ij->j", s1.astype(np.float64), s1.astype(np.float64))
    corr = sq / float(nvecs)
    cen, tiny, bad = _clip_centered(s2 - corr, s2, corr, eps)
    return cen / float(nvecs * (nvecs - 1)), tiny.astype(np.int64), bad.astype(np.int64)


def mc_diagnostic_table(l2cols, masses, ldscore, meansq_accum, mc_aggregate_sumsq, nvecs: int,
                        seed: int, rand_dist: str, dtype, n_denom: float,
                        mc_per_snp_sumsq=None) -> tuple[pd.DataFrame, np.ndarray | None]:
    """The annotation-level MC noise diagnostic (gw_ldscore.py:2241-2283) and,
    when per-SNP second sums are given, the per-SNP MC variances."""
    ldscore = np.asarray(ldscore, dtype=np.float64)
    m = ldscore.shape[0]
    ivar, clip, fail = integrated_mc_variance(meansq_accum, mc_aggregate_sumsq, nvecs)
    rms_se = np.sqrt(np.maximum(ivar, 0.0) / float(m))
    ld_rms = np.sqrt(np.einsum("ij,ij->j", ldscore, ldscore) / float(m))
    rel = rms_se / np.maximum(ld_rms, np.finfo(np.float64).tiny)
    K = len(l2cols)
    var = None
    if mc_per_snp_sumsq is None:
        p_clip = np.zeros(K, np.int64)
        p_fail = np.zeros(K, np.int64)
        p_status = np.full(K, "not_requested", dtype=object)
    else:
        var, p_clip, p_fail = mc_variance(meansq_accum, mc_per_snp_sumsq, nvecs)
        p_status = np.full(K, "ok", dtype=object)
        p_status[p_clip > 0] = "roundoff_clipped"
        p_status[p_fail > 0] = "numerical_failure"
    status = np.full(K, "ok", dtype=object)
    status[(clip > 0) | (p_clip > 0)] = "roundoff_clipped"
    status[(fail > 0) | (p_fail > 0)] = "numerical_failure"
    table = pd.DataFrame({
        "annotation": list(l2cols),
        "annotation_mass": np.asarray(masses),
        "nvecs": int(nvecs),
        "nsnps": int(m),
        "seed": int(seed),
        "probe_distribution": str(rand_dist),
        "dtype": np.dtype(dtype).name,
        "residual_correlation_denom": float(n_denom),
        "integrated_mc_variance": ivar,
        "rms_mc_se": rms_se,
        "ldscore_rms": ld_rms,
        "relative_rms_mc_se": rel,
        "numerical_status": status,
        "roundoff_clipped_terms": clip,
        "numerical_failure_terms": fail,
        "per_snp_numerical_status": p_status,
        "per_snp_roundoff_clipped_terms": p_clip,
        "per_snp_numerical_failure_terms": p_fail,
    })
    return table, var


def write_mc_variance(outpath, snpdf: pd.DataFrame, l2cols, ldscore, var,
                      chunk_rows: int = 65536) -> str:
    """``<outpath>.gw.mcvar.gz``: per SNP and annotation the MC variance, SE and
    pointwise 95 % interval, ``%.10e``."""
    path = f"{outpath}.gw.mcvar.gz"
    ldscore = np.asarray(ldscore, dtype=np.float64)
    snpdf = snpdf.reset_index(drop=True)
    with gzip.open(path, "wt", encoding="utf-8") as fh:
        for a in range(0, ldscore.shape[0], chunk_rows):
            b = min(ldscore.shape[0], a + chunk_rows)
            v = np.asarray(var[a:b], dtype=np.float64)
            se = np.sqrt(v)
            cols = {}
            for k, name in enumerate(l2cols):
                cols[f"{name}_MC_VAR"] = v[:, k]
                cols[f"{name}_MC_SE"] = se[:, k]
                cols[f"{name}_MC_CI95_LO"] = ldscore[a:b, k] - Z95 * se[:, k]
                cols[f"{name}_MC_CI95_HI"] = ldscore[a:b, k] + Z95 * se[:, k]
            part = pd.concat([snpdf.iloc[a:b].reset_index(drop=True), pd.DataFrame(cols)], axis=1)
            part.to_csv(fh, sep="\t", index=False, header=(a == 0), float_format="%.10e")
    return path


def write_gw_outputs(outpath, result: dict, *, snpdf: pd.DataFrame | None = None, l2cols=None,
                     masses=None, nvecs: int | None = None, seed: int = 0,
                     rand_dist: str = "rademacher", dtype=np.float64, n_denom: float | None = None,
                     snp_var=None, write_mc_var: bool = False) -> dict:
    """Write the reference's genome-wide files from a result dict
    (``ldscore`` M x K; for the MC files also ``meansq_accum``,
    ``mc_aggregate_sumsq`` and, for ``.gw.mcvar.gz``, ``mc_per_snp_sumsq``).

    ``snpdf`` holds CHR, SNP, BP (NaN columns when omitted, as the reference
    writes without a SNP list); ``l2cols`` defaults to L2_0..L2_{K-1};
    ``masses`` to the per-bin SNP counts of the result (required for the .M
    file otherwise).  Returns the paths written."""
    ld = np.asarray(result["ldscore"], dtype=np.float64)
    m, K = ld.shape
    l2cols = list(l2cols) if l2cols is not None else [f"L2_{k}" for k in range(K)]
    if snpdf is None:
        snpdf = pd.DataFrame(np.nan * np.ones((m, 3)), columns=["CHR", "SNP", "BP"])
    else:
        snpdf = snpdf[["CHR", "SNP", "BP"]].copy()
        snpdf.columns = ["CHR", "SNP", "BP"]
    paths = {"ldscore": write_gw_ldscore_table(outpath, snpdf, pd.DataFrame(ld, columns=l2cols),
                                               snp_var=snp_var)}
    if result.get("mc_aggregate_sumsq") is not None:
        if nvecs is None or n_denom is None or masses is None:
            raise ValueError("the MC diagnostic needs nvecs, n_denom and masses")
        table, var = mc_diagnostic_table(
            l2cols, masses, ld, result["meansq_accum"], result["mc_aggregate_sumsq"], nvecs, seed,
            rand_dist, dtype, n_denom,
            result.get("mc_per_snp_sumsq") if write_mc_var else None)
        path = f"{outpath}.gw.mc.tsv"
        table.to_csv(path, sep="\t", index=False, float_format="%.10e")
        paths["mc"] = path
        if write_mc_var and var is not None:
            paths["mcvar"] = write_mc_variance(outpath, snpdf, l2cols, ld, var)
    if masses is not None:
        paths["M"] = write_gw_annotation_masses(outpath, masses)
    return paths
