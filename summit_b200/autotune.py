"""Autotuner of the windowed plans' tiling, with a persistent JSON cache.

The reference tunes its CPU kernels through environment knobs
(``SUMMIT_P1_NTILE``, ``SUMMIT_P2_QPANEL``, ``SUMMIT_WIN_PANEL_MB`` and the
like, read in gwldcore.cpp and winldcore.cpp).  Here the knobs that shape the
device work of a windowed estimate are chosen by timing them on the device:

* ``p1_sb_per_cta``: how the phase-1 work list of (window, bin) super-bins is
  split across CTAs (super-bins per CTA: longer per-CTA pipelines against
  more CTAs to balance);
* ``batch_gb``: how the windows are split into launches (the sketch digits of
  one batch stay under this many GB);
* ``p2_bin_chunk``: the phase-2 CTA order (window by window, chunks of about
  this many bins in whole CTA bin groups, the window's tiles, the chunk's
  groups; 0 is the grid's order), which sets how many CTAs share a tile's
  packed codes and a (window, bin) sketch in L2;
* ``p2_bins``: bins per phase-2 CTA (0: the fewest 256-column MMA groups per
  SNP tile; 1: one bin per CTA).

The LD scores do not depend on any of them, and the tuner checks that: every
candidate's scores must equal the first candidate's bit for bit.  A
candidate's cost is the device time of one estimate, as the sum of the plan's
CUDA-event intervals inside its graph, and the minimum over repeats is kept.
The winner is stored under a key of the device name, the library build and the
workload's shape (samples, SNPs, bins, probes, window-size quantiles on a log2
grid).
"""
from __future__ import annotations

import json
import math
import os
import time
from pathlib import Path
from typing import Callable, Iterable

import numpy as np

DEFAULT_CONFIG = {"p1_sb_per_cta": 8, "batch_gb": 8.0, "p2_bin_chunk": 4, "p2_bins": 0}


def default_candidates() -> list[dict]:
    """Phase-1 split x window batching, then the phase-2 order and CTA shape."""
    return ([{"p1_sb_per_cta": s, "batch_gb": b, "p2_bin_chunk": 4, "p2_bins": 0}
             for s in (8, 16, 32, 64, 128) for b in (4.0, 8.0, 16.0)] +
            [{"p1_sb_per_cta": 64, "batch_gb": 8.0, "p2_bin_chunk": c, "p2_bins": 0}
             for c in (0, 12, 24)] +
            [{"p1_sb_per_cta": 64, "batch_gb": 8.0, "p2_bin_chunk": 2, "p2_bins": 1}])


def _apply(plan, cand: dict) -> None:
    plan.set_tiling(int(cand["p1_sb_per_cta"]))
    plan.set_p2_order(int(cand.get("p2_bin_chunk", DEFAULT_CONFIG["p2_bin_chunk"])))
    plan.set_p2_bins(int(cand.get("p2_bins", DEFAULT_CONFIG["p2_bins"])))


def cache_path() -> Path:
    env = os.environ.get("SUMMIT_B200_TUNE_CACHE")
    if env:
        return Path(env)
    return Path(os.path.expanduser("~")) / ".cache" / "summit_b200" / "autotune.json"


def _log2_bucket(x: float) -> int:
    return int(round(math.log2(max(float(x), 1.0)) * 2))  # half-octave grid


def workload_key(device: str, n: int, m: int, k: int, nvecs: int, window_starts) -> str:
    """Key of a windowed workload: device, N, M (half-octaves), K, B, and the
    10/50/90 % window sizes (half-octaves)."""
    sizes = np.diff(np.asarray(window_starts, dtype=np.int64))
    q = [_log2_bucket(v) for v in np.percentile(sizes, [10, 50, 90])] if sizes.size else [0, 0, 0]
    return (f"{device}|N{int(n)}|M{_log2_bucket(m)}|K{int(k)}|B{int(nvecs)}|"
            f"w{q[0]}-{q[1]}-{q[2]}")


def library_id() -> str:
    """Identity of the loaded build (size and mtime of liblds.so): a rebuilt
    library is tuned afresh."""
    try:
        from . import _lib

        st = os.stat(_lib.LIB_PATH)
        return f"{st.st_size:x}{int(st.st_mtime):x}"
    except OSError:
        return "nolib"


def device_name() -> str:
    try:
        import torch

        if torch.cuda.is_available():
            return torch.cuda.get_device_name()
    except Exception:  # pragma: no cover - torch is plumbing only
        pass
    return "unknown"


class TuneCache:
    """JSON file of tuned records, keyed by workload_key."""

    def __init__(self, path: str | Path | None = None):
        self.path = Path(path) if path is not None else cache_path()
        self.records: dict = {}
        if self.path.exists():
            try:
                self.records = json.loads(self.path.read_text())
            except (OSError, ValueError):
                self.records = {}

    def get(self, key: str) -> dict | None:
        return self.records.get(key)

    def put(self, key: str, record: dict) -> None:
        self.records[key] = record

    def save(self) -> None:
        self.path.parent.mkdir(parents=True, exist_ok=True)
        tmp = self.path.with_suffix(self.path.suffix + f".tmp{os.getpid()}")
        tmp.write_text(json.dumps(self.records, indent=1, sort_keys=True))
        os.replace(tmp, self.path)


def _plan_runner(session, annot, window_starts, nvecs, step, seed, rand_dist, reps):
    """Times one candidate on the device; returns (ms, ldscore)."""
    from .session import WinPlan

    def run(cand: dict):
        plan = WinPlan(session, annot, window_starts, nvecs, step, seed, rand_dist,
                       batch_gb=float(cand["batch_gb"]))
        try:
            _apply(plan, cand)
            plan.execute()  # captures the graph
            ld = plan.results(meansq=False)["ldscore"]
            best = math.inf
            for _ in range(max(1, reps)):
                plan.execute()
                best = min(best, float(sum(plan.kernel_ms().values())))
            return best, ld
        finally:
            plan.close()

    return run


def select(candidates: Iterable[dict], run: Callable[[dict], tuple]) -> dict:
    """Runs every candidate, checks that their scores agree bit for bit and
    returns the record of the fastest."""
    trials, ref = [], None
    for cand in candidates:
        ms, ld = run(cand)
        ld = np.asarray(ld)
        if ref is None:
            ref = ld
        elif not np.array_equal(ld, ref):
            raise RuntimeError(f"tiling {cand} changed the LD scores")
        trials.append({"config": dict(cand), "ms": round(float(ms), 4)})
    if not trials:
        raise ValueError("no candidates")
    best = min(trials, key=lambda t: t["ms"])
    return {"config": best["config"], "ms": best["ms"], "trials": trials,
            "tuned_at": time.strftime("%Y-%m-%dT%H:%M:%SZ", time.gmtime())}


def tune_windowed(session, annot, window_starts, nvecs: int, step: int, seed: int,
                  rand_dist: str = "rademacher", candidates: Iterable[dict] | None = None,
                  reps: int = 2, cache: TuneCache | None = None, force: bool = False,
                  run: Callable[[dict], tuple] | None = None) -> dict:
    """Tuned record for this workload: from the cache, or measured and stored."""
    annot = np.ascontiguousarray(annot, dtype=np.float64)
    cache = cache if cache is not None else TuneCache()
    key = workload_key(f"{device_name()}|{library_id()}", session.N, annot.shape[0],
                       annot.shape[1], nvecs, window_starts)
    if not force:
        hit = cache.get(key)
        if hit is not None:
            return dict(hit, key=key, cached=True)
    run = run or _plan_runner(session, annot, window_starts, nvecs, step, seed, rand_dist, reps)
    record = select(list(candidates or default_candidates()), run)
    cache.put(key, record)
    cache.save()
    return dict(record, key=key, cached=False)


def tuned_win_plan(session, annot, window_starts, nvecs: int, step: int, seed: int,
                   rand_dist: str = "rademacher", cache: TuneCache | None = None,
                   tune_if_missing: bool = True, **plan_kw):
    """A WinPlan with the tuned tiling of this workload (defaults when the
    cache has no record and tuning is off)."""
    from .session import WinPlan

    cache = cache if cache is not None else TuneCache()
    annot = np.ascontiguousarray(annot, dtype=np.float64)
    key = workload_key(f"{device_name()}|{library_id()}", session.N, annot.shape[0],
                       annot.shape[1], nvecs, window_starts)
    rec = cache.get(key)
    if rec is None and tune_if_missing:
        rec = tune_windowed(session, annot, window_starts, nvecs, step, seed, rand_dist,
                            cache=cache)
    cfg = dict(DEFAULT_CONFIG, **(rec["config"] if rec else {}))
    plan = WinPlan(session, annot, window_starts, nvecs, step, seed, rand_dist,
                   batch_gb=float(cfg["batch_gb"]), **plan_kw)
    _apply(plan, cfg)
    return plan
