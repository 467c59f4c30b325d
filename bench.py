#!/usr/bin/env python3
"""Benchmark of the genotype x probe hot path: windowed + partitioned LD scores.

Workload (one "step" = one complete estimate over one synthetic BED batch):
    N = 50,000 samples x M = 500,000 SNPs (HWE hard calls, AR(1) latent LD,
    1% missing), contiguous windows of 200-5,000 SNPs (log-uniform sizes),
    K = 24 Bernoulli(0.1) annotations, B = 50 Rademacher probes, SNP blocks of
    1,000 (the reference's default --block-size), mean imputation; all windows
    in one CUDA-graph launch.  The genome-wide form of the same workload is
    reported beside it (``genome_wide``).
Metric: geno x probe TOPS = (2 N nnz(A) B  [phase 1]  +  2 N M K B  [phase 2]) / time,
2 ops per multiply-accumulate (nnz over window x annotation members).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

``value`` is device time of the estimate's kernels with the genotype image
resident in HBM (CUDA events on the library stream, max over ranks); ``e2e``
is the same estimate through the C ABI (lds_gw_ldscore) from pinned host
buffers, host<->device copies included.  ``--impl reference`` times the
reference's own native CPU code (compiled unchanged into oracle/_ref) on a
bounded SNP sample of the same workload with all host cores.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

N_SAMPLES = 50_000
M_SNPS = 500_000
K_BINS = 24
B_PROBES = 50
BLOCK = 1_000
DATA_SEED = 20260501
ANNOT_SEED = 7
PROBE_SEED = 12345
WINDOW_SEED = 2025
METRIC = "geno x probe TOPS (windowed + partitioned LD scores)"
WORKLOAD = "windowed_partitioned_ldscore_n50k_m500k_w200-5000_k24_b50_rademacher"


def annotations(m: int, k: int = K_BINS) -> np.ndarray:
    rng = np.random.default_rng(ANNOT_SEED)
    return (rng.random((m, k)) < 0.1).astype(np.float64)


def windows(m: int, seed: int = WINDOW_SEED) -> np.ndarray:
    """Contiguous window starts with log-uniform sizes in [200, 5000] (last may be shorter)."""
    rng = np.random.default_rng(seed)
    starts = [0]
    while starts[-1] < m:
        size = int(np.exp(rng.uniform(np.log(200.0), np.log(5000.0))))
        starts.append(min(m, starts[-1] + size))
    return np.asarray(starts, dtype=np.int64)


def algorithmic_ops(n: int, annot: np.ndarray, b: int) -> tuple[float, float]:
    """(phase-1 ops, phase-2 ops), 2 per multiply-accumulate."""
    nnz = float((annot > 0).sum())
    m, k = annot.shape
    return 2.0 * n * nnz * b, 2.0 * n * m * k * b


def env_int(name: str, default: int) -> int:
    try:
        return int(os.environ.get(name, default))
    except ValueError:
        return default


# ---------------------------------------------------------------------------
# clocks sampler (nvidia-smi during the timed region)
# ---------------------------------------------------------------------------
class Clocks:
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def __enter__(self):
        try:
            self.p = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self.f, stderr=subprocess.DEVNULL)
        except (OSError, ValueError):
            self.p = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.p is not None:
            self.p.terminate()
            try:
                self.p.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.p.kill()

    def summary(self) -> dict:
        self.f.flush()
        self.f.seek(0)
        rows = [r.split(",") for r in self.f.read().strip().splitlines() if r.strip()]
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                mx = max(mx, float(r[2]))
                for nm, v in zip(names, r[5:9]):
                    if v.strip().lower() == "active":
                        reasons.add(nm)
            except (ValueError, IndexError):
                continue
        load = [s for s in sm if s > 0.5 * mx] or sm
        return {"sm_mhz": statistics.median(load) if load else None,
                "sm_max_mhz": mx or None, "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
# CPU legs: the reference's own native code on a bounded SNP sample
# ---------------------------------------------------------------------------
def reference_sample(m_sample: int, tmpdir: str, packed=None) -> tuple[str, np.ndarray]:
    """Write the first m_sample SNPs of the workload as a BED fileset.

    ``packed`` (the workload's rows, when already generated) is sliced;
    otherwise the rows come from the CPU copy of the generator in oracle/."""
    from summit_b200 import bedfile

    if packed is None:
        from oracle.oracle import Oracle

        packed = Oracle().synth_bed_rows(N_SAMPLES, m_sample, DATA_SEED)
    prefix = bedfile.write_plink(Path(tmpdir) / f"sample{m_sample}", packed=packed[:m_sample],
                                 n=N_SAMPLES)
    return prefix, annotations(M_SNPS)[:m_sample]


def run_reference_windows(packed: np.ndarray, annot: np.ndarray, ws: np.ndarray, threads: int,
                          tmpdir: str) -> float:
    """The reference's per-block native calls run window by window (each window
    is the genome-wide estimator on its SNPs, probe root window_seed(seed, w));
    returns seconds of reference compute."""
    from oracle.oracle import Reference
    from summit_b200 import bedfile
    from summit_b200.bedfile import mix64

    ref = Reference()
    ref.set_threads(threads)
    total = 0.0
    sys.stderr.flush()
    saved = os.dup(2)
    devnull = os.open(os.devnull, os.O_WRONLY)
    os.dup2(devnull, 2)
    try:
        for w in range(len(ws) - 1):
            a, c = int(ws[w]), int(ws[w + 1])
            pre = bedfile.write_plink(Path(tmpdir) / f"win{w}", packed=packed[a:c], n=N_SAMPLES)
            seed_w = int(mix64(np.uint64(PROBE_SEED) ^ mix64(np.uint64(0x77696E646F77 + w))))
            t0 = time.perf_counter()
            ref.gw_ldscore(pre, N_SAMPLES, c - a, annot[a:c], B_PROBES, BLOCK, seed_w,
                           dist="rademacher", impute="mean", dtype=np.float32)
            total += time.perf_counter() - t0
    finally:
        os.dup2(saved, 2)
        os.close(saved)
        os.close(devnull)
    return total


def run_reference(prefix: str, annot: np.ndarray, threads: int) -> float:
    """One reference estimate (float32, the CLI default dtype); returns seconds.

    The reference prints a per-block "[phase2-watch]" line on stderr; it is
    silenced for the duration of the run."""
    from oracle.oracle import Reference

    ref = Reference()
    ref.set_threads(threads)
    m = annot.shape[0]
    sys.stderr.flush()
    saved = os.dup(2)
    devnull = os.open(os.devnull, os.O_WRONLY)
    os.dup2(devnull, 2)
    try:
        t0 = time.perf_counter()
        ref.gw_ldscore(prefix, N_SAMPLES, m, annot, B_PROBES, BLOCK, PROBE_SEED,
                       dist="rademacher", impute="mean", dtype=np.float32)
        return time.perf_counter() - t0
    finally:
        os.dup2(saved, 2)
        os.close(saved)
        os.close(devnull)


def cpu_threads() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def calibrated_reference(target_s: float, tmpdir: str, threads: int, packed=None):
    """Pick a SNP sample whose reference run takes about target_s seconds."""
    m0 = 2000
    prefix, annot = reference_sample(m0, tmpdir, packed)
    t = run_reference(prefix, annot, threads)
    m = int(min(M_SNPS, max(m0, round(m0 * target_s / max(t, 1e-3) / BLOCK) * BLOCK)))
    if m != m0:
        prefix, annot = reference_sample(m, tmpdir, packed)
    return prefix, annot, m


def reference_sample_windows(target_s: float, threads: int, tmpdir: str, packed=None):
    """Leading windows of the workload totalling about target_s seconds of reference work."""
    ws_all = windows(M_SNPS)
    annot_all = annotations(M_SNPS)
    # calibrate on the first window(s) covering >= 2000 SNPs
    k = int(np.searchsorted(ws_all, 2000)) + 1
    m_cal = int(ws_all[k])
    if packed is None:
        from oracle.oracle import Oracle

        packed = Oracle().synth_bed_rows(N_SAMPLES, m_cal, DATA_SEED)
    t = run_reference_windows(packed[:m_cal], annot_all, ws_all[:k + 1], threads, tmpdir)
    m_target = min(M_SNPS, int(m_cal * target_s / max(t, 1e-3)))
    k = max(1, int(np.searchsorted(ws_all, m_target)))
    m_s = int(ws_all[k])
    if packed.shape[0] < m_s:
        from oracle.oracle import Oracle

        packed = Oracle().synth_bed_rows(N_SAMPLES, m_s, DATA_SEED)
    return packed[:m_s], annot_all[:m_s], ws_all[:k + 1]


def reference_arm(args) -> None:
    rank = env_int("RANK", 0)
    if rank != 0:
        return
    threads = cpu_threads()
    os.environ.setdefault("OMP_NUM_THREADS", str(threads))
    with tempfile.TemporaryDirectory() as td:
        packed, annot, ws = reference_sample_windows(float(os.environ.get("LDS_REF_STEP_S", "8")),
                                                     threads, td)
        ops = sum(algorithmic_ops(N_SAMPLES, annot, B_PROBES))
        for _ in range(args.warmup):
            run_reference_windows(packed, annot, ws, threads, td)
        times = [run_reference_windows(packed, annot, ws, threads, td) for _ in range(args.steps)]
    from oracle.oracle import Reference

    sec = float(np.mean(times))
    value = ops / sec / 1e12
    m = packed.shape[0]
    sample = (f"first {len(ws) - 1} windows ({m} of {M_SNPS} SNPs), N={N_SAMPLES}, K={K_BINS}, "
              f"B={B_PROBES}; reference gwldcore.cpp+genotype.cpp compiled unchanged (float32 "
              f"path) run per window, OpenMP+{' '.join(Reference().blas_config().split()[0:2])}")
    line = {
        "impl": "reference", "metric": METRIC, "value": round(value, 6), "unit": "TOPS",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(sec * 1e3, 3), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": WORKLOAD, "sample_snps": m, "sample_windows": len(ws) - 1,
                   "l2": "inputs larger than L2"},
        "cpu_baseline": {"value": round(value, 6), "unit": "TOPS", "cores": threads,
                         "kind": "reference", "sample": sample},
        "e2e": {"value": round(value, 6), "unit": "TOPS", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------
def read_traffic() -> dict | None:
    """DRAM bytes of the windowed phase-2 kernel per full-size estimate, from the
    committed ncu summary (a captured launch scaled by the CTA count)."""
    f = ROOT / "profiles" / "p2_kernel_windowed_n50k_m100k.md"
    if not f.exists():
        return None
    for line in f.read_text().splitlines():
        if line.startswith("traffic_bytes_per_estimate:"):
            try:
                return {"bytes": float(line.split(":", 1)[1].strip())}
            except ValueError:
                return None
    return None


def ld_errors(est, truth) -> dict:
    """Relative error of each bin's mean LD score (max over bins; the
    reference's accuracy metric, manuscript/scripts/ld/numvec_error.py:86) and
    the per-SNP relative RMSE (mean over bins)."""
    est, truth = np.asarray(est, dtype=np.float64), np.asarray(truth, dtype=np.float64)
    mean_rel = np.abs(est.mean(0) - truth.mean(0)) / np.abs(truth.mean(0))
    rr = np.sqrt(((est - truth) ** 2).mean(0)) / np.sqrt((truth ** 2).mean(0))
    return {"mean_ld_rel_err": round(float(mean_rel.max()), 6),
            "snp_rel_rmse": round(float(rr.mean()), 5)}


def learned_vs_plain(sess, annot, ws, stream) -> dict:
    """LD-score time and error of the plain windowed estimator and of the
    learned control variate (B = 10) on the same resident image, compared
    with the exact expectation of the estimator (exact windowed Gram
    kernel) and against the plain estimator at B = 1,000.  Wall times are
    from the resident image to host results (plan set-up, probe streams and
    any training included), with every code path warmed once beforehand,
    the better of two independent runs for each estimator; device times the
    better of two steady-state executes."""
    import math

    import torch

    from summit_b200 import _lib
    from summit_b200.learned_cv import CvConfig, LearnedCV
    from summit_b200.session import WinPlan

    lib = _lib.load()
    out = {}
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    truth = sess.partition_ld_expectation(annot, ws)
    wall = time.perf_counter() - t0
    buf = np.zeros(4)
    lib.lds_last_timings(_lib.ptr(buf), 4)
    out["exact"] = {"wall_ms": round(wall * 1e3, 1), "device_ms": round(float(buf[0]), 2),
                    "mean_ld_rel_err": 0.0, "snp_rel_rmse": 0.0,
                    "method": "exact expectation of the estimator (int8 Gram tensor-core kernel)"}

    # Both estimators get the same treatment: wall = the better of two
    # independent runs from the resident image (plan set-up to host results),
    # device = the better of two steady-state executes.
    def plain(B, device=True, seed=PROBE_SEED, reps=2):
        wall, dev, ld = math.inf, math.inf, None
        for _ in range(reps):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            p = WinPlan(sess, annot, ws, B, BLOCK, seed, "rademacher")
            p.execute()
            ld = p.results()["ldscore"]
            wall = min(wall, time.perf_counter() - t0)
            if device:
                for _ in range(2):
                    e0 = torch.cuda.Event(enable_timing=True)
                    e1 = torch.cuda.Event(enable_timing=True)
                    e0.record(stream)
                    p.execute()
                    e1.record(stream)
                    torch.cuda.synchronize()
                    dev = min(dev, e0.elapsed_time(e1))
            p.close()
        rec = {"B": B, "wall_ms": round(wall * 1e3, 1), **ld_errors(ld, truth)}
        if device:
            rec["device_ms"] = round(dev, 2)
        return ld, rec

    _, out["plain_b10"] = plain(10)
    p100, out["plain_b100"] = plain(100)
    p1000, out["plain_b1000"] = plain(1000, device=False, seed=PROBE_SEED + 7, reps=1)
    cfg = CvConfig(nvecs=10)
    # Warm the code paths once (first use of the torch and network kernels
    # loads them), as the plain runs above are warm from the headline runs;
    # the timed run below then builds everything afresh from the image.
    warm = LearnedCV(sess, annot, ws, BLOCK, PROBE_SEED + 2, cfg=cfg)
    warm.run()
    warm.close()
    wall, best = math.inf, None
    for _ in range(2):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        cv = LearnedCV(sess, annot, ws, BLOCK, PROBE_SEED + 1, cfg=cfg)
        res = cv.run()
        torch.cuda.synchronize()
        wall = min(wall, time.perf_counter() - t0)
        for _ in range(2):
            res = cv.run()  # steady state (graph captured, workspace allocated)
            if best is None or res["timings"]["total_ms"] < best["timings"]["total_ms"]:
                best = res
        cv.close()
    res = best
    ld = res["ldscore"].double().cpu().numpy()
    near = res["nearcv_ldscore"].double().cpu().numpy()
    out["learned_b10"] = {"B": 10, "wall_ms": round(wall * 1e3, 1),
                          "device_ms": round(res["timings"]["total_ms"], 2),
                          "stages_ms": {k: round(v, 2) for k, v in res["timings"].items()},
                          **ld_errors(ld, truth),
                          "near_field_only": ld_errors(near, truth)}
    # Plain probes needed for the learned estimator's per-SNP error (error ~ B^-1/2).
    ratio = out["plain_b100"]["snp_rel_rmse"] / max(out["learned_b10"]["snp_rel_rmse"], 1e-12)
    b_eq = int(math.ceil(100.0 * ratio * ratio / 10.0) * 10)
    if b_eq <= 2000:
        _, out["plain_matched"] = plain(b_eq)  # same seed as above: the same estimate each rep
        out["speedup_at_matched_snp_error"] = {
            "wall": round(out["plain_matched"]["wall_ms"] / out["learned_b10"]["wall_ms"], 2),
            "device": round(out["plain_matched"]["device_ms"] / out["learned_b10"]["device_ms"], 2)}
    out["vs_plain_b1000"] = {"learned_b10": ld_errors(ld, p1000),
                                "plain_b100": ld_errors(p100, p1000)}
    out["time_to_1pct"] = time_to_target(sess, annot, ws, truth, target=0.01)
    out["error_metric"] = ("mean_ld_rel_err: max over bins of |mean est - mean truth| / |mean truth|; "
                           "snp_rel_rmse: per-SNP RMS error / RMS truth, mean over bins")
    return out


def time_to_target(sess, annot, ws, truth, target: float = 0.01, sweep=(2, 4, 6, 10),
                   seeds: int = 3) -> dict:
    """The metric's own criterion: wall time to reach <= `target` relative
    error of every bin's mean LD score (the reference's accuracy metric,
    numvec_error.py:86) against the exact expectation.  Each estimator runs at
    the probe counts of `sweep` with `seeds` independent probe seeds; a count
    qualifies when its worst seed meets the target, and the estimator's time is
    the median wall time (resident image to host results) at the smallest
    qualifying count."""
    import torch

    from summit_b200.learned_cv import CvConfig, LearnedCV
    from summit_b200.session import WinPlan

    def run_plain(B, seed):
        p = WinPlan(sess, annot, ws, B, BLOCK, seed, "rademacher")
        p.execute()
        ld = p.results()["ldscore"]
        p.close()
        return ld

    def run_learned(B, seed):
        cv = LearnedCV(sess, annot, ws, BLOCK, seed, cfg=CvConfig(nvecs=B))
        ld = cv.run()["ldscore"].double().cpu().numpy()
        cv.close()
        return ld

    out = {"target": target, "seeds": seeds, "criterion": "max over seeds of the max over bins "
           "of |mean est - mean exact| / |mean exact|"}
    for name, fn in (("plain", run_plain), ("learned", run_learned)):
        fn(sweep[0], PROBE_SEED + 500)  # warm this path's kernels
        rows = []
        for B in sweep:
            errs, walls = [], []
            for s in range(seeds):
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                ld = fn(B, PROBE_SEED + 300 + 17 * s)
                torch.cuda.synchronize()
                walls.append((time.perf_counter() - t0) * 1e3)
                errs.append(ld_errors(ld, truth)["mean_ld_rel_err"])
            rows.append({"B": B, "max_mean_ld_rel_err": round(max(errs), 6),
                         "wall_ms": round(float(np.median(walls)), 1)})
        hit = next((r for r in rows if r["max_mean_ld_rel_err"] <= target), None)
        out[name] = {"sweep": rows, "B": None if hit is None else hit["B"],
                     "wall_ms": None if hit is None else hit["wall_ms"]}
    if out["plain"]["wall_ms"] and out["learned"]["wall_ms"]:
        out["learned_speedup"] = round(out["plain"]["wall_ms"] / out["learned"]["wall_ms"], 2)
    return out


def ours_arm(args) -> None:
    import torch

    rank = env_int("RANK", 0)
    world = env_int("WORLD_SIZE", 1)
    local = env_int("LOCAL_RANK", 0)
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))

    from summit_b200 import _lib, gwldcore
    from summit_b200.session import GwSession, WinPlan, set_stream, windowed_ldscore

    lib = _lib.load()
    stream = torch.cuda.Stream()
    set_stream(stream.cuda_stream)

    n, m = N_SAMPLES, env_int("LDS_BENCH_M", M_SNPS)
    seed = DATA_SEED + rank  # weak scaling: every rank estimates its own batch
    pinned = torch.empty((m, (n + 3) // 4), dtype=torch.uint8, pin_memory=True)
    bed_host = gwldcore.synth_bed_rows(n, m, seed, out=pinned.numpy())
    annot = annotations(m)
    ws = windows(m)
    ops1, ops2 = algorithmic_ops(n, annot, B_PROBES)
    ops = ops1 + ops2

    def barrier():
        if dist is not None:
            dist.barrier()

    def timed(execute, steps):
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        barrier()
        torch.cuda.synchronize()
        ev0.record(stream)
        for _ in range(steps):
            execute()
        ev1.record(stream)
        torch.cuda.synchronize()
        barrier()
        return ev0.elapsed_time(ev1) / steps

    sess = GwSession(bed_host, n, impute_mode="mean")

    # ---- tiling of the windowed plans: the project's autotuner, timed on this
    # device before the measured region (phase-1 split, window batching,
    # phase-2 CTA order; every candidate's scores must agree bit for bit) ----
    from summit_b200 import autotune

    cands = ([{"p1_sb_per_cta": s, "batch_gb": 8.0} for s in (8, 16, 32, 64, 128)] +
             [{"p1_sb_per_cta": 64, "batch_gb": b} for b in (4.0, 16.0)] +
             [{"p1_sb_per_cta": 128, "batch_gb": 8.0, "p2_bin_chunk": c} for c in (0, 12, 24)] +
             [{"p1_sb_per_cta": 128, "batch_gb": 8.0, "p2_bin_chunk": 2, "p2_bins": 1}])
    t_tune = time.perf_counter()
    tune = autotune.tune_windowed(sess, annot, ws, B_PROBES, BLOCK, PROBE_SEED, "rademacher",
                                  candidates=cands, reps=1)
    tune_s = time.perf_counter() - t_tune

    # ---- headline: windowed + partitioned, one graph launch per estimate ----
    wplan = autotune.tuned_win_plan(sess, annot, ws, B_PROBES, BLOCK, PROBE_SEED, "rademacher",
                                    tune_if_missing=False)
    for _ in range(args.warmup):
        wplan.execute()
    torch.cuda.synchronize()
    wplan.kernel_ms()
    launches0 = lib.lds_kernel_launches()
    with Clocks(local) as clk:
        ms = timed(wplan.execute, args.steps)
    launches = int(lib.lds_kernel_launches() - launches0)
    kms = wplan.kernel_ms()  # last estimate, per kernel kind (events inside the graph)
    res = wplan.results()
    assert np.isfinite(res["ldscore"]).all()
    # graph launches run kernels the launch counter does not see: count them per graph
    wplan.close()

    # ---- the same estimate with exact product checks (tensor-core checksums
    # against a CUDA-core recomputation, compared on the host) ----
    product_checks = None
    if not os.environ.get("LDS_SKIP_CHECKS"):
        cplan = autotune.tuned_win_plan(sess, annot, ws, B_PROBES, BLOCK, PROBE_SEED, "rademacher",
                                        tune_if_missing=False)
        cplan.set_checks(True)
        for _ in range(args.warmup):
            cplan.execute()
        torch.cuda.synchronize()
        cms = timed(cplan.execute, args.steps)
        chk = cplan.check_products()
        same = bool(np.array_equal(cplan.results()["ldscore"], res["ldscore"]))
        cplan.close()
        if chk["mismatches"] or not same:
            raise RuntimeError(f"product checks failed: {chk['mismatches']} SNPs, "
                               f"scores identical: {same}")
        product_checks = {"ms_per_step": round(cms, 3), "overhead": round(cms / ms - 1.0, 4),
                          "check_kernels_ms": round(chk["check_ms"], 3), "mismatches": 0,
                          "scores_identical": same}

    # ---- secondary: genome-wide form of the same workload ----
    plan = sess.plan(annot, B_PROBES, BLOCK, PROBE_SEED, "rademacher")
    for _ in range(args.warmup):
        plan.execute()
    torch.cuda.synchronize()
    plan.kernel_ms()
    gw_ms = timed(plan.execute, args.steps)
    gw_kms = plan.kernel_ms()
    plan.close()

    # ---- the same windowed estimate on an HWE-completed image: no call is
    # missing after imputation, so phase 2 runs no observed-count products ----
    hwe = None
    if not os.environ.get("LDS_SKIP_HWE"):
        sess_h = GwSession(bed_host, n, impute_mode="hwe", impute_seed=PROBE_SEED)
        hplan = autotune.tuned_win_plan(sess_h, annot, ws, B_PROBES, BLOCK, PROBE_SEED,
                                        "rademacher", tune_if_missing=False)
        for _ in range(args.warmup):
            hplan.execute()
        torch.cuda.synchronize()
        hplan.kernel_ms()
        h_ms = timed(hplan.execute, args.steps)
        hkms = hplan.kernel_ms()
        hplan.close()
        sess_h.close()
        hwe = {"value": round(world * ops / (h_ms * 1e-3) / 1e12, 3), "unit": "TOPS",
               "ms_per_step": round(h_ms, 3), "impute": "hwe",
               "kernel_ms": {k: round(v, 3) for k, v in hkms.items()}}

    # ---- learned control variate vs plain (config-2 shape, B = 10 vs 100) ----
    lvp = None
    if rank == 0 and not os.environ.get("LDS_SKIP_LEARNED"):
        lvp = learned_vs_plain(sess, annot, ws, stream)

    # ---- end to end through the one-call C ABI entry from pinned host buffers ----
    chunks = env_int("LDS_E2E_CHUNKS", 8)

    def e2e_once():
        return windowed_ldscore(bed_host, n, annot, ws, B_PROBES, BLOCK, PROBE_SEED,
                                "rademacher", impute_mode="mean", chunks=chunks,
                                tiling=tune["config"])

    e2e_steps = max(1, env_int("LDS_E2E_STEPS", args.steps))
    e2e_once()  # warm
    torch.cuda.synchronize()
    barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        out = e2e_once()
    torch.cuda.synchronize()
    e2e_ms = (time.perf_counter() - t0) * 1e3 / e2e_steps
    stage = np.zeros(4)
    lib.lds_last_timings(_lib.ptr(stage), 4)  # host stage times of the last call
    barrier()
    assert np.allclose(out["ldscore"], res["ldscore"], rtol=0, atol=0)
    nnz = int((annot > 0).sum())
    # uploads: BED rows, member lists (index + scale), per-SNP scale and window
    # index, per-window bin totals; downloads: per-SNP code counts and LD scores
    nw = int(len(ws) - 1)
    h2d = int(bed_host.nbytes + nnz * 12 + m * 12 + nw * K_BINS * 8)
    d2h = int(m * 16 + m * K_BINS * 8)
    sess.close()

    t = torch.tensor([ms, e2e_ms, gw_ms], dtype=torch.float64, device="cuda")
    if dist is not None:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms, e2e_ms, gw_ms = float(t[0]), float(t[1]), float(t[2])

    if rank == 0:
        peaks = {}
        pf = ROOT / "MEASURED_PEAKS.json"
        if pf.exists():
            peaks = json.loads(pf.read_text())
        peak = float(peaks.get("bf16_tflops", 1590.0))
        p2_ms = kms["phase2"]
        achieved = ops2 / (p2_ms * 1e-3) / 1e12 if p2_ms > 0 else None
        tr = read_traffic()
        clocks = clk.summary()
        line = {
            "metric": METRIC, "value": round(world * ops / (ms * 1e-3) / 1e12, 3), "unit": "TOPS",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(ms, 3), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "int8-digit exact products, f64 epilogue",
            "data": "synthetic (seeded HWE/AR(1) generator on device)",
            "config": {"workload": WORKLOAD, "N": n, "M": m, "windows": int(len(ws) - 1),
                       "K": K_BINS, "B": B_PROBES, "block": BLOCK, "impute": "mean",
                       "digits": lib.lds_get_slices(), "parallelism": f"partition x{world} (each rank its own chromosome; no collective)",
                       "graph": "one CUDA graph launch per estimate",
                       "tiling": {"config": tune["config"], "tuned_ms": tune["ms"],
                                  "cached": tune["cached"], "tune_s": round(tune_s, 1),
                                  "trials": tune.get("trials")},
                       "l2": "inputs larger than L2 (6.3 GB genotype image per step)"},
            "kernel_ms": {k: round(v, 3) for k, v in kms.items()},
            "genome_wide": {"value": round(world * ops / (gw_ms * 1e-3) / 1e12, 3),
                            "unit": "TOPS", "ms_per_step": round(gw_ms, 3),
                            "kernel_ms": {k: round(v, 3) for k, v in gw_kms.items()}},
            "roofline": {
                "kernel": "p2_umma_kernel (windowed phase 2: X^T Y + LD epilogue, all launches "
                          "of one estimate)", "bound": "tensor",
                "achieved": None if achieved is None else round(achieved, 3),
                "peak": peak, "unit": "TFLOP/s",
                "frac": None if achieved is None else round(achieved / peak, 4),
                "peak_source": "MEASURED_PEAKS.json bf16_tflops (burst)" if peaks else "fallback",
                "traffic": None if tr is None else tr["bytes"],
                "traffic_source": "profiles/p2_kernel_windowed_n50k_m100k.md (per estimate)",
                "algorithmic_ops_per_launch": ops2},
            "e2e": {"value": round(world * ops / (e2e_ms * 1e-3) / 1e12, 3), "unit": "TOPS",
                    "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "ms_per_step": round(e2e_ms, 1), "steps": e2e_steps,
                    "call": f"lds_win_ldscore (upload streamed in window-aligned chunks, n_chunks={chunks})",
                    "stages_ms": {"first_estimate_enqueued": round(float(stage[0]), 1),
                                  "all_enqueued": round(float(stage[1]), 1),
                                  "results_copied": round(float(stage[2]), 1),
                                  "buffers_released": round(float(stage[3]), 1)}},
            "gpu_launches": launches,
            "clocks": clocks,
        }
        if hwe is not None:
            line["windowed_hwe"] = hwe
        if product_checks is not None:
            line["product_checks"] = product_checks
        if lvp is not None:
            line["learned_vs_plain"] = lvp
        if world == 1 and not os.environ.get("LDS_SKIP_CPU_BASELINE"):
            threads = cpu_threads()
            with tempfile.TemporaryDirectory() as td:
                pk, ann_s, ws_s = reference_sample_windows(
                    float(os.environ.get("LDS_CPU_BASELINE_S", "12")), threads, td, bed_host)
                sec = run_reference_windows(pk, ann_s, ws_s, threads, td)
            cops = sum(algorithmic_ops(n, ann_s, B_PROBES))
            line["cpu_baseline"] = {
                "value": round(cops / sec / 1e12, 6), "unit": "TOPS", "cores": threads,
                "kind": "reference",
                "sample": f"first {len(ws_s) - 1} windows ({pk.shape[0]} SNPs) of the workload "
                          f"(N={n}, K={K_BINS}, B={B_PROBES}); reference gwldcore.cpp compiled "
                          f"unchanged, float32, run per window, {sec:.1f} s"}
        print(json.dumps(line), flush=True)

    set_stream(None)
    if dist is not None:
        dist.destroy_process_group()


# ---------------------------------------------------------------------------
# Exact windowed LD scores (winldcore form) over the config-2 windows: unbiased
# r^2 within each window (the partition is expressed as base-pair positions 1e9
# apart between windows and a 5 kb window), tensor-core Gram products.
# Value: 2 N sum_w L_w^2 / time (the reference's FP64 SYRK/GEMM work).
# ---------------------------------------------------------------------------
EXACT_METRIC = "pair-product TOPS (exact windowed LD scores, unbiased r^2)"


def partition_positions(ws: np.ndarray) -> np.ndarray:
    win = np.repeat(np.arange(ws.size - 1), np.diff(ws))
    return (win.astype(np.int64) * 1_000_000_000 + (np.arange(ws[-1]) - ws[win]) + 1).astype(np.int64)


def exact_arm(args) -> None:
    import torch

    from summit_b200 import _lib, gwldcore
    from summit_b200.session import GwSession

    torch.cuda.set_device(env_int("LOCAL_RANK", 0))
    n, m = N_SAMPLES, env_int("LDS_BENCH_M", M_SNPS)
    rows = gwldcore.synth_bed_rows(n, m, DATA_SEED)
    pinned = torch.empty(rows.shape, dtype=torch.uint8, pin_memory=True)
    pinned.numpy()[:] = rows
    bed = pinned.numpy()  # the end-to-end copy starts from pinned host memory
    del rows
    annot = annotations(m)
    ws = windows(m)
    win = np.repeat(np.arange(ws.size - 1), np.diff(ws))
    lo, hi = ws[win], ws[win + 1]
    ops = 2.0 * n * float((np.diff(ws).astype(np.float64) ** 2).sum())
    lib = _lib.load()
    sess = GwSession(bed, n)
    buf = np.zeros(4)
    for _ in range(args.warmup):
        sess.window_ld(lo, hi, annot, corr_dim=n - 1)
    times, gram = [], []
    launches0 = lib.lds_kernel_launches()
    with Clocks(env_int("LOCAL_RANK", 0)) as clk:
        for _ in range(args.steps):
            out = sess.window_ld(lo, hi, annot, corr_dim=n - 1)
            lib.lds_last_timings(buf.ctypes.data_as(__import__("ctypes").c_void_p), 4)
            times.append(float(buf[0]))
            gram.append(float(buf[1]))
    launches = int(lib.lds_kernel_launches() - launches0) // max(args.steps, 1)
    ms = float(np.mean(times))
    gram_ms = float(np.mean(gram))
    pf = ROOT / "MEASURED_PEAKS.json"
    peaks = json.loads(pf.read_text()) if pf.exists() else {}
    peak = float(peaks.get("bf16_tflops", 1590.0))
    # Tensor-core work the Gram kernel issues: 4 int8 planes (GG, GO, OG, OO)
    # over every 128 x 128 tile pair of the band, 2 N_pad ops per product.
    tiles = 0
    for w in range(ws.size - 1):
        t = -(-int(ws[w + 1] - ws[w]) // 128)
        tiles += t * t
    issued = 4.0 * 2.0 * 128 * 128 * (-(-n // 256) * 256) * tiles
    t0 = time.perf_counter()
    s2 = GwSession(bed, n)
    out2 = s2.window_ld(lo, hi, annot, corr_dim=n - 1)
    e2e_s = time.perf_counter() - t0
    s2.close()
    assert np.array_equal(out, out2)
    line = {"metric": EXACT_METRIC, "value": round(ops / (ms * 1e-3) / 1e12, 3), "unit": "TOPS",
            "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms, 2),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "int8 exact Gram sums, f64 r and sums", "data": "synthetic",
            "config": {"workload": "exact_windowed_ld_n50k_m500k_w200-5000_k24", "N": n, "M": m,
                       "windows": int(ws.size - 1), "K": K_BINS,
                       "snp_pairs": float((np.diff(ws).astype(np.float64) ** 2).sum())},
            "e2e": {"value": round(ops / e2e_s / 1e12, 3), "unit": "TOPS",
                    "h2d_bytes_per_step": int(bed.nbytes + annot.nbytes + lo.nbytes + hi.nbytes),
                    "d2h_bytes_per_step": int(out.nbytes), "ms_per_step": round(e2e_s * 1e3, 1)},
            "kernel_ms": {"gram_ld": round(gram_ms, 3), "total": round(ms, 3)},
            "roofline": {"kernel": "gram_ld_kernel (int8 GG/GO/OG/OO tile products + LD epilogue)",
                         "bound": "tensor", "achieved": round(ops / (gram_ms * 1e-3) / 1e12, 3),
                         "peak": peak, "unit": "TFLOP/s",
                         "frac": round(ops / (gram_ms * 1e-3) / 1e12 / peak, 4),
                         "issued_int8_tops": round(issued / (gram_ms * 1e-3) / 1e12, 3),
                         "peak_source": ("MEASURED_PEAKS.json bf16_tflops (burst)" if peaks
                                         else "fallback"),
                         "traffic": None, "algorithmic_ops_per_launch": ops},
            "gpu_launches": launches, "clocks": clk.summary()}
    if not os.environ.get("LDS_SKIP_CPU_BASELINE"):
        from oracle.oracle import ReferenceWindowed
        from summit_b200 import bedfile

        threads = cpu_threads()
        ref = ReferenceWindowed()
        ref.set_threads(threads)
        k = int(np.searchsorted(ws, env_int("LDS_EXACT_CPU_SNPS", 6000))) + 1
        k = min(k, ws.size - 1)
        ms_ = int(ws[k])
        with tempfile.TemporaryDirectory() as td:
            pre = bedfile.write_plink(Path(td) / "exact", packed=bed[:ms_], n=n)
            bp = partition_positions(ws[:k + 1])
            t0 = time.perf_counter()
            ref.compute_windowed_ld_chr(pre, 0, ms_, bp, annot[:ms_], 5.0, 1000)
            sec = time.perf_counter() - t0
        cops = 2.0 * n * float((np.diff(ws[:k + 1]).astype(np.float64) ** 2).sum())
        line["cpu_baseline"] = {"value": round(cops / sec / 1e12, 6), "unit": "TOPS", "cores": threads,
                                "kind": "reference",
                                "sample": f"first {k} windows ({ms_} SNPs); reference winldcore.cpp "
                                          f"compiled unchanged, FP64 OpenBLAS, {sec:.1f} s"}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# SUMMIT-GxE workload (config-3 shape): N = 100,000 x M = 1,000,000, 8 exposures
# (6 continuous N(0,1) with pairwise correlation 0.2, 2 categorical with 3 and 5
# levels, level-coded and standardized), K = 1 bin, B = 100 Gaussian probes.
# One step = one whole reference build: source panel, projection, sealed pair,
# target scores, normalization.
# ---------------------------------------------------------------------------
GXE_N, GXE_M, GXE_E, GXE_B = 100_000, 1_000_000, 8, 100
GXE_METRIC = "geno x probe TOPS (SUMMIT-GxE multi-environment reference)"
GXE_WORKLOAD = "gxe_reference_n100k_m1m_e8_k1_b100_gaussian"


def gxe_ops(n: int, m: int, E: int, K: int, B: int) -> float:
    """2 N M C (source) + 2 N M 2C (target pair), C = E 2 K B columns."""
    C = E * 2 * K * B
    return 2.0 * n * m * C + 2.0 * n * m * 2 * C


def gxe_reference_sample(n: int, snps: int, threads: int, seed: int = DATA_SEED) -> tuple[float, str]:
    """The reference's gxeldcore.cpp (compiled unchanged) on the first `snps`
    SNPs: source_block + project_sources + target_score_block, dense FP64
    genotypes from the reference's standardization; returns seconds."""
    from oracle.gxe_oracle import design
    from oracle.oracle import Oracle, ReferenceGxe

    os.environ["OMP_NUM_THREADS"] = str(threads)
    ora = Oracle()
    rows = ora.synth_bed_rows(n, snps, seed)
    X = ora.standardize(rows, n, 0, snps)[0]
    d = design(n, GXE_E, seed=3, categorical=2)
    ref = ReferenceGxe()
    ker = ref.kernel(d["environments"], d["feature_basis"], d["power_indices"], d["power_offsets"],
                     d["ranks"], d["gram_values"], d["gram_offsets"], d["e2_gram_values"],
                     d["common_basis"], d["directions"], 1, 1, threads)
    rng = np.random.default_rng(5)
    z = np.asfortranarray(rng.normal(size=(snps, GXE_B)))
    ones = np.ones((snps, GXE_E), order="F")
    cols = GXE_E * 2 * GXE_B
    t0 = time.perf_counter()
    target = np.zeros((n, cols), order="F")
    ker.source_block(target, X, z, np.ones((snps, 1)), ones, ones, 0)
    ker.project_sources(target, GXE_B, 0)
    pair = ker.pair(target, d["environments"])
    accs = [np.zeros((GXE_E * snps, 1)) for _ in range(4)]
    ker.target_score_block(X, pair, ones, ones, accs, 0, snps, GXE_B, 0)
    ker.normalize_scores(accs, GXE_B)
    sec = time.perf_counter() - t0
    ref.lib.refg_pair_destroy(pair)
    return sec, (f"first {snps} SNPs of the workload (N={n}, E={GXE_E}, B={GXE_B}); reference "
                 f"gxeldcore.cpp MultiEnvironmentKernel compiled unchanged, FP64 OpenBLAS, "
                 f"{threads} threads, {sec:.1f} s")


def gxe_arm(args) -> None:
    import torch

    rank = env_int("RANK", 0)
    world = env_int("WORLD_SIZE", 1)
    local = env_int("LOCAL_RANK", 0)
    torch.cuda.set_device(local)
    from summit_b200 import _lib, gwldcore
    from summit_b200.gxe import GxeReference, synthetic_design
    from summit_b200.session import GwSession

    n, m = env_int("LDS_GXE_N", GXE_N), env_int("LDS_GXE_M", GXE_M)
    E, B, K = GXE_E, GXE_B, 1
    # host BED rows in pinned memory (the end-to-end leg uploads them each step)
    pinned = torch.empty((m, (n + 3) // 4), dtype=torch.uint8, pin_memory=True)
    bed = gwldcore.synth_bed_rows(n, m, DATA_SEED + rank, out=pinned.numpy())
    d = synthetic_design(n, E, seed=3, categorical=2)
    dev = torch.device("cuda")
    g = torch.Generator(device=dev)
    g.manual_seed(1234 + rank)
    probes = torch.randn((B, m), generator=g, dtype=torch.float64, device=dev).T
    annot = torch.ones((K, m), dtype=torch.float64, device=dev).T
    scale = torch.ones((E, m), dtype=torch.float64, device=dev).T
    lib = _lib.load()
    keys = ("environments", "feature_basis", "power_indices", "power_offsets", "ranks",
            "gram_values", "gram_offsets", "e2_gram_values", "common_basis", "directions")

    def build(sess):
        gx = GxeReference(sess, *[d[k] for k in keys], annotation_bins=K)
        return gx, gx.run(probes, annot, scale, scale)

    t0 = time.perf_counter()
    sess = GwSession(bed, n)
    torch.cuda.synchronize()
    upload_s = time.perf_counter() - t0
    gx, res = build(sess)  # warm-up
    launches0 = lib.lds_kernel_launches()
    with Clocks(local) as clk:
        times = []
        for _ in range(args.steps):
            res = gx.run(probes, annot, scale, scale)
            times.append(res["timings"]["total"])
    launches = int(lib.lds_kernel_launches() - launches0) // max(args.steps, 1)
    ms = float(np.mean(times))
    ops = gxe_ops(n, m, E, K, B)
    # end to end: host BED rows -> resident image -> scores back on the host
    t0 = time.perf_counter()
    sess2 = GwSession(bed, n)
    gx2, res2 = build(sess2)
    host = {k: res2[k].cpu().numpy() for k in ("accum_xx", "accum_xw", "accum_wx", "accum_ww")}
    e2e_s = time.perf_counter() - t0
    sess2.close()
    for k, v in host.items():
        assert np.isfinite(v).all(), k
    line = {
        "metric": GXE_METRIC, "value": round(world * ops / (ms * 1e-3) / 1e12, 3), "unit": "TOPS",
        "n_gpus": world, "steps": args.steps, "warmup": 1, "ms_per_step": round(ms, 1),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "int8-digit exact products, f64 projection and reductions",
        "data": "synthetic (seeded HWE/AR(1) generator; Gaussian probes on device)",
        "config": {"workload": GXE_WORKLOAD, "N": n, "M": m, "E": E, "K": K, "B": B,
                   "columns": E * 2 * K * B, "scales": "ones (unscaled kernel mode)",
                   "l2": "inputs larger than L2 (genotype image %.1f GB)" % (bed.nbytes / 1e9)},
        "stage_ms": {k: round(v, 1) for k, v in res["timings"].items()},
        "max_leakage": float(np.max(res["leakages"])),
        "e2e": {"value": round(world * ops / e2e_s / 1e12, 3), "unit": "TOPS",
                "h2d_bytes_per_step": int(bed.nbytes), "d2h_bytes_per_step": int(4 * E * m * K * 8),
                "ms_per_step": round(e2e_s * 1e3, 1), "upload_ms": round(upload_s * 1e3, 1)},
        "gpu_launches": launches,
        "clocks": clk.summary(),
    }
    if not os.environ.get("LDS_SKIP_CHECKS"):
        # the same build with the target's exact product checks (outside the
        # timed region): overhead, mismatches, accumulators unchanged
        gxc = GxeReference(sess, *[d[k] for k in keys], annotation_bins=K, product_checks=True)
        resc = gxc.run(probes, annot, scale, scale)
        rc = gxc.last_check()
        same = all(torch.equal(resc[k], res[k])
                   for k in ("accum_xx", "accum_xw", "accum_wx", "accum_ww"))
        line["product_checks"] = {
            "target_ms": round(resc["timings"]["target"], 1),
            "unchecked_target_ms": round(res["timings"]["target"], 1),
            "rows": rc["rows"], "mismatches": rc["mismatches"], "scores_identical": bool(same)}
        gxc.close()
    if rank == 0 and world == 1 and not os.environ.get("LDS_SKIP_CPU_BASELINE"):
        threads = cpu_threads()
        snps = env_int("LDS_GXE_CPU_SNPS", 400)
        sec, sample = gxe_reference_sample(n, snps, threads)
        line["cpu_baseline"] = {"value": round(gxe_ops(n, snps, E, K, B) / sec / 1e12, 6),
                                "unit": "TOPS", "cores": threads, "kind": "reference",
                                "sample": sample}
    if rank == 0:
        print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# Generalized per-variant GxE two-pass estimator (summit_b200.generalized_gxe):
# N = 50,000 x M = 100,000, Q = 3 context bases (1, E, 0.3 E^2 + noise), R = 2
# orthonormal fixed effects, K = 4 continuous annotations (20 % zeros),
# B = 50 global-variant probes.  One step = pass 1 + pass 2 from the resident
# image to host results.
# ---------------------------------------------------------------------------
GEN_N, GEN_M, GEN_Q, GEN_R, GEN_K, GEN_B = 50_000, 100_000, 3, 2, 4, 50
GEN_METRIC = "geno x probe TOPS (generalized per-variant GxE two-pass estimator)"
GEN_WORKLOAD = "generalized_gxe_two_pass_n50k_m100k_q3_r2_k4_b50"


def gen_inputs(n: int, m: int, seed: int = 4242):
    rng = np.random.default_rng(seed)
    env, cov = rng.normal(size=n), rng.normal(size=n)
    basis = np.asfortranarray(np.column_stack([np.ones(n), env, 0.3 * env ** 2 + rng.normal(size=n)]))
    u, _s, _vt = np.linalg.svd(np.column_stack([np.ones(n), cov]), full_matrices=False)
    annot = rng.uniform(0.1, 1.4, size=(m, GEN_K))
    annot[rng.random((m, GEN_K)) < 0.2] = 0.0
    annot[0] = 0.7
    return basis, np.asfortranarray(u), annot


def gen_ops(n: int, annot: np.ndarray, b: int, families: int) -> float:
    """2 ops per MAC: pass 1 X (sqrt(a) o Z) over the annotation nonzeros,
    pass 2 X^T of the K * B * families right-hand-side columns."""
    nnz = float((annot > 0).sum())
    m, k = annot.shape
    return 2.0 * n * nnz * b + 2.0 * n * m * k * b * families


def generalized_arm(args) -> None:
    import torch

    local = env_int("LOCAL_RANK", 0)
    torch.cuda.set_device(local)
    from summit_b200 import _lib, gwldcore
    from summit_b200 import generalized_gxe as gg
    from summit_b200.session import GwSession

    n, m = env_int("LDS_GEN_N", GEN_N), env_int("LDS_GEN_M", GEN_M)
    bed = gwldcore.synth_bed_rows(n, m, DATA_SEED)
    basis, fixed, annot = gen_inputs(n, m)
    spec = gg.GlobalVariantProbeSpec(root_seed=2027, probe_offset=0, probe_count=GEN_B)
    families = GEN_Q * GEN_Q  # fixed effects: every ordered (t, s)
    ops = gen_ops(n, annot, GEN_B, families)

    def run(sess):
        p1, p2 = gg.two_pass(sess, basis, fixed, annot, spec)
        return p2

    sess = GwSession(bed, n)
    p2 = run(sess)  # warm-up
    lib = _lib.load()
    launches0 = lib.lds_kernel_launches()
    times = []
    with Clocks(local) as clk:
        for _ in range(args.steps):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            p2 = run(sess)
            torch.cuda.synchronize()
            times.append(time.perf_counter() - t0)
    launches = int(lib.lds_kernel_launches() - launches0) // max(args.steps, 1)
    assert np.isfinite(p2.directional_ldscores).all()
    sec = float(np.median(times))
    # end to end: host BED rows -> resident image -> both passes -> host results
    t0 = time.perf_counter()
    sess2 = GwSession(bed, n)
    run(sess2)
    e2e_s = time.perf_counter() - t0
    sess2.close()
    line = {
        "metric": GEN_METRIC, "value": round(ops / sec / 1e12, 3), "unit": "TOPS", "n_gpus": 1,
        "steps": args.steps, "warmup": 1, "ms_per_step": round(sec * 1e3, 1),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "int8-digit exact products, f64 projection, scores and diagonals",
        "data": "synthetic (seeded HWE/AR(1) generator; global variant x probe signs on device)",
        "config": {"workload": GEN_WORKLOAD, "N": n, "M": m, "Q": GEN_Q, "R": GEN_R, "K": GEN_K,
                   "B": GEN_B, "rhs_columns": GEN_K * GEN_B * families,
                   "timing": "wall clock from the resident image to host results (host "
                             "orientation-term set-up and PCIe transfers between the steps "
                             "included)"},
        "e2e": {"value": round(ops / e2e_s / 1e12, 3), "unit": "TOPS",
                "h2d_bytes_per_step": int(bed.nbytes),
                "d2h_bytes_per_step": int(p2.directional_ldscores.nbytes),
                "ms_per_step": round(e2e_s * 1e3, 1)},
        "gpu_launches": launches,
        "clocks": clk.summary(),
    }
    if not os.environ.get("LDS_SKIP_CPU_BASELINE"):
        line["cpu_baseline"] = generalized_cpu_sample(bed, n, basis, fixed, annot, spec, families)
    sess.close()
    print(json.dumps(line), flush=True)


def generalized_cpu_sample(bed, n, basis, fixed, annot, spec, families) -> dict:
    """The oracle's dense FP64 restatement of both passes (NumPy / OpenBLAS,
    all host threads) on the first S SNPs of the workload, as a genome of S
    SNPs: decode excluded, products, projection and scores timed."""
    from oracle import generalized_oracle as go
    from oracle.oracle import Oracle
    from summit_b200 import generalized_gxe as gg

    s = env_int("LDS_GEN_CPU_SNPS", 2000)
    X, _m, _i = Oracle().standardize(bed[:s], n, 0, s)
    a = annot[:s]
    t0 = time.perf_counter()
    z = go.global_probes(spec.root_seed, range(s), range(spec.probe_offset,
                                                         spec.probe_offset + spec.probe_count),
                         spec.namespace)
    probe_s = time.perf_counter() - t0
    t0 = time.perf_counter()
    base = go.source_product(X, 0, s, a, z)                   # N x K*B
    k_count, b_count, q_count = a.shape[1], spec.probe_count, basis.shape[1]
    src = base.T.reshape(k_count, b_count, n).transpose(0, 2, 1)
    rhs = np.empty((n, k_count * b_count * families), order="F")
    fam = [(t, u) for t in range(q_count) for u in range(q_count)]
    for k in range(k_count):
        for q in range(q_count):
            w = basis[:, q, None] * src[k]
            ctx = w - fixed @ (fixed.T @ w)
            for f, (t, u) in enumerate(fam):
                if u == q:
                    rhs[:, (np.arange(b_count) + k * b_count) * families + f] = basis[:, t, None] * ctx
    pairs = gg.pair_order(q_count)
    index = {pr: f for f, pr in enumerate(fam)}
    off, f1, f2 = [0], [], []
    for tp in pairs:
        for sp in pairs:
            for tl, tr in ((tp[0], tp[0]),) if tp[0] == tp[1] else ((tp[0], tp[1]), (tp[1], tp[0])):
                for sl, sr in ((sp[0], sp[0]),) if sp[0] == sp[1] else ((sp[0], sp[1]), (sp[1], sp[0])):
                    f1.append(index[(tr, sl)])
                    f2.append(index[(tl, sr)])
            off.append(len(f1))
    go.pass2_scores(X, rhs, k_count, b_count, families, len(pairs), off, f1, f2,
                    float(n - fixed.shape[1]), a)
    sec = time.perf_counter() - t0
    ops = gen_ops(n, a, b_count, families)
    return {"value": round(ops / sec / 1e12, 6), "unit": "TOPS", "cores": cpu_threads(),
            "kind": "port", "sample": f"first {s} SNPs as a genome of {s} SNPs (N={n}); "
                                      f"oracle/generalized_oracle.py dense FP64 products and "
                                      f"scores, {sec:.1f} s (probe stream {probe_s:.1f} s, "
                                      f"decode excluded)"}


# ---------------------------------------------------------------------------
# Biobank-scale workload (config-5 shape): N = 400,000 x M = 800,000 (80 GB of
# packed codes, resident in HBM, generated on the device), B = 50 +-1 probes.
# One step = one plain genome-wide estimate (K = 1); the GxE reference build
# with E = 4 continuous exposures (B = 50 +-1 probes) is timed beside it.
# ---------------------------------------------------------------------------
BIO_N, BIO_M, BIO_B, BIO_E = 400_000, 800_000, 50, 4
BIO_METRIC = "geno x probe TOPS (biobank-scale genome-wide LD scores, HBM-resident BED)"


def biobank_learned(sess, m: int, stream=None) -> dict:
    """Learned control variate at B = 8 on the biobank image (one window: the
    genome-wide estimator with the near-field control variate and the network
    far field) against the plain estimator at B = 8 and 50, all measured against the
    plain estimator at B = 1,000 (an exact Gram of 800k SNPs is out of reach;
    that estimate's own per-SNP noise is about sqrt(8/1000) of plain B = 8's)."""
    import math

    import torch

    from summit_b200.learned_cv import CvConfig, LearnedCV
    from summit_b200.session import WinPlan

    annot = np.ones((m, 1))
    ws = np.array([0, m], dtype=np.int64)

    def plain(B, seed=PROBE_SEED):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        p = WinPlan(sess, annot, ws, B, BLOCK, seed, "rademacher")
        p.execute()
        ld = p.results(meansq=False)["ldscore"]
        wall = time.perf_counter() - t0
        p.execute()
        dev = float(sum(p.kernel_ms().values()))
        p.close()
        return ld, {"B": B, "wall_ms": round(wall * 1e3, 1), "device_ms": round(dev, 2)}

    # the B = 1,000 estimate draws its own probes (a shared seed would make its first
    # probes those of the plain runs and understate their error)
    hi_est, rj = plain(1000, seed=PROBE_SEED + 7)
    out = {"plain_b1000": rj}
    for B in (8, 50):
        ld, rec = plain(B)
        out[f"plain_b{B}"] = dict(rec, **ld_errors(ld, hi_est))
    cfg = CvConfig(nvecs=8)
    warm = LearnedCV(sess, annot, ws, BLOCK, PROBE_SEED + 2, cfg=cfg)
    warm.run()
    warm.close()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    cv = LearnedCV(sess, annot, ws, BLOCK, PROBE_SEED + 1, cfg=cfg)
    res = cv.run()
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    res = cv.run()
    cv.close()
    ld = res["ldscore"].double().cpu().numpy()
    out["learned_b8"] = {"B": 8, "wall_ms": round(wall * 1e3, 1),
                         "device_ms": round(res["timings"]["total_ms"], 2),
                         "stages_ms": {k: round(v, 2) for k, v in res["timings"].items()},
                         **ld_errors(ld, hi_est),
                         "near_field_only": ld_errors(res["nearcv_ldscore"].double().cpu().numpy(),
                                                      hi_est)}
    # plain probes for the learned per-SNP error (error ~ B^-1/2), from B = 50
    ratio = out["plain_b50"]["snp_rel_rmse"] / max(out["learned_b8"]["snp_rel_rmse"], 1e-12)
    b_eq = int(math.ceil(50.0 * ratio * ratio / 10.0) * 10)
    out["plain_B_for_learned_snp_error"] = b_eq
    # The B = 1,000 estimate's own per-SNP noise inflates every error: with
    # plain variance c/B, plain B=8 measures c/8 + c/1000 against it, so c
    # follows, and the learned estimator's variance net of that noise gives the
    # plain probe count that matches it without that bias.
    c = out["plain_b8"]["snp_rel_rmse"] ** 2 / (1.0 / 8 + 1.0 / 1000)
    net = out["learned_b8"]["snp_rel_rmse"] ** 2 - c / 1000
    out["plain_b1000_noise_snp_rel_rmse"] = round(math.sqrt(c / 1000), 5)
    out["plain_B_for_learned_snp_error_net_of_noise"] = (int(round(c / net)) if net > 0 else None)
    if b_eq <= 1000:
        ld, rec = plain(b_eq)
        out["plain_matched"] = dict(rec, **ld_errors(ld, hi_est))
        out["speedup_at_matched_snp_error"] = {
            "wall": round(out["plain_matched"]["wall_ms"] / out["learned_b8"]["wall_ms"], 2),
            "device": round(out["plain_matched"]["device_ms"] / out["learned_b8"]["device_ms"], 2)}
    out["error_metric"] = ("vs plain B=1000: mean_ld_rel_err = |mean est - mean B1000| / "
                           "|mean B1000|; snp_rel_rmse = per-SNP RMS difference / RMS B1000")
    return out


def biobank_arm(args) -> None:
    import torch

    torch.cuda.set_device(env_int("LOCAL_RANK", 0))
    from summit_b200 import _lib
    from summit_b200.gxe import GxeReference, synthetic_design
    from summit_b200.session import GwSession

    n, m = env_int("LDS_BIO_N", BIO_N), env_int("LDS_BIO_M", BIO_M)
    B, E = BIO_B, BIO_E
    lib = _lib.load()
    t0 = time.perf_counter()
    sess = GwSession.synthetic(n, m, DATA_SEED)
    torch.cuda.synchronize()
    gen_s = time.perf_counter() - t0
    image_bytes = m * (-(-n // 256) * 256) // 4
    annot = np.ones((m, 1))
    plan = sess.plan(annot, B, BLOCK, PROBE_SEED, "rademacher")
    for _ in range(args.warmup):
        plan.execute()
    torch.cuda.synchronize()
    plan.kernel_ms()
    stream_ms = []
    launches0 = lib.lds_kernel_launches()
    with Clocks(env_int("LOCAL_RANK", 0)) as clk:
        for _ in range(args.steps):
            plan.execute()
            km = plan.kernel_ms()
            stream_ms.append(km)
    launches = int(lib.lds_kernel_launches() - launches0) // max(args.steps, 1)
    res = plan.results()
    assert np.isfinite(res["ldscore"]).all()
    p1 = float(np.mean([k["phase1"] for k in stream_ms]))
    p2 = float(np.mean([k["phase2"] for k in stream_ms]))
    ms = float(np.mean([sum(k.values()) for k in stream_ms]))
    ops = 4.0 * n * m * B  # 2 N M B (phase 1, K = 1) + 2 N M B (phase 2)
    plan.close()
    # GxE reference build on the same image: E continuous exposures, +-1 probes
    d = synthetic_design(n, E, seed=3, categorical=0)
    dev = torch.device("cuda")
    g = torch.Generator(device=dev)
    g.manual_seed(4321)
    probes = (torch.randint(0, 2, (B, m), generator=g, device=dev).double() * 2.0 - 1.0).T
    ones1 = torch.ones((1, m), dtype=torch.float64, device=dev).T
    scale = torch.ones((E, m), dtype=torch.float64, device=dev).T
    keys = ("environments", "feature_basis", "power_indices", "power_offsets", "ranks",
            "gram_values", "gram_offsets", "e2_gram_values", "common_basis", "directions")
    gx = GxeReference(sess, *[d[k] for k in keys], annotation_bins=1)
    gx.run(probes, ones1, scale, scale)  # warm-up
    gres = gx.run(probes, ones1, scale, scale)
    gxe_ms = gres["timings"]["total"]
    gxe_ops_ = gxe_ops(n, m, E, 1, B)
    del gx
    learned = None
    if not os.environ.get("LDS_SKIP_LEARNED"):
        learned = biobank_learned(sess, m)
    sess.close()
    line = {
        "metric": BIO_METRIC, "value": round(ops / (ms * 1e-3) / 1e12, 3), "unit": "TOPS",
        "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms, 2),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "int8-digit exact products, f64 epilogue",
        "data": "synthetic (seeded HWE/AR(1) generator, image generated on the device)",
        "config": {"workload": "biobank_gw_n400k_m800k_k1_b50_rademacher", "N": n, "M": m, "K": 1,
                   "B": B, "image_gb": round(image_bytes / 1e9, 2),
                   "l2": "inputs larger than L2 (%.0f GB image)" % (image_bytes / 1e9)},
        "kernel_ms": {"phase1": round(p1, 2), "phase2": round(p2, 2)},
        "decode_stream_gbs": {"phase1": round(image_bytes / (p1 * 1e-3) / 1e9, 1),
                              "phase2": round(image_bytes / (p2 * 1e-3) / 1e9, 1),
                              "note": "packed image bytes streamed per phase / phase time"},
        "image_generation_s": round(gen_s, 2),
        "gxe_reference": {"E": E, "B": B, "columns": E * 2 * B, "ms": round(gxe_ms, 1),
                          "TOPS": round(gxe_ops_ / (gxe_ms * 1e-3) / 1e12, 3),
                          "stage_ms": {k: round(v, 1) for k, v in gres["timings"].items()},
                          "max_leakage": float(np.max(gres["leakages"]))},
        "learned_vs_plain": learned,
        "e2e": None,
        "e2e_note": ("not measured: the 80 GB BED would have to be staged in pinned host "
                     "memory; the image is generated on the device"),
        "gpu_launches": launches, "clocks": clk.summary(),
    }
    if not os.environ.get("LDS_SKIP_CPU_BASELINE"):
        # The reference's per-block native calls (gwldcore.cpp, compiled
        # unchanged) on the leading SNPs of the same data (the generator's
        # first L SNPs do not depend on M).
        from oracle.oracle import Reference
        from summit_b200 import bedfile, gwldcore

        threads = cpu_threads()
        L = env_int("LDS_BIO_CPU_SNPS", 2000)
        ref = Reference()
        ref.set_threads(threads)
        with tempfile.TemporaryDirectory() as td:
            pre = bedfile.write_plink(Path(td) / "bio", packed=gwldcore.synth_bed_rows(n, L, DATA_SEED),
                                      n=n)
            t0 = time.perf_counter()
            ref.gw_ldscore(pre, n, L, np.ones((L, 1)), B, BLOCK, PROBE_SEED, dist="rademacher",
                           impute="mean", dtype=np.float32)
            sec = time.perf_counter() - t0
        line["cpu_baseline"] = {"value": round(4.0 * n * L * B / sec / 1e12, 6), "unit": "TOPS",
                                "cores": threads, "kind": "reference",
                                "sample": f"first {L} SNPs of the workload (N={n}, K=1, B={B}); "
                                          f"reference gwldcore.cpp compiled unchanged, float32, "
                                          f"{sec:.1f} s"}
    print(json.dumps(line), flush=True)


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=["windowed", "gxe", "exact", "biobank", "generalized"],
                    default="windowed")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.workload == "biobank":
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "workload": "biobank",
                              "unavailable": "the biobank workload has no reference arm; "
                                             "the reference arm runs the default workload"}))
            return
        biobank_arm(args)
    elif args.workload == "exact":
        exact_arm(args)
    elif args.workload == "generalized":
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "workload": "generalized",
                              "unavailable": "the generalized workload has no reference arm; "
                                             "its cpu_baseline times the oracle port"}))
            return
        generalized_arm(args)
    elif args.workload == "gxe":
        if args.impl == "reference":
            sec, sample = gxe_reference_sample(GXE_N, env_int("LDS_GXE_CPU_SNPS", 400),
                                               cpu_threads())
            v = gxe_ops(GXE_N, env_int("LDS_GXE_CPU_SNPS", 400), GXE_E, 1, GXE_B) / sec / 1e12
            print(json.dumps({"impl": "reference", "metric": GXE_METRIC, "value": round(v, 6),
                              "unit": "TOPS", "cpu_baseline": {"value": round(v, 6), "unit": "TOPS",
                                                               "cores": cpu_threads(),
                                                               "kind": "reference", "sample": sample}}))
        else:
            gxe_arm(args)
    elif args.impl == "reference":
        reference_arm(args)
    else:
        ours_arm(args)


if __name__ == "__main__":
    main()
