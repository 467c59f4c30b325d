"""Learned control variate for windowed + partitioned stochastic LD scores.

No counterpart in the reference; it cuts the probes a windowed estimate needs.
The plain estimator of SNP j's score in bin k averages u_jv^2 over V probes,
u_jv = sum_{i in window} c_ji annot_ik z_iv.  Two steps reduce its variance:

1. Exact near field (a control variate with known mean).  a_jv, the part of
   u_jv from the SNPs within ``band`` positions of j (same window), uses the
   same probes; its mean E[a^2] = mu_jk is known exactly from the exact
   neighbour products (lds_nn_band).  a and the far part f are independent, so
   R = mean_v (u^2 - a^2) + mu keeps the mean with the optimal coefficient 1:
   T = R - mu is an unbiased estimate of the far-field score.
2. Learned far field.  A small network (liblds's own kernels: 3 x 128 GELU,
   BF16 weights, FP32 accumulation) is trained on T for a random subset of
   SNPs, from per-SNP features: MAF, the annotations, exact r^2 to the 2*band
   nearest SNPs, the near-field scores mu_j., and the window geometry.  Its
   prediction h is combined with T per bin, mu + h + lambda_k (T - h), where
   lambda_k = b^2 / (b^2 + s^2) is the MSE-optimal weight given the network's
   squared bias b^2 (validation residual minus noise) and the noise s^2 of T,
   itself measured from two independent halves of the probes; adding
   (1 - lambda_k) mean_j (T - h) keeps each bin's mean over SNPs equal to the
   unbiased near-field estimate's.

The plain estimator stays available (``plain_ldscore``) and is the yardstick:
tests and the benchmark compare both against the exact expectation of the
windowed estimator (GwSession.partition_ld_expectation, exact tensor-core Gram
products) and against plain runs with 10x and 100x the probes.
Everything runs on the device; torch only provides memory and elementwise glue.
"""
from __future__ import annotations

import time
from dataclasses import dataclass

import numpy as np

from .session import GwSession, WinPlan
from .surrogate import Surrogate


@dataclass
class CvConfig:
    nvecs: int = 10            # probes of the control-variate run, split in two halves
    band: int = 8              # exact near field |i - j| <= band (4, 8 or 15)
    train_frac: float = 0.1    # SNPs whose noisy far-field scores train the network
    val_frac: float = 0.05     # disjoint SNPs that set the shrinkage weights
    epochs: int = 10
    min_steps: int = 30        # at least this many optimizer steps (small training sets)
    batch: int = 4096
    lr: float = 2e-3
    seed: int = 0


class LearnedCV:
    def __init__(self, session: GwSession, annot, window_starts, step: int, seed: int,
                 rand_dist: str = "rademacher", cfg: CvConfig | None = None,
                 batch_gb: float = 8.0):
        import torch

        self.cfg = cfg = cfg or CvConfig()
        if cfg.nvecs < 2:
            raise ValueError("the control-variate run needs at least 2 probes (two halves)")
        annot = np.ascontiguousarray(annot, dtype=np.float64)
        ws = np.ascontiguousarray(window_starts, dtype=np.int64)
        self.M, self.K = annot.shape
        self.N = session.N
        half = (cfg.nvecs + 1) // 2
        self.plan = WinPlan(session, annot, ws, cfg.nvecs, step, seed, rand_dist,
                            batch_gb=batch_gb)
        self.plan.set_cv(annot, split_tiles=True, band=cfg.band)
        self.tiles = [half, cfg.nvecs - half]  # the two probe halves
        dev = torch.device("cuda")
        M, K, D = self.M, self.K, cfg.band
        W = ws.size - 1
        sizes = np.diff(ws)
        self.annot = self.plan.cv_annot_view()  # the plan's device copy, no second upload
        ws_t = torch.from_numpy(ws).to(dev)
        win = torch.repeat_interleave(torch.arange(W, device=dev), torch.from_numpy(sizes).to(dev))
        # correlation null M_k(window) / (N - ddof), as the plain estimator applies it:
        # the plan's per-window annotation totals (W x K, SNP order), gathered per SNP
        mkw = torch.from_numpy(self.plan.bin_totals()).to(dev)
        nd = float(session.N - 1)
        self.null = mkw[win] / nd
        # static features: MAF, annotations, window geometry
        mean = torch.from_numpy(session.stats()["mean"]).to(dev)
        p = torch.clamp(mean / 2.0, 0.0, 1.0)
        maf = torch.minimum(p, 1.0 - p)
        pos = torch.arange(M, device=dev) - ws_t[win]
        size = ws_t[win + 1] - ws_t[win]
        edge = torch.minimum(pos, size - 1 - pos).double()
        geo = torch.stack([torch.log(size.double()) / np.log(5000.0),
                           edge / torch.clamp(size, min=1).double(),
                           torch.clamp(edge, max=100.0) / 100.0], 1)
        self.static = torch.cat([2.0 * maf[:, None], self.annot, geo], 1).float().contiguous()
        gen = torch.Generator(device=dev)
        gen.manual_seed(cfg.seed)
        perm = torch.randperm(M, generator=gen, device=dev)
        ntr = max(1, int(round(cfg.train_frac * M)))
        nva = max(1, int(round(cfg.val_frac * M)))
        self.train_rows = torch.sort(perm[:ntr]).values
        self.val_rows = torch.sort(perm[ntr:ntr + nva]).values
        T = 2
        f64 = dict(dtype=torch.float64, device=dev)
        self.meansq = torch.empty((T, M, K), **f64)
        self.C = torch.empty((T, M, K), **f64)
        self.mu = torch.empty((M, K), **f64)
        self.xx = torch.empty((M, D + 1), **f64)
        self.n_features = self.static.shape[1] + 2 * D + K
        self.timings = {}

    def _neighbour_r2(self):
        """r^2 to the band nearest SNPs on each side (0 past the ends)."""
        import torch

        xx, D, M = self.xx, self.cfg.band, self.M
        self_ss = xx[:, 0].clamp_min(1e-300)
        cols = []
        for d in range(1, D + 1):  # right neighbours j + d
            r = torch.zeros(M, dtype=torch.float64, device=xx.device)
            r[: M - d] = xx[: M - d, d] ** 2 / (self_ss[: M - d] * self_ss[d:])
            cols.append(r)
        for d in range(1, D + 1):  # left neighbours j - d: stored at row j - d
            r = torch.zeros(M, dtype=torch.float64, device=xx.device)
            r[d:] = xx[: M - d, d] ** 2 / (self_ss[: M - d] * self_ss[d:])
            cols.append(r)
        return torch.stack(cols, 1)

    def run(self) -> dict:
        import torch

        cfg, M, K = self.cfg, self.M, self.K
        B = float(sum(self.tiles))
        V1, V2 = (float(v) for v in self.tiles)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        self.plan.execute()
        self.plan.cv_outputs_device(self.meansq.data_ptr(), self.C.data_ptr(), self.mu.data_ptr(),
                                    self.xx.data_ptr())
        t1 = time.perf_counter()
        E1 = (self.meansq[0] - self.C[0]) / V1 + self.mu
        E2 = (self.meansq[1] - self.C[1]) / V2 + self.mu
        R = ((self.meansq[0] - self.C[0]) + (self.meansq[1] - self.C[1])) / B + self.mu
        noise = (E1 - E2) ** 2 * (V1 * V2) / (B * B)       # Var(R) per (SNP, bin)
        target = (R - self.mu).float()                      # far-field score (noisy)
        feats = torch.cat([self.static, self._neighbour_r2().float(), self.mu.float()], 1)
        tr, va = self.train_rows, self.val_rows
        fmean, fstd = feats[tr].mean(0), feats[tr].std(0).clamp_min(1e-6)
        X = ((feats - fmean) / fstd).contiguous()
        tmean, tstd = target[tr].mean(0), target[tr].std(0).clamp_min(1e-12)
        Y = ((target - tmean) / tstd).contiguous()
        net = Surrogate(self.n_features, K, seed=cfg.seed)
        Xtr, Ytr = X[tr].contiguous(), Y[tr].contiguous()
        t2 = time.perf_counter()
        per_epoch = -(-Xtr.shape[0] // cfg.batch)
        epochs = max(cfg.epochs, -(-cfg.min_steps // per_epoch))
        losses = net.train(Xtr, Ytr, epochs=epochs, batch=cfg.batch, lr=cfg.lr, seed=cfg.seed)
        t3 = time.perf_counter()
        h = (net.forward(X).double() * tstd.double() + tmean.double())
        resid2 = ((target.double()[va] - h[va]) ** 2).mean(0)
        nv = noise[va].mean(0)
        bias2 = (resid2 - nv).clamp_min(0.0)
        lam = bias2 / (bias2 + nv).clamp_min(1e-300)
        # Per-SNP shrinkage toward the network, plus (1 - lambda) times the mean
        # residual of each bin: the bin's mean over SNPs then equals the
        # unbiased near-field estimate's, whatever the network's average bias.
        resid = target.double() - h
        est = self.mu + h + lam[None, :] * resid + (1.0 - lam)[None, :] * resid.mean(0, keepdim=True)
        ld = est - self.null
        torch.cuda.synchronize()
        t4 = time.perf_counter()
        plain = (self.meansq[0] + self.meansq[1]) / B - self.null
        self.timings = {"estimate_ms": (t1 - t0) * 1e3, "features_ms": (t2 - t1) * 1e3,
                        "train_ms": (t3 - t2) * 1e3, "combine_ms": (t4 - t3) * 1e3,
                        "total_ms": (t4 - t0) * 1e3}
        return {"ldscore": ld, "plain_ldscore": plain, "nearcv_ldscore": R - self.null,
                "lambda": lam, "train_loss": losses, "timings": dict(self.timings)}

    def close(self) -> None:
        self.plan.close()
