"""SNP-sharded genome-wide estimate on CPU ranks (gloo, world size 2 and 3).

The driver (summit_b200.sharded.ShardedGw) runs with an engine that does each
shard's phase 1 / phase 2 on the oracle (FP64 restatement of gwldcore.cpp's
kernels); the test checks that the gathered sharded estimate equals the
oracle's unsharded estimate (gw_ldscore.py's driver restated), i.e. that the
shard bounds, probe-stream keys, sketch all-reduce per V-tile, bin totals and
the gather are right.  The same driver runs on liblds's kernels with NCCL.
"""
from __future__ import annotations

import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from summit_b200.sharded import ShardedGw, shard_bounds


class OracleShard:
    """Oracle engine of one SNP shard (CPU tensors, so gloo reduces them)."""

    device = torch.device("cpu")

    def __init__(self, bed_rows, n, snp_offset, annot, nvecs, step, seed, vtile=None, ddof=1,
                 with_mc=False):
        from oracle.oracle import Oracle, bounded_vtile_sizes, compute_blocks

        self.ora = Oracle()
        self.M = bed_rows.shape[0]
        self.N = n
        self.K = annot.shape[1]
        self.annot = np.ascontiguousarray(annot, dtype=np.float64)
        self.off, self.seed, self.nvecs, self.ddof = snp_offset, seed, nvecs, ddof
        self.blocks = compute_blocks(self.M, step)
        self.std = [self.ora.standardize(bed_rows, n, s, e, None, ddof)[0] for s, e in self.blocks]
        self.inv = np.concatenate([self.ora.inv_resvar(g) for g in self.std])
        self.vt = bounded_vtile_sizes(nvecs, vtile or nvecs)
        self.v0 = np.concatenate([[0], np.cumsum(self.vt)])
        self.Mk = self.annot.sum(axis=0)
        self.meansq = np.zeros((self.M, self.K))
        self.mc_agg = np.zeros(self.K) if with_mc else None
        self.mc_snp = np.zeros((self.M, self.K)) if with_mc else None

    def tile_sizes(self):
        return list(self.vt)

    def new_sketch(self, t):
        return torch.zeros((self.K * self.vt[t], self.N), dtype=torch.float64)

    def phase1(self, t, y):
        Xz = y.numpy().T  # N x K*V, column-major view of the tensor
        init = np.zeros(self.K, dtype=np.uint8)
        V = self.vt[t]
        for (s, e), g in zip(self.blocks, self.std):
            Z = self.ora.probes(self.seed, self.off + s, int(self.v0[t]), e - s, V)
            self.ora.phase1_block(g, self.annot[s:e], self.inv[s:e], Z, Xz, init)
        for k in np.flatnonzero(init == 0):
            Xz[:, k * V:(k + 1) * V] = 0.0

    def phase2(self, t, y):
        Xz = y.numpy().T
        for (s, e), g in zip(self.blocks, self.std):
            self.ora.phase2_block(g, s, self.inv[s:e], self.vt[t], Xz, self.meansq,
                                  self.N - self.ddof + 1, self.mc_agg, self.mc_snp)

    def bin_totals(self):
        return self.Mk.copy()

    def set_bin_totals(self, Mk):
        self.Mk = np.asarray(Mk, dtype=np.float64).copy()

    def results(self):
        ld = self.meansq / float(self.nvecs) - (self.Mk / float(self.N - self.ddof))[None, :]
        return {"ldscore": ld, "meansq_accum": self.meansq, "inv": self.inv,
                "mc_aggregate_sumsq": self.mc_agg, "mc_per_snp_sumsq": self.mc_snp}


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _case(n, m, step, nvecs, vtile, K, seed):
    from oracle.oracle import Oracle

    rows = Oracle().synth_bed_rows(n, m, seed)
    rng = np.random.default_rng(seed)
    annot = (rng.random((m, K)) < 0.3).astype(np.float64)
    annot[:, 0] = 1.0
    # a bin with members only in the first two blocks: empty in later shards
    annot[:, K - 1] = 0.0
    annot[: 2 * step, K - 1] = rng.random(2 * step)
    return rows, annot


def _rank_main(rank, world, port, params, out_dir):
    import torch.distributed as dist

    os.environ["OMP_NUM_THREADS"] = "1"
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world)
    try:
        n, m, step, nvecs, vtile, K, seed = params
        rows, annot = _case(n, m, step, nvecs, vtile, K, seed)
        bounds = shard_bounds(m, world, step)
        s, e = bounds[rank]
        eng = OracleShard(rows[s:e], n, s, annot[s:e], nvecs, step, 77, vtile, with_mc=True)
        res = ShardedGw(eng, bounds).run()
        np.save(os.path.join(out_dir, f"ld_{rank}.npy"), res.ldscore)
        np.save(os.path.join(out_dir, f"mc_{rank}.npy"), res.mc_aggregate_sumsq)
        np.save(os.path.join(out_dir, f"local_{rank}.npy"), res.local["ldscore"])
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,params", [
    (2, (301, 700, 100, 20, None, 3, 11)),   # uneven shards (3 + 4 blocks), one V-tile
    (3, (260, 530, 64, 130, 64, 2, 12)),     # ragged last block, three V-tiles (64, 64, 2)
])
def test_sharded_matches_unsharded(world, params, oracle, tmp_path):
    n, m, step, nvecs, vtile, K, seed = params
    port = _free_port()
    mp.start_processes(_rank_main, args=(world, port, params, str(tmp_path)), nprocs=world,
                       join=True, start_method="spawn")
    rows, annot = _case(*params)
    want = oracle.gw_ldscore(rows, n, annot, nvecs, step, 77, vtile=vtile, with_mc=True)
    bounds = shard_bounds(m, world, step)
    for r in range(world):
        got = np.load(tmp_path / f"ld_{r}.npy")
        np.testing.assert_allclose(got, want["ldscore"], rtol=1e-10, atol=1e-12)
        np.testing.assert_allclose(np.load(tmp_path / f"mc_{r}.npy"), want["mc_aggregate_sumsq"],
                                   rtol=1e-10)
        s, e = bounds[r]
        np.testing.assert_allclose(np.load(tmp_path / f"local_{r}.npy"), want["ldscore"][s:e],
                                   rtol=1e-10, atol=1e-12)


def test_shard_bounds():
    assert shard_bounds(700, 2, 100) == [(0, 300), (300, 700)]
    assert shard_bounds(530, 3, 64) == [(0, 192), (192, 384), (384, 530)]
    for M, W, step in [(1, 4, 10), (0, 2, 5), (1000, 8, 7), (999, 3, 1000)]:
        b = shard_bounds(M, W, step)
        assert len(b) == W and b[0][0] == 0 and b[-1][1] == M
        assert all(x[1] == y[0] for x, y in zip(b, b[1:]))
        assert all(s % step == 0 or s == M for s, _ in b)
    with pytest.raises(ValueError):
        shard_bounds(10, 0, 5)


def test_driver_rejects_mismatched_shard(oracle):
    rows, annot = _case(101, 200, 50, 4, None, 2, 5)
    eng = OracleShard(rows[:100], 101, 0, annot[:100], 4, 50, 1)
    with pytest.raises(ValueError):
        ShardedGw(eng, [(0, 200)]).run()  # one rank must hold the whole range
