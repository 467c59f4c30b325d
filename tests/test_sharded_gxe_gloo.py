"""SNP-sharded SUMMIT-GxE reference build on CPU ranks (gloo, world size 2
and 3).  Each rank's engine runs its shard's source, projection and target on
the oracle (FP64 restatement of gxeldcore.cpp's MultiEnvironmentKernel);
the driver (summit_b200.sharded.ShardedGxe) all-reduces the source panel and
gathers the accumulators.  The gathered result must equal the unsharded
oracle build, i.e. the shard bounds, the panel all-reduce, the per-shard
target rows and the gather are right.  The same driver runs on liblds's
kernels with NCCL (DeviceGxeShard)."""
from __future__ import annotations

import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from summit_b200.sharded import ShardedGxe, shard_bounds


class OracleGxeShard:
    device = torch.device("cpu")

    def __init__(self, X, d, K):
        from oracle import gxe_oracle as G

        self.G, self.X, self.d, self.K = G, X, d, K
        self.N, self.M = X.shape
        self.E = d["environments"].shape[1]

    def new_panel(self, cols):
        return torch.zeros((cols, self.N), dtype=torch.float64)

    def source(self, panel, probes, annotation, sx, sw, env_start):
        self._sx, self._sw = sx, sw
        self.G.source_block(panel.numpy().T, self.X, probes, annotation, sx, sw,
                            self.d["environments"], env_start)

    def project(self, panel, cpe, env_start):
        d = self.d
        return self.G.project_sources(panel.numpy().T, cpe, env_start, d["common_basis"],
                                      d["directions"], d["fixed_bases"])

    def target(self, panel, env_start, B):
        T = self._sx.shape[1]
        w = self.d["environments"][:, env_start:env_start + T]
        pair = self.G.row_weighted_pair(panel.numpy().T, w)
        accs = [np.zeros((self.E * self.M, self.K)) for _ in range(4)]
        self.G.target_score_block(self.X, pair, self._sx, self._sw, accs, 0, self.M, B, env_start,
                                  self.d["ranks"], self.K)
        return torch.from_numpy(np.stack(accs))


def _case(n, m, E, K, B, T, seed):
    from oracle import gxe_oracle as G
    from oracle.oracle import Oracle

    ora = Oracle()
    rows = ora.synth_bed_rows(n, m, seed)
    X = ora.standardize(rows, n, 0, m)[0]
    d = G.design(n, E, seed=seed, categorical=1)
    rng = np.random.default_rng(seed)
    probes = G.rademacher_block(5, 0, m, range(B))
    ann = rng.random((m, K)) + 0.05
    sx = 0.5 + rng.random((m, T))
    sw = 0.5 + rng.random((m, T))
    return X, d, probes, ann, sx, sw


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, params, out_dir):
    import torch.distributed as dist

    os.environ["OMP_NUM_THREADS"] = "1"
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world)
    try:
        n, m, E, K, B, T, env_start, step, seed = params
        X, d, probes, ann, sx, sw = _case(n, m, E, K, B, T, seed)
        bounds = shard_bounds(m, world, step)
        s, e = bounds[rank]
        eng = OracleGxeShard(X[:, s:e], d, K)
        res = ShardedGxe(eng, bounds).run(probes[s:e], ann[s:e], sx[s:e], sw[s:e], env_start)
        for name, a in res.accums.items():
            np.save(os.path.join(out_dir, f"{name}_{rank}.npy"), a)
        np.save(os.path.join(out_dir, f"leak_{rank}.npy"), res.leakages)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,params", [
    (2, (211, 150, 3, 1, 4, 3, 0, 32, 3)),   # uneven shards
    (3, (180, 130, 3, 2, 3, 2, 1, 20, 4)),   # environment tile starting at 1, two bins
])
def test_sharded_gxe_matches_unsharded(world, params, tmp_path):
    from oracle import gxe_oracle as G

    n, m, E, K, B, T, env_start, step, seed = params
    mp.start_processes(_rank_main, args=(world, _free_port(), params, str(tmp_path)),
                       nprocs=world, join=True, start_method="spawn")
    X, d, probes, ann, sx, sw = _case(n, m, E, K, B, T, seed)
    cols = T * 2 * K * B
    panel = np.zeros((n, cols), order="F")
    G.source_block(panel, X, probes, ann, sx, sw, d["environments"], env_start)
    leak = G.project_sources(panel, K * B, env_start, d["common_basis"], d["directions"],
                             d["fixed_bases"])
    pair = G.row_weighted_pair(panel, d["environments"][:, env_start:env_start + T])
    accs = [np.zeros((E * m, K)) for _ in range(4)]
    G.target_score_block(X, pair, sx, sw, accs, 0, m, B, env_start, d["ranks"], K)
    G.normalize_scores(accs, B)
    for r in range(world):
        for name, want in zip(("accum_xx", "accum_xw", "accum_wx", "accum_ww"), accs):
            got = np.load(tmp_path / f"{name}_{r}.npy")
            np.testing.assert_allclose(got, want, rtol=1e-10, atol=1e-300, err_msg=name)
        assert np.load(tmp_path / f"leak_{r}.npy").max() < 1e-9
    assert leak.max() < 1e-9
