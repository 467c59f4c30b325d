"""SNP shards on liblds (one GPU, shards run one after another in one process).

Each shard is its own genotype image and shard plan; the partial sketches of
phase 1 are summed with torch (the all-reduce of a multi-GPU run), then every
shard runs phase 2 from the summed sketch.  The concatenated estimate must
equal the oracle's unsharded estimate within the int8-digit bound (1e-6
relative, as for the unsharded path), and the sharded driver with one rank
must equal the unsharded plan.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu

LD_RTOL = 1e-6


def _case(n, m, K, seed):
    from oracle.oracle import Oracle

    rows = Oracle().synth_bed_rows(n, m, seed)
    rng = np.random.default_rng(seed)
    annot = np.ones((m, K))
    annot[:, 1] = rng.random(m) < 0.3
    annot[:, 2:] = rng.random((m, K - 2)) * (rng.random((m, K - 2)) < 0.5)
    annot[300:, K - 1] = 0.0  # bin empty in every shard but the first
    return rows, annot


@pytest.mark.parametrize("world,vtile", [(2, None), (3, 64)])
def test_device_shards_match_unsharded(oracle, world, vtile):
    import torch

    from summit_b200.session import GwSession, set_stream
    from summit_b200.sharded import shard_bounds

    n, m, K, step, nvecs, seed = 1000, 2600, 4, 250, 150, 21
    rows, annot = _case(n, m, K, 5)
    want = oracle.gw_ldscore(rows, n, annot, nvecs, step, seed, vtile=vtile, with_mc=True)
    # one non-default stream for the library and torch (torch's default
    # stream has the handle 0, which lds_set_stream reads as "own stream")
    stream = torch.cuda.Stream()
    set_stream(stream.cuda_stream)
    try:
        with torch.cuda.stream(stream):
            sess, plans = [], []
            bounds = shard_bounds(m, world, step)
            for s, e in bounds:
                g = GwSession(rows[s:e], n)
                sess.append(g)
                plans.append(g.shard_plan(annot[s:e], nvecs, step, seed, s, vtile=vtile,
                                          with_mc=True))
            sizes, nrows = plans[0].tiles()
            assert all(p.tiles() == (sizes, nrows) for p in plans)
            assert sum(sizes) == nvecs
            Mk = np.sum([p.bin_totals() for p in plans], axis=0)
            np.testing.assert_allclose(Mk, annot.sum(axis=0), rtol=1e-14)
            for p in plans:
                p.set_bin_totals(Mk)
            for t, V in enumerate(sizes):
                parts = [torch.empty((K * V, nrows), dtype=torch.float64, device="cuda")
                         for _ in plans]
                for p, y in zip(plans, parts):
                    p.phase1(t, y.data_ptr())
                total = torch.stack(parts).sum(0)
                assert torch.isfinite(total).all()
                for p in plans:
                    p.phase2(t, total.data_ptr())
            res = [p.results() for p in plans]
        torch.cuda.synchronize()
    finally:
        set_stream(None)
    ld = np.concatenate([r["ldscore"] for r in res])
    ms = np.concatenate([r["meansq_accum"] for r in res])
    mca = np.sum([r["mc_aggregate_sumsq"] for r in res], axis=0)
    assert rel_err(ms, want["meansq_accum"]) < LD_RTOL
    assert rel_err(ld, want["ldscore"]) < LD_RTOL
    assert rel_err(mca, want["mc_aggregate_sumsq"]) < 10 * LD_RTOL
    for p in plans:
        p.close()
    for g in sess:
        g.close()


def test_single_rank_driver_equals_plan(oracle):
    import torch

    from summit_b200.session import GwSession
    from summit_b200.sharded import DeviceShard, ShardedGw, shard_bounds

    n, m, K, step, nvecs, seed = 700, 1500, 3, 200, 64, 9
    rows, annot = _case(n, m, K, 8)
    eng = DeviceShard(rows, n, 0, annot, nvecs, step, seed)
    try:
        got = ShardedGw(eng, shard_bounds(m, 1, step)).run()
    finally:
        eng.close()
    g = GwSession(rows, n)
    p = g.plan(annot, nvecs, step, seed)
    p.execute()
    want = p.results()
    torch.cuda.synchronize()
    np.testing.assert_array_equal(got.ldscore, want["ldscore"])
    p.close()
    g.close()


def test_shard_offset_must_be_block_aligned():
    from summit_b200.session import GwSession

    rows, annot = _case(300, 500, 3, 4)
    g = GwSession(rows[100:], 300)
    with pytest.raises(RuntimeError, match="block boundary"):
        g.shard_plan(annot[100:], 16, 64, 1, 100)
    g.close()
    h = GwSession(rows[128:], 300, impute_mode="hwe", impute_seed=3)
    with pytest.raises(RuntimeError, match="mean"):
        h.shard_plan(annot[128:], 16, 64, 1, 128)
    h.close()
