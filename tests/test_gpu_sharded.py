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


def test_gxe_device_shards_match_unsharded_build(oracle):
    """SNP-sharded GxE build on liblds (two shards run one after another on
    one GPU; source panels summed with torch, the all-reduce of a multi-GPU
    run), against the unsharded GxeReference build on the whole image, and
    the one-rank ShardedGxe driver against the same build."""
    import torch

    from oracle.gxe_oracle import design, rademacher_block
    from summit_b200.gxe import GxeReference
    from summit_b200.session import GwSession, set_stream
    from summit_b200.sharded import DeviceGxeShard, ShardedGxe, shard_bounds

    n, m, E, K, B, T, step = 600, 900, 3, 1, 8, 3, 128
    rows = oracle.synth_bed_rows(n, m, 13)
    d = design(n, E, seed=2, categorical=1)
    rng = np.random.default_rng(3)
    probes = rademacher_block(9, 0, m, range(B))
    ann = rng.random((m, K)) + 0.05
    sx = 0.5 + rng.random((m, T))
    sw = 0.5 + rng.random((m, T))
    names = ("accum_xx", "accum_xw", "accum_wx", "accum_ww")

    def cm(a):
        return torch.from_numpy(np.ascontiguousarray(a.T)).cuda().T

    g = GwSession(rows, n)
    ref = GxeReference(g, d["environments"], d["feature_basis"], d["power_indices"],
                       d["power_offsets"], d["ranks"], d["gram_values"], d["gram_offsets"],
                       d["e2_gram_values"], d["common_basis"], d["directions"], K)
    want = ref.run(cm(probes), cm(ann), cm(sx), cm(sw), 0)
    want = {k: want[k].cpu().numpy() for k in names}
    ref.close()
    g.close()

    # one rank: the driver equals the unsharded build
    eng = DeviceGxeShard(rows, n, d, K)
    try:
        one = ShardedGxe(eng, shard_bounds(m, 1, step)).run(probes, ann, sx, sw, 0)
    finally:
        eng.close()
    for k in names:
        np.testing.assert_allclose(one.accums[k], want[k], rtol=1e-12, atol=0, err_msg=k)

    # two shards on one device
    bounds = shard_bounds(m, 2, step)
    engines = [DeviceGxeShard(rows[s:e], n, d, K) for s, e in bounds]
    stream = torch.cuda.Stream()
    set_stream(stream.cuda_stream)
    try:
        with torch.cuda.stream(stream):
            cols = T * 2 * K * B
            panels = []
            for eng_, (s, e) in zip(engines, bounds):
                p = eng_.new_panel(cols)
                eng_.source(p, probes[s:e], ann[s:e], sx[s:e], sw[s:e], 0)
                panels.append(p)
            total = torch.stack(panels).sum(0)
            parts = []
            for eng_ in engines:
                p = total.clone()
                assert eng_.project(p, K * B, 0).max() < 1e-9
                parts.append(eng_.target(p, 0, B).reshape(4, E, eng_.M, K))
            full = (torch.cat(parts, dim=2).reshape(4, -1, K) / float(B)).cpu().numpy()
        torch.cuda.synchronize()
    finally:
        set_stream(None)
        for eng_ in engines:
            eng_.close()
    for i, k in enumerate(names):
        assert rel_err(full[i], want[k]) < 1e-6, k
