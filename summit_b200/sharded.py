"""SNP-sharded genome-wide LD scores: one process per GPU, one SNP shard each.

The reference runs the estimator in one process: phase 1 sums the sketch
Xz = sum over SNP blocks of X_blk W_blk (gw_ldscore.py:1934-2019, kernel
gwldcore.cpp:1582-1894), then phase 2 scores every SNP against the finished
sketch (gw_ldscore.py:2060-2160, kernel gwldcore.cpp:2329-2600).  Phase 1 is a
sum over blocks, so the SNPs split into contiguous shards on block boundaries:
rank r holds only its shard's genotype image, computes the partial sketch of
its SNPs, the ranks sum the partial sketches (one all-reduce per V-tile), and
phase 2 then runs independently per shard.  Each block keeps its probe stream
(keyed by the block's start in the fileset), so the sharded estimate is the
unsharded one up to the order of the final FP64 sums.  The annotation totals
M_k of the finalize and the Monte-Carlo aggregate sums are all-reduced too.

``ShardedGw.run`` is the driver; the shard's work comes from an engine:
``DeviceShard`` runs it on liblds's kernels (sketch buffers in device memory;
the library and torch share one created stream, so the NCCL all-reduce is
ordered after phase 1 and before phase 2).
"""
from __future__ import annotations

import contextlib
from dataclasses import dataclass

import numpy as np


def shard_bounds(M: int, world: int, step: int) -> list[tuple[int, int]]:
    """Contiguous SNP shards [start, stop) for `world` ranks, on multiples of
    `step` (the SNP-block size), with block counts differing by at most one."""
    if M < 0 or world <= 0 or step <= 0:
        raise ValueError("shard_bounds needs M >= 0, world > 0 and step > 0")
    nblk = -(-M // step)
    out = []
    for r in range(world):
        b0, b1 = r * nblk // world, (r + 1) * nblk // world
        out.append((min(M, b0 * step), min(M, b1 * step)))
    return out


class DeviceShard:
    """One rank's SNP shard on liblds: a resident genotype image of the shard's
    BED rows and a shard plan (probe streams keyed by the fileset position)."""

    def __init__(self, bed_rows: np.ndarray, n_total: int, snp_offset: int, annot, nvecs: int,
                 step_size: int, seed: int, rand_dist: str = "rademacher",
                 vtile: int | None = None, eps: float = 1e-10, as_float: bool = False,
                 with_mc: bool = False, ddof: int = 1, row_sel=None):
        import torch

        from .session import GwSession, set_stream

        self.torch = torch
        self.device = torch.device("cuda", torch.cuda.current_device())
        # A stream of its own shared by the library and torch (and so the NCCL
        # all-reduce): torch's default stream has the handle 0, which the
        # library reads as "use your own stream".
        self.stream = torch.cuda.Stream()
        set_stream(self.stream.cuda_stream)
        self.session = GwSession(bed_rows, n_total, "mean", 0, ddof, row_sel)
        self.plan = self.session.shard_plan(annot, nvecs, step_size, seed, snp_offset, rand_dist,
                                            vtile, eps, as_float, with_mc)
        self.K = self.plan.K
        self.M = self.session.M
        self.N = self.session.N
        self.ddof = ddof
        self._sizes, self._rows = self.plan.tiles()

    def context(self):
        """Run torch work (sketch buffers, collectives) on the library's stream."""
        return self.torch.cuda.stream(self.stream)

    def tile_sizes(self) -> list[int]:
        return list(self._sizes)

    def new_sketch(self, tile: int):
        # N_pad x K*V column-major == a contiguous (K*V, N_pad) tensor
        return self.torch.empty((self.K * self._sizes[tile], self._rows), dtype=self.torch.float64,
                                device=self.device)

    def phase1(self, tile: int, sketch) -> None:
        self.plan.phase1(tile, sketch.data_ptr())

    def phase2(self, tile: int, sketch) -> None:
        self.plan.phase2(tile, sketch.data_ptr())

    def bin_totals(self) -> np.ndarray:
        return self.plan.bin_totals()

    def set_bin_totals(self, Mk) -> None:
        self.plan.set_bin_totals(Mk)

    def results(self) -> dict:
        return self.plan.results()

    def close(self) -> None:
        from .session import set_stream

        self.plan.close()
        self.session.close()
        set_stream(None)


@dataclass
class ShardedResult:
    bounds: list          # (start, stop) of every rank's shard
    local: dict           # this rank's rows: ldscore, meansq_accum, inv, mc_per_snp_sumsq
    ldscore: np.ndarray | None          # all SNPs (M x K), when gathered
    mc_aggregate_sumsq: np.ndarray | None


class ShardedGw:
    """Driver of the sharded estimate.  `group` is a torch.distributed process
    group (None: the default group; a run without torch.distributed is one
    shard)."""

    def __init__(self, engine, bounds: list[tuple[int, int]], group=None):
        self.engine = engine
        self.bounds = [tuple(map(int, b)) for b in bounds]
        self.group = group

    def _dist(self):
        import torch.distributed as dist

        if dist.is_available() and dist.is_initialized():
            return dist
        return None

    def _allreduce_np(self, x: np.ndarray) -> np.ndarray:
        dist = self._dist()
        if dist is None:
            return x
        import torch

        t = torch.from_numpy(np.ascontiguousarray(x, dtype=np.float64)).to(self.engine.device)
        dist.all_reduce(t, group=self.group)
        return t.cpu().numpy()

    def run(self, gather: bool = True) -> ShardedResult:
        dist = self._dist()
        world = 1 if dist is None else dist.get_world_size(self.group)
        rank = 0 if dist is None else dist.get_rank(self.group)
        if len(self.bounds) != world:
            raise ValueError(f"{len(self.bounds)} shard bounds for {world} ranks")
        b0, b1 = self.bounds[rank]
        if b1 - b0 != self.engine.M:
            raise ValueError(f"rank {rank} holds {self.engine.M} SNPs, its shard is [{b0}, {b1})")
        eng = self.engine
        ctx = eng.context() if hasattr(eng, "context") else contextlib.nullcontext()
        with ctx:
            # every rank takes the same collective steps in the same order
            eng.set_bin_totals(self._allreduce_np(eng.bin_totals()))
            for t in range(len(eng.tile_sizes())):
                y = eng.new_sketch(t)
                eng.phase1(t, y)
                if dist is not None and world > 1:
                    dist.all_reduce(y, group=self.group)
                eng.phase2(t, y)
            loc = eng.results()
        mca = loc.get("mc_aggregate_sumsq")
        if mca is not None:
            mca = self._allreduce_np(mca)
        ld = None
        if gather:
            ld = loc["ldscore"]
            if dist is not None and world > 1:
                import torch

                mmax = max(e - s for s, e in self.bounds)
                K = ld.shape[1]
                buf = torch.zeros((mmax, K), dtype=torch.float64, device=eng.device)
                buf[: ld.shape[0]] = torch.from_numpy(ld).to(eng.device)
                parts = [torch.empty_like(buf) for _ in range(world)]
                dist.all_gather(parts, buf, group=self.group)
                ld = np.concatenate([parts[r][: e - s].cpu().numpy()
                                     for r, (s, e) in enumerate(self.bounds)])
        return ShardedResult(self.bounds, loc, ld, mca)


# ---------------------------------------------------------------------------
# SNP-sharded SUMMIT-GxE reference (generate_multi_environment_references,
# gxe_multi.py:6509).  The source panel is a sum over SNP blocks
# (MultiEnvironmentKernel.source_block, gxeldcore.cpp:11008-11240), so rank r
# adds its shard's contribution, the ranks sum the panels (one all-reduce),
# and every rank then projects the same summed panel (project_sources,
# :11583-11729; deterministic, so identical on all ranks), seals the
# [S, phi o S] pair and scores its own SNPs (target_score_block,
# :11731-11936).  The four accumulators ((E M_r) x K per rank) are gathered
# into the (E M) x K layout of the unsharded build and divided by the probe
# count (normalize_scores, :12490-12557).
# ---------------------------------------------------------------------------
class DeviceGxeShard:
    """One rank's GxE shard on liblds: a resident genotype image of the
    shard's BED rows and the kernel's context on it; panels are torch CUDA
    tensors on one stream shared by the library and torch (so the NCCL
    all-reduce is ordered between source and projection)."""

    def __init__(self, bed_rows: np.ndarray, n_total: int, design: dict, annotation_bins: int = 1,
                 ddof: int = 1):
        import torch

        from .gxe import GxeReference
        from .session import GwSession, set_stream

        self.torch = torch
        self.device = torch.device("cuda", torch.cuda.current_device())
        self.stream = torch.cuda.Stream()
        set_stream(self.stream.cuda_stream)
        self.session = GwSession(bed_rows, n_total, "mean", 0, ddof)
        d = design
        self.ref = GxeReference(self.session, d["environments"], d["feature_basis"],
                                d["power_indices"], d["power_offsets"], d["ranks"],
                                d["gram_values"], d["gram_offsets"], d["e2_gram_values"],
                                d["common_basis"], d["directions"], annotation_bins, ddof)
        self.M, self.N, self.E, self.K = self.session.M, self.session.N, self.ref.E, self.ref.K
        self._env = np.asfortranarray(d["environments"], dtype=np.float64)

    def context(self):
        return self.torch.cuda.stream(self.stream)

    def _cm(self, a):
        """Host (rows x cols) array -> device tensor with column-major storage."""
        return self.torch.from_numpy(np.ascontiguousarray(np.asarray(a, np.float64).T)).to(
            self.device).T

    def new_panel(self, cols: int):
        return self.torch.zeros((cols, self.N), dtype=self.torch.float64, device=self.device)

    def source(self, panel, probes, annotation, scale_x, scale_w, env_start: int) -> None:
        from . import _lib
        from ._lib import check
        from .gxe import _dp

        self._in = [self._cm(x) for x in (probes, annotation, scale_x, scale_w)]
        z, a, sx, sw = self._in
        T, B = sx.shape[1], z.shape[1]
        check(_lib.load().lds_gxe_source_block(self.ref.h, 0, self.M, _dp(z), B, _dp(a), 0,
                                               _dp(sx), _dp(sw), T, env_start, _dp(panel), 1))

    def project(self, panel, cols_per_env: int, env_start: int) -> np.ndarray:
        import ctypes as C

        from . import _lib
        from ._lib import check
        from .gxe import _dp

        T = panel.shape[0] // (2 * cols_per_env)
        leak = np.zeros(T)
        check(_lib.load().lds_gxe_project_sources(self.ref.h, _dp(panel), panel.shape[0],
                                                  cols_per_env, env_start,
                                                  leak.ctypes.data_as(C.c_void_p), 1))
        return leak

    def target(self, panel, env_start: int, probe_count: int):
        import ctypes as C

        from . import _lib
        from ._lib import check
        from .gxe import _dp

        lib = _lib.load()
        z, a, sx, sw = self._in
        T = sx.shape[1]
        w = self.torch.from_numpy(self._env[:, env_start:env_start + T].T.copy()).to(self.device)
        pair = C.c_int64(0)
        check(lib.lds_gxe_pair_create(self.ref.h, _dp(panel), panel.shape[0], _dp(w), T, 1,
                                      C.byref(pair)))
        accs = self.torch.zeros((4, self.E * self.M, self.K), dtype=self.torch.float64,
                                device=self.device)
        try:
            check(lib.lds_gxe_target_score_block(
                self.ref.h, 0, self.M, pair.value, _dp(sx), _dp(sw), T, _dp(accs[0]),
                _dp(accs[1]), _dp(accs[2]), _dp(accs[3]), 0, self.M, probe_count, env_start, 1))
        finally:
            lib.lds_gxe_pair_destroy(pair.value)
        return accs

    def close(self) -> None:
        from .session import set_stream

        self.ref.close()
        self.session.close()
        set_stream(None)


@dataclass
class ShardedGxeResult:
    bounds: list
    accums: dict | None        # accum_xx, accum_xw, accum_wx, accum_ww: (E M) x K, normalized
    local: dict                # this rank's unnormalized (E M_r) x K accumulators
    leakages: np.ndarray


class ShardedGxe:
    """Driver of the SNP-sharded GxE build; `engine` is this rank's shard
    (DeviceGxeShard, or any object with the same methods)."""

    def __init__(self, engine, bounds: list[tuple[int, int]], group=None):
        self.engine = engine
        self.bounds = [tuple(map(int, b)) for b in bounds]
        self.group = group

    def run(self, probes, annotation, scale_x, scale_w, environment_start: int = 0,
            gather: bool = True) -> ShardedGxeResult:
        """probes (M_r x B), annotation (M_r x K), scale_x / scale_w (M_r x T):
        this rank's rows of the genome-wide arrays (host numpy)."""
        import torch

        dist = ShardedGw._dist(self)
        world = 1 if dist is None else dist.get_world_size(self.group)
        rank = 0 if dist is None else dist.get_rank(self.group)
        if len(self.bounds) != world:
            raise ValueError(f"{len(self.bounds)} shard bounds for {world} ranks")
        b0, b1 = self.bounds[rank]
        eng = self.engine
        if b1 - b0 != eng.M or np.asarray(probes).shape[0] != eng.M:
            raise ValueError(f"rank {rank} holds {eng.M} SNPs, its shard is [{b0}, {b1})")
        B, K, T = np.asarray(probes).shape[1], eng.K, np.asarray(scale_x).shape[1]
        cols = T * 2 * K * B
        ctx = eng.context() if hasattr(eng, "context") else contextlib.nullcontext()
        with ctx:
            panel = eng.new_panel(cols)
            eng.source(panel, probes, annotation, scale_x, scale_w, environment_start)
            if dist is not None and world > 1:
                dist.all_reduce(panel, group=self.group)
            leak = eng.project(panel, K * B, environment_start)
            accs = eng.target(panel, environment_start, B)  # (4, E M_r, K), unnormalized
            local = {n: accs[i] for i, n in enumerate(("accum_xx", "accum_xw", "accum_wx",
                                                       "accum_ww"))}
            out = None
            if gather:
                E = eng.E
                parts = [accs]
                if dist is not None and world > 1:
                    mmax = max(e - s for s, e in self.bounds)
                    buf = torch.zeros((4, E, mmax, K), dtype=torch.float64, device=eng.device)
                    buf[:, :, : eng.M] = accs.reshape(4, E, eng.M, K)
                    parts = [torch.empty_like(buf) for _ in range(world)]
                    dist.all_gather(parts, buf, group=self.group)
                    parts = [p[:, :, : e - s] for p, (s, e) in zip(parts, self.bounds)]
                else:
                    parts = [accs.reshape(4, E, eng.M, K)]
                full = torch.cat(parts, dim=2).reshape(4, -1, K) / float(B)
                out = {n: full[i].cpu().numpy() for i, n in
                       enumerate(("accum_xx", "accum_xw", "accum_wx", "accum_ww"))}
        return ShardedGxeResult(self.bounds, out, local, leak)
