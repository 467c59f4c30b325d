// Phase 2 on SM pairs: tcgen05.mma.cta_group::2 (M = 256) over two 128-SNP
// tiles that share one sketch tile.
//
// Work[j, c] = x_j^T Y[:, c] as in p2_umma_kernel (lds_umma.cu), with a
// cluster of two CTAs per pair of SNP tiles (rank r holds SNP rows
// jt0 + 128 r .. + 127).  Each CTA decodes its own G and O operand tiles;
// the sketch tile of a K-step (N digit columns x 128 samples) is split by
// columns, rank r holding columns [r N/2, (r+1) N/2) in its own shared memory,
// so each SM stores and supplies half of it: per K-step an SM moves about
// 104 KB through shared memory instead of 150 KB, which is what limits the
// one-SM kernel.  Rank 0 issues the MMAs for both SMs; each CTA's TMEM holds
// the accumulators of its own 128 rows (G at column 0, O at column 256), and
// each CTA runs the same LD-score epilogue on them.
//
// Cross-CTA protocol (rank 0 = leader):
//   * sketch halves: each rank's producer copies its half with a cta_group::2
//     TMA that completes its bytes on the LEADER's b_full barrier; only the
//     leader arrives there (with the bytes of both halves);
//   * decoded operand tiles: the decoders of both ranks arrive on the leader's
//     a_full barrier (release at cluster scope after a proxy fence);
//   * the leader's MMA commits arrive on a_empty / b_empty / acc_full of both
//     ranks (one tcgen05.commit addressed to both, mask 0b11);
//   * the epilogue threads of both ranks arrive on the leader's acc_empty.
// Remote barrier addresses come from mapa; every TMA copy lands in the issuing
// CTA's own shared memory.
// Every mbarrier wait is bounded (status code on timeout); both CTAs always
// reach the final cluster barrier, after the leader's MMAs have drained, so
// no CTA exits while its peer can still read its shared memory.
#include <cstdint>
#include <cstdio>
#include <cuda.h>
#include <cuda_runtime.h>

#include "lds_device.cuh"
#include "lds_internal.h"
#include "lds_tc.cuh"
#include "lds_umma.h"

namespace lds {
namespace umma {

namespace pair {
constexpr int kBM = 128;              // SNP rows per CTA (M = 256 per pair)
constexpr int kBK = 128;              // samples per stage
constexpr int kPkBytes = kBM * 32;    // packed tile: 128 rows x 32 bytes
constexpr int kATile = kBM * kBK;     // 16 KB
constexpr int kPkStages = 8;
constexpr int kAStages = 3;
constexpr int kBStages = 6;
constexpr int kDecSets = 2;
constexpr int kThreads = 96 + 128 * kDecSets;
constexpr uint32_t kTmemCols = 512;
constexpr uint32_t kOCol = 256;

struct Layout {
    uint32_t b_slot;  // one sketch half: box_rows/2 rows x 128 bytes, 1 KB multiple
    __host__ __device__ explicit Layout(int box_rows)
        : b_slot((uint32_t)((((box_rows / 2) * kBK) + 1023) / 1024 * 1024)) {}
    __host__ __device__ uint32_t a_off(int s) const { return (uint32_t)s * 2 * kATile; }
    __host__ __device__ uint32_t b_off(int s) const { return kAStages * 2 * kATile + s * b_slot; }
    __host__ __device__ uint32_t pk_off(int s) const {
        return kAStages * 2 * kATile + kBStages * b_slot + s * kPkBytes;
    }
    __host__ __device__ uint32_t bar_off() const { return pk_off(kPkStages); }
    __host__ __device__ uint32_t bytes() const { return bar_off() + 512; }
};

__device__ __forceinline__ uint32_t cluster_rank() {
    uint32_t r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
    return r;
}
// Address of the same shared-memory object in CTA `rank` of the cluster.
__device__ __forceinline__ uint32_t map_to_rank(const void* p, uint32_t rank) {
    uint32_t d;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(d) : "r"(smem_u32(p)), "r"(rank));
    return d;
}
__device__ __forceinline__ void arrive_cluster(uint32_t cluster_addr) {
    asm volatile("mbarrier.arrive.release.cluster.shared::cluster.b64 _, [%0];" ::"r"(cluster_addr)
                 : "memory");
}
// Bounded wait with cluster-scope acquire (arrivals may come from the peer).
__device__ __forceinline__ bool wait_cluster(uint64_t* bar, uint32_t parity) {
    const uint32_t addr = smem_u32(bar);
    const long long limit = wait_limit();
    for (long long i = 0; i < limit; ++i) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.acquire.cluster.shared::cta.b64 p, [%1], %2, %3;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(addr), "r"(parity), "n"(kSuspendNs)
            : "memory");
        if (done) return true;
    }
    return false;
}
__device__ __forceinline__ void umma_i8_pair(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc,
                                             uint32_t idesc, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::2.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate));
}
// Completion of the issuing thread's MMAs arrives on `bar` in both CTAs.
__device__ __forceinline__ void commit_both(uint64_t* bar) {
    const uint16_t mask = 0x3;
    asm volatile(
        "tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.multicast::cluster.b64 "
        "[%0], %1;" ::"r"(smem_u32(bar)),
        "h"(mask)
        : "memory");
}
__device__ __forceinline__ void commit_own(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     smem_u32(bar))
                 : "memory");
}
// Tile copy into this CTA's shared memory whose bytes complete on the
// barrier at `bar_cluster` (the leader's).
__device__ __forceinline__ void tma_load_2d_pair(void* dst, const CUtensorMap* map, int x, int y,
                                                 uint32_t bar_cluster) {
    asm volatile(
        "cp.async.bulk.tensor.2d.cta_group::2.shared::cluster.global.mbarrier::complete_tx::bytes "
        "[%0], [%1, {%2, %3}], [%4];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(bar_cluster)
        : "memory");
}
__device__ __forceinline__ void cluster_sync_all() {
    asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::
                     : "memory");
}
}  // namespace pair

__global__ void __launch_bounds__(pair::kThreads, 1)
    p2_umma_pair_kernel(const __grid_constant__ CUtensorMap tmA,
                        const __grid_constant__ CUtensorMap tmB, P2UArgs a) {
    using namespace pair;
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>(
        (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    const Layout lay(a.box_rows);
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem + lay.bar_off());
    uint64_t* pk_full = bars;                          // [kPkStages] local
    uint64_t* pk_empty = pk_full + kPkStages;          // [kPkStages] local
    uint64_t* a_full = pk_empty + kPkStages;           // [kAStages] leader's: both ranks' decoders
    uint64_t* a_empty = a_full + kAStages;             // [kAStages] both: leader's commits
    uint64_t* b_full = a_empty + kAStages;             // [kBStages] leader's: both halves' bytes
    uint64_t* b_empty = b_full + kBStages;             // [kBStages] both: leader's commits
    uint64_t* acc_full = b_empty + kBStages;           // both: leader's commit
    uint64_t* acc_empty = acc_full + 1;                // leader's: both ranks' epilogues
    uint64_t* mma_done = acc_empty + 1;                // leader: drain of its MMAs
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(mma_done + 1);
    volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const uint32_t rank = cluster_rank();
    const bool leader = rank == 0;
    const int k0 = blockIdx.y * a.bins_per_cta;
    const int nbk = min(a.bins_per_cta, a.K - k0);
    const int cols = a.bins_per_cta * a.ncolp;
    int64_t jt0, jend;
    int sb = 0;
    if (a.tiles) {
        const int4 t = a.tiles[blockIdx.x >> 1];  // one entry per pair
        jt0 = t.x + (int64_t)rank * kBM;
        jend = t.y;
        sb = t.z;
    } else {
        jt0 = a.j0 + (int64_t)blockIdx.x * kBM;
        jend = a.j1;
    }
    const int kb = sb + k0;

    if (tid == 0) {
        for (int s = 0; s < kPkStages; ++s) {
            mbar_init(&pk_full[s], 1);
            mbar_init(&pk_empty[s], 128);
        }
        for (int s = 0; s < kAStages; ++s) {
            mbar_init(&a_full[s], 2 * 128);
            mbar_init(&a_empty[s], 1);
        }
        for (int s = 0; s < kBStages; ++s) {
            mbar_init(&b_full[s], 1);
            mbar_init(&b_empty[s], 1);
        }
        mbar_init(acc_full, 1);
        mbar_init(acc_empty, 2 * 128);
        mbar_init(mma_done, 1);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32(tmem_slot)),
                     "r"(kTmemCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;");
    }
    tc_fence_before();
    __syncthreads();
    cluster_sync_all();  // both CTAs' barriers initialized and TMEM allocated
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;
    const uint32_t a_full_l = map_to_rank(a_full, 0);      // leader's a_full[0]
    const uint32_t b_full_l = map_to_rank(b_full, 0);      // leader's b_full[0]
    const uint32_t acc_empty_l = map_to_rank(acc_empty, 0);

    auto fail = [&](int code) {
        atomicCAS(a.status, 0u, (unsigned)code);
        *abort_flag = 1;
    };

    const int ngroups = a.ngroups;
    const int total = ngroups * a.nkt;
    const int half_rows = a.box_rows / 2;
    if (warp == 0) {
        // ---------------- packed-code producer (own SNP tile) ----------------
        if (lane == 0) {
            for (int it = 0; it < total; ++it) {
                const int s = it % kPkStages;
                if (it >= kPkStages &&
                    !mbar_wait(&pk_empty[s], ((uint32_t)(it / kPkStages) & 1u) ^ 1u)) { fail(21); break; }
                if (*abort_flag) break;
                mbar_expect_tx(&pk_full[s], (uint32_t)kPkBytes);
                tma_load_2d(smem + lay.pk_off(s), &tmA, (it % a.nkt) * 32, (int)jt0, &pk_full[s]);
            }
        }
    } else if (warp == 2) {
        // ---------------- sketch-half producer ----------------
        if (lane == 0) {
            for (int it = 0; it < total; ++it) {
                const int s = it % kBStages;
                if (it >= kBStages &&
                    !mbar_wait(&b_empty[s], ((uint32_t)(it / kBStages) & 1u) ^ 1u)) { fail(22); break; }
                if (*abort_flag) break;
                const int g = it / a.nkt, kt = it % a.nkt;
                const int ncols = min(256, cols - g * 256);
                if (leader) mbar_expect_tx(&b_full[s], (uint32_t)(2 * half_rows * kBK));
                tma_load_2d_pair(smem + lay.b_off(s), &tmB, kt * kBK,
                                 kb * a.ncolp + g * 256 + (int)rank * (ncols / 2),
                                 b_full_l + (uint32_t)(s * 8));
            }
        }
    } else if (warp == 1) {
        // ---------------- MMA issuer (leader only) ----------------
        if (lane == 0 && leader) {
            int it = 0;
            for (int g = 0; g < ngroups && !*abort_flag; ++g) {
                const int ncols = min(256, cols - g * 256);
                const uint32_t idesc = idesc_i8(2 * kBM, ncols);
                if (g > 0 && !wait_cluster(acc_empty, (uint32_t)(g - 1) & 1u)) { fail(23); break; }
                tc_fence_after();
                for (int kt = 0; kt < a.nkt; ++kt, ++it) {
                    const int sa = it % kAStages, sbs = it % kBStages;
                    if (!wait_cluster(&a_full[sa], (uint32_t)(it / kAStages) & 1u) ||
                        !wait_cluster(&b_full[sbs], (uint32_t)(it / kBStages) & 1u)) { fail(24); break; }
                    if (*abort_flag) break;
                    tc_fence_after();
                    const uint64_t dG = sw128_desc(smem + lay.a_off(sa));
                    const uint64_t dO = sw128_desc(smem + lay.a_off(sa) + kATile);
                    const uint64_t dB = sw128_desc(smem + lay.b_off(sbs));
#pragma unroll
                    for (int kk = 0; kk < kBK / 32; ++kk) {
                        const uint32_t acc = (kt | kk) ? 1u : 0u;
                        umma_i8_pair(tmem, dG + 2 * kk, dB + 2 * kk, idesc, acc);
                        umma_i8_pair(tmem + kOCol, dO + 2 * kk, dB + 2 * kk, idesc, acc);
                    }
                    commit_both(&a_empty[sa]);
                    commit_both(&b_empty[sbs]);
                }
                commit_both(acc_full);
            }
            // Drain: every MMA issued here (they read both CTAs' shared memory)
            // completes before either CTA passes the final cluster barrier.
            commit_own(mma_done);
            mbar_wait(mma_done, 0u);
        }
    } else {
        // ---------------- decoders (warps 3..) + epilogue (warps 3..6) ----------------
        const int dset = (warp - 3) >> 2;
        const int r = (tid - 96) & 127;
        const int q = warp & 3;
        const int row = q * 32 + lane;
        const int64_t j = jt0 + row;
        const bool stats = (j < a.M) && a.mean && a.sdinv;
        const double mu = stats ? a.mean[j] : 0.0;
        const double sd = stats ? a.sdinv[j] : 0.0;
        double run2 = 0.0, run4 = 0.0, run2b = 0.0;
        int cur = 0;
        auto flush = [&]() {
            if (!*abort_flag && j < jend && !a.raw_g && cur < nbk) {
                const double ls = a.left_scale[j];
                double upd = (run2 + run2b) * ls;
                const double seg = (double)a.V;
                const bool nonfinite = !isfinite(upd);
                const bool extreme = !nonfinite && isfinite(a.extreme_warn) && seg > 0.0 &&
                                     upd > a.extreme_warn * seg;
                if (a.guard_counts) {
                    if (nonfinite) atomicAdd(&a.guard_counts[0], 1ULL);
                    else if (extreme) atomicAdd(&a.guard_counts[1], 1ULL);
                }
                if (!(nonfinite || (extreme && a.drop_extreme))) {
                    if (upd < 0.0) upd = 0.0;
                    const int64_t o = (j - a.out_row0) * a.K + k0 + cur;
                    if (a.accum2) {
                        a.accum[o] += run2 * ls;
                        a.accum2[o] += run2b * ls;
                    } else {
                        a.accum[o] += upd;
                    }
                    if (a.mc) a.mc[o] += run4 * ls * ls;
                }
            }
            run2 = run4 = run2b = 0.0;
        };
        int it = 0;
        for (int g = 0; g < ngroups; ++g) {
            for (int kt = 0; kt < a.nkt; ++kt, ++it) {
                if (it % kDecSets != dset) continue;
                const int sp = it % kPkStages, sa = it % kAStages;
                if (!mbar_wait(&pk_full[sp], (uint32_t)(it / kPkStages) & 1u)) { fail(25); break; }
                if (*abort_flag) break;
                const uint4* pk = reinterpret_cast<const uint4*>(smem + lay.pk_off(sp) + r * 32);
                const uint4 p0 = pk[0], p1 = pk[1];
                mbar_arrive(&pk_empty[sp]);
                if (it >= kAStages &&
                    !mbar_wait(&a_empty[sa], ((uint32_t)(it / kAStages) & 1u) ^ 1u)) { fail(26); break; }
                uint8_t* gRow = smem + lay.a_off(sa) + (r >> 3) * 1024 + (r & 7) * 128;
                decode_row_sw128(p0, p1, gRow, gRow + kATile, r);
                fence_async_smem();
                arrive_cluster(a_full_l + (uint32_t)(sa * 8));
            }
            if (*abort_flag) break;
            if (dset != 0) continue;
            if (!mbar_wait(acc_full, (uint32_t)g & 1u)) { fail(27); break; }
            tc_fence_after();
            const int ncols = min(256, cols - g * 256);
            const uint32_t tbase = tmem + ((uint32_t)(q * 32) << 16);
            for (int c0 = 0; c0 < ncols; c0 += 32) {
                int rg[32], ro[32];
                tmem_ld32(tbase + (uint32_t)c0, rg);
                tmem_ld32(tbase + kOCol + (uint32_t)c0, ro);
                tmem_wait_ld();
#pragma unroll
                for (int p = 0; p < 8; ++p) {
                    const int gc = g * 256 + c0 + 4 * p;
                    const int bo = gc / a.ncolp;
                    const int v = (gc - bo * a.ncolp) >> 2;
                    if (bo >= nbk || v >= a.V) continue;
                    if (bo != cur) {
                        flush();
                        cur = bo;
                    }
                    const long long TG =
                        (((long long)rg[4 * p] * 128 + rg[4 * p + 1]) * 128 + rg[4 * p + 2]) * 128 +
                        rg[4 * p + 3];
                    const long long TO =
                        (((long long)ro[4 * p] * 128 + ro[4 * p + 1]) * 128 + ro[4 * p + 2]) * 128 +
                        ro[4 * p + 3];
                    if (a.raw_g) {
                        if (j < jend) {
                            a.raw_g[(j - a.out_row0) * a.V + v] = TG;
                            a.raw_o[(j - a.out_row0) * a.V + v] = TO;
                        }
                        continue;
                    }
                    const double wv = sd * a.colscale[(int64_t)(kb + bo) * a.V + v] *
                                      ((double)TG - mu * (double)TO);
                    const double w2 = wv * wv;
                    if (a.accum2 && v >= a.split_v) run2b += w2;
                    else run2 += w2;
                    run4 += w2 * w2;
                }
            }
            tc_fence_before();
            arrive_cluster(acc_empty_l);
        }
        if (dset == 0) flush();
    }
    tc_fence_before();
    __syncthreads();
    cluster_sync_all();  // the leader's MMAs have drained; no peer reads remain
    if (warp == 1) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                     "r"(kTmemCols));
    }
}

size_t p2_umma_pair_smem_bytes(int box_rows) { return (size_t)pair::Layout(box_rows).bytes() + 1024; }

void prepare_p2_umma_pair() {
    cudaFuncSetAttribute(p2_umma_pair_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)p2_umma_pair_smem_bytes(256));
}

void launch_p2_umma_pair(const CUtensorMap& tmA, const CUtensorMap& tmB, const P2UArgs& a,
                         cudaStream_t st) {
    const int64_t rows = a.j1 - a.j0;
    if ((!a.tiles && rows <= 0) || a.K <= 0) return;
    static std::atomic<unsigned long long> attr{0};
    once_per_device(attr, [] { prepare_p2_umma_pair(); });
    // With a tile table, j1 - j0 carries the number of PAIRS.
    const int nb = a.bins_per_cta > 0 ? a.bins_per_cta : 1;
    const int64_t pairs = a.tiles ? rows : (rows + 2 * pair::kBM - 1) / (2 * pair::kBM);
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)(2 * pairs), (unsigned)((a.K + nb - 1) / nb));
    cfg.blockDim = dim3(pair::kThreads);
    cfg.dynamicSmemBytes = p2_umma_pair_smem_bytes(a.box_rows);
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = 2;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, p2_umma_pair_kernel, tmA, tmB, a);
    count_launch();
}

}  // namespace umma
}  // namespace lds
