// Exact windowed LD scores on tcgen05 tensor cores (the deterministic
// estimator of compute_windowed_ld_chr_impl, winldcore.cpp:783-931).
//
// For SNPs j, i of one window the reference forms r_ij = x~_j . x~_i / N from
// restandardized columns (winldcore.cpp:215-267, :480-594).  Mathematically
// r_ij = c_ji / sqrt(c_jj c_ii) with
//   c_ji = sum_n o_jn o_in (g_jn - mu_j)(g_in - mu_i)
//        = GG - mu_i GO - mu_j OG + mu_j mu_i OO,
// where GG = sum g_j g_i, GO = sum g_j o_i, OG = sum o_j g_i, OO = sum o_j o_i
// are exact integer Gram sums of the decoded planes (g in {0,1,2}, o in {0,1}).
// One CTA owns a tile J of 128 SNPs and walks a run of partner tiles I: per
// K-step of 128 samples it decodes the packed codes of both tiles into
// SWIZZLE_128B int8 operands (A = G_J and O_J, B = [G_I | O_I], 256 rows) and
// issues two tcgen05.mma.kind::i8 (M=128, N=256, K=32) x 4 into TMEM:
//   columns   0..255: G_J [G_I | O_I]^T  -> GG | GO
//   columns 256..511: O_J [G_I | O_I]^T  -> OG | OO
// exact in int32 (|sums| <= 4N).  The epilogue turns them into r in FP64,
// applies f(r) = r^2 or the unbiased r^2 - (1 - r^2)/(corr_dim - 1)
// (winldcore.cpp:409-432), zeroes pairs outside the SNP's partner interval
// (:434-478) and accumulates f(r) annot[i, :] into this CTA's partial-sum slot.
// A second kernel adds the slots of each tile in a fixed order, so results
// are deterministic.
//
// Roles (192 threads): warp 0 TMA producer of packed-code tiles; warp 1 TMEM
// allocation and the single MMA-issuing thread; warps 2-5 decode operand rows
// and, after each partner tile, read the accumulators out.  Every mbarrier
// wait is bounded; on timeout the kernel records a code in `status`, stops
// issuing work, drains its copies and MMAs, and releases TMEM.
#include <cstdint>

#include "lds_internal.h"
#include "lds_tc.cuh"

namespace lds {
namespace gram {

using namespace umma;

constexpr int kBM = 128;           // SNPs per tile
constexpr int kBK = 128;           // samples per K-step
constexpr int kTile = kBM * kBK;   // 16 KB int8 operand tile
constexpr int kPk = 6;             // packed-code ring (J + I rows, 8 KB per stage)
constexpr int kPkBytes = 2 * kBM * 32;
constexpr int kStages = 2;         // decoded operand stages: G_J, O_J, G_I, O_I (64 KB)
constexpr int kThreads = 192;
constexpr uint32_t kTmemCols = 512;
constexpr int kKC = 8;             // annotation columns per epilogue pass

__host__ __device__ constexpr uint32_t stage_off(int s) { return (uint32_t)s * 4 * kTile; }
__host__ __device__ constexpr uint32_t pk_off(int s) {
    return (uint32_t)kStages * 4 * kTile + (uint32_t)s * kPkBytes;
}
__host__ __device__ constexpr uint32_t bar_off() { return pk_off(kPk); }
constexpr size_t kSmemBytes = (size_t)bar_off() + 256 + 1024;

__global__ void __launch_bounds__(kThreads, 1)
    gram_ld_kernel(const __grid_constant__ CUtensorMap tmC, GramArgs a) {
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>(
        (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem + bar_off());
    uint64_t* pk_full = bars;                    // [kPk] packed rows landed (TMA)
    uint64_t* pk_empty = pk_full + kPk;          // [kPk] packed rows read by the decoders
    uint64_t* a_full = pk_empty + kPk;           // [kStages] operands decoded
    uint64_t* a_empty = a_full + kStages;        // [kStages] operands consumed by the MMAs
    uint64_t* acc_full = a_empty + kStages;      // accumulators hold a finished tile pair
    uint64_t* acc_empty = acc_full + 1;          // accumulators read out
    uint64_t* mma_done = acc_empty + 1;          // drain of the issuer's MMAs
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(mma_done + 1);
    volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int4 item = a.items[blockIdx.x];
    const int64_t jrow0 = item.x, irow0 = item.y;
    const int nI = item.z, slot = item.w;
    const int total = nI * a.nkt;

    if (tid == 0) {
        for (int s = 0; s < kPk; ++s) {
            mbar_init(&pk_full[s], 1);
            mbar_init(&pk_empty[s], 128);
        }
        for (int s = 0; s < kStages; ++s) {
            mbar_init(&a_full[s], 128);
            mbar_init(&a_empty[s], 1);
        }
        mbar_init(acc_full, 1);
        mbar_init(acc_empty, 128);
        mbar_init(mma_done, 1);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32(tmem_slot)),
                     "r"(kTmemCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;
    auto fail = [&](int code) {
        atomicCAS(a.status, 0u, (unsigned)code);
        *abort_flag = 1;
    };

    if (warp == 0) {
        // ---------------- packed-code producer ----------------
        if (lane == 0) {
            int it = 0;
            for (; it < total; ++it) {
                const int s = it % kPk;
                if (it >= kPk && !mbar_wait(&pk_empty[s], ((uint32_t)(it / kPk) & 1u) ^ 1u)) {
                    fail(31);
                    break;
                }
                if (*abort_flag) break;
                const int t = it / a.nkt, kt = it - t * a.nkt;
                mbar_expect_tx(&pk_full[s], (uint32_t)kPkBytes);
                tma_load_2d(smem + pk_off(s), &tmC, kt * 32, (int)jrow0, &pk_full[s]);
                tma_load_2d(smem + pk_off(s) + kBM * 32, &tmC, kt * 32, (int)(irow0 + (int64_t)kBM * t),
                            &pk_full[s]);
            }
            // Drain: no copy may still be landing when the CTA exits.
            for (int j = max(0, it - kPk); j < it; ++j)
                mbar_wait(&pk_full[j % kPk], (uint32_t)(j / kPk) & 1u);
        }
    } else if (warp == 1) {
        // ---------------- MMA issuer ----------------
        if (lane == 0) {
            const uint32_t idesc = idesc_i8(kBM, 256);
            int it = 0;
            for (int t = 0; t < nI && !*abort_flag; ++t) {
                if (t > 0 && !mbar_wait(acc_empty, (uint32_t)(t - 1) & 1u)) { fail(32); break; }
                tc_fence_after();
                for (int kt = 0; kt < a.nkt; ++kt, ++it) {
                    const int sa = it % kStages;
                    if (!mbar_wait(&a_full[sa], (uint32_t)(it / kStages) & 1u)) { fail(33); break; }
                    if (*abort_flag) break;
                    tc_fence_after();
                    uint8_t* st = smem + stage_off(sa);
                    const uint64_t dGJ = sw128_desc(st);
                    const uint64_t dOJ = sw128_desc(st + kTile);
                    const uint64_t dB = sw128_desc(st + 2 * kTile);
#pragma unroll
                    for (int kk = 0; kk < kBK / 32; ++kk) {
                        const uint32_t acc = (kt | kk) ? 1u : 0u;
                        umma_i8(tmem, dGJ + 2 * kk, dB + 2 * kk, idesc, acc);
                        umma_i8(tmem + 256, dOJ + 2 * kk, dB + 2 * kk, idesc, acc);
                    }
                    umma_commit(&a_empty[sa]);
                }
                if (*abort_flag) break;
                umma_commit(acc_full);
            }
            // Drain: every MMA issued here completes before TMEM is released.
            umma_commit(mma_done);
            mbar_wait(mma_done, 0u);
        }
    } else {
        // ---------------- decoders + epilogue (warps 2..5) ----------------
        const int r = tid - 64;                 // operand row this thread decodes
        const int q = warp & 3;                 // TMEM lane quadrant of this warp
        const int jl = q * 32 + lane;           // accumulator row (SNP of tile J)
        const int64_t j = jrow0 + jl;
        const bool jvalid = j < a.row1;
        const int64_t lo = jvalid ? (int64_t)a.lo[j - a.row0] : 0;
        const int64_t hi = jvalid ? (int64_t)a.hi[j - a.row0] : 0;
        const double mu_j = jvalid ? a.mean[j] : 0.0;
        const double rs_j = jvalid ? a.rs[j] : 0.0;
        const uint32_t rowoff = (uint32_t)((r >> 3) * 1024 + (r & 7) * 128);
        int it = 0;
        for (int t = 0; t < nI && !*abort_flag; ++t) {
            for (int kt = 0; kt < a.nkt; ++kt, ++it) {
                const int sp = it % kPk, sa = it % kStages;
                if (!mbar_wait(&pk_full[sp], (uint32_t)(it / kPk) & 1u)) { fail(34); break; }
                if (*abort_flag) break;
                const uint4* pj = reinterpret_cast<const uint4*>(smem + pk_off(sp) + r * 32);
                const uint4* pi = reinterpret_cast<const uint4*>(smem + pk_off(sp) + kBM * 32 + r * 32);
                const uint4 j0 = pj[0], j1 = pj[1], i0 = pi[0], i1 = pi[1];
                mbar_arrive(&pk_empty[sp]);
                if (it >= kStages &&
                    !mbar_wait(&a_empty[sa], ((uint32_t)(it / kStages) & 1u) ^ 1u)) { fail(35); break; }
                uint8_t* st = smem + stage_off(sa);
                decode_row_sw128(j0, j1, st + rowoff, st + kTile + rowoff, r);
                decode_row_sw128(i0, i1, st + 2 * kTile + rowoff, st + 3 * kTile + rowoff, r);
                fence_async_smem();
                mbar_arrive(&a_full[sa]);
            }
            if (*abort_flag) break;
            // ---- epilogue of partner tile t ----
            if (!mbar_wait(acc_full, (uint32_t)t & 1u)) { fail(36); break; }
            tc_fence_after();
            const int64_t ib = irow0 + (int64_t)kBM * t;
            const uint32_t tb = tmem + ((uint32_t)(q * 32) << 16);
            for (int kc = 0; kc < a.K; kc += kKC) {
                double acc[kKC];
#pragma unroll
                for (int b = 0; b < kKC; ++b) acc[b] = 0.0;
                for (int c0 = 0; c0 < kBM; c0 += 16) {
                    if (ib + c0 >= a.row1) break;  // warp-uniform
                    int gg[16], go[16], og[16], oo[16];
                    tmem_ld16(tb + (uint32_t)c0, gg);
                    tmem_ld16(tb + 128u + (uint32_t)c0, go);
                    tmem_ld16(tb + 256u + (uint32_t)c0, og);
                    tmem_ld16(tb + 384u + (uint32_t)c0, oo);
                    tmem_wait_ld();
#pragma unroll
                    for (int u = 0; u < 16; ++u) {
                        const int64_t i = ib + c0 + u;  // warp-uniform
                        if (i >= a.row1) continue;
                        const double mu_i = __ldg(a.mean + i), rs_i = __ldg(a.rs + i);
                        const double c = (double)gg[u] - mu_i * (double)go[u] -
                                         mu_j * (double)og[u] + mu_j * mu_i * (double)oo[u];
                        const double rr = c * rs_j * rs_i;
                        double f = rr * rr;
                        if (a.corr_den > 0.0) f -= (1.0 - f) * a.corr_den;
                        if (!(jvalid && i >= lo && i < hi)) f = 0.0;
                        const double* an = a.annot + (i - a.row0) * a.K + kc;
#pragma unroll
                        for (int b = 0; b < kKC; ++b)
                            if (kc + b < a.K) acc[b] += f * __ldg(an + b);
                    }
                }
                if (jvalid) {
                    double* out = a.partial + ((int64_t)slot * kBM + jl) * a.K + kc;
#pragma unroll
                    for (int b = 0; b < kKC; ++b)
                        if (kc + b < a.K) out[b] += acc[b];
                }
            }
            tc_fence_before();
            mbar_arrive(acc_empty);
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                     "r"(kTmemCols));
    }
}

// out[(j - row0) ld_row + b ld_col] = sum over the slots of j's tile, in slot order.
__global__ void gram_reduce_kernel(const double* __restrict__ partial,
                                   const int32_t* __restrict__ slot_beg, int64_t row0, int64_t row1,
                                   int K, double* __restrict__ out, int64_t ld_row, int64_t ld_col) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t n = (row1 - row0) * K;
    if (t >= n) return;
    const int64_t jr = t / K;
    const int b = (int)(t - jr * K);
    const int64_t T = jr / kBM;
    const int jl = (int)(jr - T * kBM);
    double s = 0.0;
    for (int32_t sl = slot_beg[T]; sl < slot_beg[T + 1]; ++sl)
        s += partial[((int64_t)sl * kBM + jl) * K + b];
    out[jr * ld_row + (int64_t)b * ld_col] = s;
}

}  // namespace gram

size_t gram_ld_smem_bytes() { return gram::kSmemBytes; }

void launch_gram_ld(const CUtensorMap& tmC, const GramArgs& a, int n_items, cudaStream_t st) {
    if (n_items <= 0) return;
    static std::atomic<unsigned long long> attr{0};
    once_per_device(attr, [] {
        cudaFuncSetAttribute(gram::gram_ld_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)gram::kSmemBytes);
    });
    gram::gram_ld_kernel<<<(unsigned)n_items, gram::kThreads, gram::kSmemBytes, st>>>(tmC, a);
    count_launch();
}

void launch_gram_reduce(const double* partial, const int32_t* slot_beg, int64_t row0, int64_t row1,
                        int K, double* out, int64_t ld_row, int64_t ld_col, cudaStream_t st) {
    const int64_t n = (row1 - row0) * K;
    if (n <= 0) return;
    gram::gram_reduce_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(
        partial, slot_beg, row0, row1, K, out, ld_row, ld_col);
    count_launch();
}

}  // namespace lds
