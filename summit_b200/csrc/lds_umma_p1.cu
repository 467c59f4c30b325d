// Phase 1 on tcgen05 tensor cores: Y[:, (k, v)] = sum_{j in bin k} x_j w_{j,(k,v)}.
//
// UMMA shape per CTA: M = 128 samples, N = the bin's digit columns (4 per
// probe, <= 256 per pass), K = 128 member SNPs per stage.  The A operand is
// the decoded genotype tile in MN-major SWIZZLE_128B layout: a packed SNP row
// already lists samples contiguously, so decoder thread t expands member SNP t
// of the stage into row t of the tile with no transpose.  G and O tiles are
// multiplied by the digits of W1 = s_j sc z and of -W2 = -mu_j W1 (both via
// TMA, SWIZZLE_128B, K-major) into ONE accumulator, so TMEM holds
// G.W1 - O.W2 = sum_j (g - mu_j o) s_j sc z directly.
//
// Roles (704 threads): warp 0 TMA producer for the digit tiles; warp 1 TMEM
// allocation and the single MMA-issuing thread; warps 2-5 gather the member
// SNPs' packed bytes from global memory (one row each, kept several stages
// ahead by cp.async) and decode them into the operand tiles; warps 6-21 (four
// per TMEM lane quadrant) read the accumulator out and split it into digits.  Two TMEM accumulators let the MMAs of the next job (super-bin,
// column group) run while the epilogue of the previous one drains, which
// matters for windowed estimates, whose super-bins are a few K-steps long.
#include <cstdint>
#include <cstdio>

#include "lds_internal.h"
#include "lds_tc.cuh"
#include "lds_umma.h"

namespace lds {
namespace umma {

namespace p1 {
constexpr int kStages = 2;
constexpr int kBM = 128;          // samples per CTA
constexpr int kBK = 128;          // member SNPs per stage
constexpr int kATile = 128 * 128; // 16 KB
constexpr int kWTile = 256 * 128; // 32 KB (max digit columns per pass)
constexpr int kStageBytes = 2 * kATile + 2 * kWTile;  // 96 KB
constexpr int kThreads = 704;
constexpr int kEpiThreads = 512;         // warps 6..21: four per TMEM lane quadrant
constexpr int kAccCols = 256;            // one accumulator: <= 256 digit columns
constexpr uint32_t kTmemCols = 512;      // two accumulators (MMA of job j+1 || epilogue of j)
constexpr int kRing = 6;                 // gathered packed rows in flight per decoder thread
constexpr int kRingSlot = 128 * 32;      // 128 member rows x 32 bytes
}  // namespace p1

__global__ void __launch_bounds__(p1::kThreads, 1)
    p1_umma_kernel(const __grid_constant__ CUtensorMap tmW, P1UArgs a) {
    using namespace p1;
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>(
        (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint8_t* ring = smem + kStages * kStageBytes;
    uint64_t* bars = reinterpret_cast<uint64_t*>(ring + kRing * kRingSlot);
    uint64_t* full_w = bars;                    // [kStages] weight tiles landed (TMA)
    uint64_t* full_dec = bars + kStages;        // [kStages] genotype tiles decoded
    uint64_t* empty = bars + 2 * kStages;       // [kStages] stage consumed by the MMAs
    uint64_t* acc_full = bars + 3 * kStages;    // [2] accumulator b holds a finished job
    uint64_t* acc_empty = acc_full + 2;         // [2] accumulator b read out
    uint64_t* mma_done = acc_empty + 2;         // drain of the issuer's MMAs
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(mma_done + 1);
    volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int64_t i0 = (int64_t)blockIdx.x * kBM;
    // This CTA's super-bins: [kb0, kb1); a job is one (super-bin, column group).
    const int kb0 = blockIdx.y * a.sb_per_cta;
    const int kb1 = min(a.K, kb0 + a.sb_per_cta);

    if (tid == 0) {
        for (int s = 0; s < kStages; ++s) {
            mbar_init(&full_w[s], 1);
            mbar_init(&full_dec[s], 4);            // one arrival per decoder warp
            mbar_init(&empty[s], 1);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(&acc_full[b], 1);
            mbar_init(&acc_empty[b], kEpiThreads / 32);  // one arrival per epilogue warp
        }
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
    auto nkt_of = [&](int k) { return (int)((a.bin_off[k + 1] - a.bin_off[k]) / kBK); };

    if (warp == 0) {
        // ---------------- TMA producer of weight-digit tiles ----------------
        if (lane == 0) {
            int it = 0;
            for (int k = kb0; k < kb1 && !*abort_flag; ++k) {
                const int nkt = nkt_of(k);
                for (int g = 0; g < a.ngroups && !*abort_flag; ++g) {
                    for (int kt = 0; kt < nkt; ++kt, ++it) {
                        const int s = it % kStages;
                        const uint32_t ph = (uint32_t)(it / kStages) & 1u;
                        if (it >= kStages && !mbar_wait(&empty[s], ph ^ 1u)) { fail(11); break; }
                        if (*abort_flag) break;
                        uint8_t* st = smem + s * kStageBytes;
                        mbar_expect_tx(&full_w[s], (uint32_t)(2 * a.box_rows * kBK));
                        const int y0 = k * 2 * a.ncolp + g * 256;
                        tma_load_2d(st + 2 * kATile, &tmW, kt * kBK, y0, &full_w[s]);
                        tma_load_2d(st + 2 * kATile + kWTile, &tmW, kt * kBK, y0 + a.ncolp,
                                    &full_w[s]);
                    }
                }
            }
            // Drain: no tile copy may still be landing when the CTA exits
            // (only reachable with copies outstanding after an abort).
            for (int j = max(0, it - kStages); j < it; ++j)
                mbar_wait(&full_w[j % kStages], (uint32_t)(j / kStages) & 1u);
        }
    } else if (warp == 1) {
        // ---------------- MMA issuer ----------------
        if (lane == 0) {
            int it = 0, au = 0;  // stage counter, jobs (accumulator uses)
            for (int k = kb0; k < kb1 && !*abort_flag; ++k) {
                const int nkt = nkt_of(k);
                if (nkt == 0) continue;
                for (int g = 0; g < a.ngroups && !*abort_flag; ++g, ++au) {
                    const int b = au & 1, u = au >> 1;
                    const int ncols = min(kAccCols, a.ncolp - g * 256);
                    const uint32_t idesc = idesc_i8_amn(kBM, ncols);
                    const uint32_t acc = tmem + (uint32_t)(b * kAccCols);
                    if (u > 0 && !mbar_wait(&acc_empty[b], (uint32_t)(u - 1) & 1u)) { fail(12); break; }
                    tc_fence_after();
                    for (int kt = 0; kt < nkt; ++kt, ++it) {
                        const int s = it % kStages;
                        const uint32_t ph = (uint32_t)(it / kStages) & 1u;
                        if (!mbar_wait(&full_dec[s], ph) || !mbar_wait(&full_w[s], ph)) {
                            fail(13);
                            break;
                        }
                        if (*abort_flag) break;
                        tc_fence_after();
                        uint8_t* st = smem + s * kStageBytes;
                        const uint64_t dG = sw128_desc_mn(st);
                        const uint64_t dO = sw128_desc_mn(st + kATile);
                        const uint64_t dW1 = sw128_desc(st + 2 * kATile);
                        const uint64_t dW2 = sw128_desc(st + 2 * kATile + kWTile);
#pragma unroll
                        for (int kk = 0; kk < kBK / 32; ++kk) {
                            // A advances 32 K-rows = 4 swizzle atoms (4 KB); B advances 32 bytes.
                            umma_i8(acc, dG + 256 * kk, dW1 + 2 * kk, idesc, (kt | kk) ? 1u : 0u);
                            umma_i8(acc, dO + 256 * kk, dW2 + 2 * kk, idesc, 1u);
                        }
                        umma_commit(&empty[s]);
                    }
                    umma_commit(&acc_full[b]);
                }
            }
            // Drain: every MMA issued here completes before TMEM is released.
            umma_commit(mma_done);
            mbar_wait(mma_done, 0u);
        }
    } else if (warp < 6) {
        // ---------------- gather + decode (warps 2..5) ----------------
        const int t = tid - 64;
        const uint8_t* codes = a.codes + i0 / 4;
        // Gather prefetcher: walks the same (super-bin, group, K-step) sequence
        // kRing steps ahead, copying this thread's member row into a ring slot.
        // The member row of the step being fetched is read from rowind one step
        // earlier (row_next), so that load's latency overlaps a step of work
        // instead of stalling the cp.async that needs the address.
        int pk = kb0, pg = 0, pkt = 0, pit = 0;
        auto cursor_row = [&]() -> int64_t {  // rowind of the cursor's step, or -1 past the end
            while (pk < kb1 && nkt_of(pk) == 0) { ++pk; pg = 0; pkt = 0; }
            if (pk >= kb1) return -1;
            int64_t row = a.rowind[a.bin_off[pk] + (int64_t)pkt * kBK + t];
            // bounds-checked build: a member row outside the image is not gathered
            if (!in_range(a.m_pad == 0 || (row >= 0 && row < a.m_pad), 0x1001u)) row = -2;
            if (++pkt == nkt_of(pk)) {
                pkt = 0;
                if (++pg == a.ngroups) { pg = 0; ++pk; }
            }
            return row;
        };
        int64_t row_next = cursor_row();
        auto prefetch_one = [&]() {
            const int64_t row = row_next;
            row_next = cursor_row();
            if (row >= 0) {
                const uint8_t* src = codes + row * a.nbp;
                uint8_t* dst = ring + (pit % kRing) * kRingSlot + t * 32;
                cp_async16(dst, src);
                cp_async16(dst + 16, src + 16);
            }
            cp_async_commit();
            ++pit;
        };
        for (int d = 0; d < kRing - 1; ++d) prefetch_one();
        int it = 0;
        for (int k = kb0; k < kb1 && !__any_sync(0xffffffffu, *abort_flag != 0); ++k) {
            const int nkt = nkt_of(k);
            for (int g = 0; g < a.ngroups && nkt > 0 && !__any_sync(0xffffffffu, *abort_flag != 0); ++g) {
                for (int kt = 0; kt < nkt; ++kt, ++it) {
                    const int s = it % kStages;
                    const uint32_t ph = (uint32_t)(it / kStages) & 1u;
                    prefetch_one();  // step it + kRing - 1
                    asm volatile("cp.async.wait_group %0;\n" ::"n"(kRing - 1));
                    const uint4* src =
                        reinterpret_cast<const uint4*>(ring + (it % kRing) * kRingSlot + t * 32);
                    const uint4 c0 = src[0], c1 = src[1];
                    if (it >= kStages && !__all_sync(0xffffffffu, mbar_wait(&empty[s], ph ^ 1u))) {
                        fail(14);
                        break;
                    }
                    if (__any_sync(0xffffffffu, *abort_flag != 0)) break;
                    uint8_t* st = smem + s * kStageBytes;
                    uint8_t* gRow = st + (t >> 3) * 1024 + (t & 7) * 128;
                    decode_row_sw128(c0, c1, gRow, gRow + kATile, t);
                    fence_async_smem();
                    __syncwarp();  // orders the warp's operand stores before its one arrival
                    if (lane == 0) mbar_arrive(&full_dec[s]);
                }
            }
        }
        cp_async_wait_all();  // no gather copy may outlive the CTA (abort path)
    } else {
        // ---------------- epilogue (warps 6..21) ----------------
        const int e = tid - 192;
        const int q = warp & 3;                  // TMEM lane quadrant of this warp
        const int h = (warp - 6) >> 2;           // which quarter of the 16-column chunks
        const int64_t i = i0 + q * 32 + lane;    // sample row of this thread's accumulator lane
        int au = 0;
        for (int k = kb0; k < kb1 && !__any_sync(0xffffffffu, *abort_flag != 0); ++k) {
            const int nkt = nkt_of(k);
            // This sample tile's block of super-bin k in phase 2's digit layout
            // (digit_offset): ncolp rows of 128 bytes.
            int8_t* const yblk =
                a.yq ? a.yq + ((int64_t)blockIdx.x * a.K * a.ncolp + (int64_t)k * a.ncolp) * 128
                     : nullptr;
            if (a.yq) {
                // Digit padding rows 4V..ncolp of this tile read as zero in phase 2.
                for (int idx = e; idx < (a.ncolp - 4 * a.V) * 8; idx += kEpiThreads)
                    *reinterpret_cast<uint4*>(yblk + (4 * a.V + (idx >> 3)) * 128 + (idx & 7) * 16) =
                        make_uint4(0, 0, 0, 0);
            }
            if (nkt == 0) {
                // Bin without members: its sketch columns are zero (the
                // reference's untouched-bin zeroing, gw_ldscore.py:2017-2019).
                if (a.yq) {
                    for (int idx = e; idx < 4 * a.V * 8; idx += kEpiThreads)
                        *reinterpret_cast<uint4*>(yblk + (idx >> 3) * 128 + (idx & 7) * 16) =
                            make_uint4(0, 0, 0, 0);
                } else {
                    for (int idx = e; idx < a.V * 64; idx += kEpiThreads)
                        *reinterpret_cast<uint4*>(a.Y + ((int64_t)k * a.V + (idx >> 6)) * a.N_pad +
                                                  i0 + (idx & 63) * 2) = make_uint4(0, 0, 0, 0);
                }
                continue;
            }
            for (int g = 0; g < a.ngroups && !__any_sync(0xffffffffu, *abort_flag != 0); ++g, ++au) {
                const int b = au & 1, u = au >> 1;
                // This group's 64 per-probe shifts (or scales), two per lane, loaded
                // before the accumulator wait so the loads overlap the MMAs; the
                // loop below broadcasts them with shuffles (warp-local, no barrier).
                int shA = 0, shB = 0;
                double scA = 0.0, scB = 0.0;
                {
                    const int va = g * 64 + lane, vb = va + 32;
                    const int64_t o = (int64_t)k * a.V;
                    if (a.yq) {
                        if (va < a.V) shA = a.yshift[o + va];
                        if (vb < a.V) shB = a.yshift[o + vb];
                    } else {
                        if (va < a.V) scA = a.colscale[o + va];
                        if (vb < a.V) scB = a.colscale[o + vb];
                    }
                }
                if (!__all_sync(0xffffffffu, mbar_wait(&acc_full[b], (uint32_t)u & 1u))) {
                    fail(15);
                    break;
                }
                tc_fence_after();
                const int ncols = min(kAccCols, a.ncolp - g * 256);
                const uint32_t tbase = tmem + (uint32_t)(b * kAccCols) + ((uint32_t)(q * 32) << 16);
                if (a.yq) {
                    // Digits straight into phase 2's operand layout, 8 probes (32
                    // digit columns) per TMEM load; the quadrant's four warps take
                    // every fourth chunk.  With y = T 2^(eW-28) and the column
                    // exponent eY fixed in advance by a bound on |y|, the sketch's
                    // 28-bit value is R = rint(T 2^(eW-eY)) (round half to even);
                    // its balanced base-128 digits are exact integer work.  A 4 x 4
                    // byte transpose within each lane quad turns the lanes' digit
                    // words (4 digits of one sample) into words of one digit for 4
                    // consecutive samples, stored straight to global memory (a warp
                    // writes 4 digit rows x 32 samples per probe).  Lane 4a + t
                    // stores digit row 4v + t, samples s = 32 q + 4a of the block:
                    // 16-byte chunk s / 16 = 2q + a / 4, swizzled with the row's
                    // low three bits, (4 v + t) & 7 = 4 (v & 1) + t.
                    const int qd = lane & 3;
                    const uint32_t selA = qd < 2 ? 0x5410u : 0x3276u;
                    const uint32_t selB = (qd & 1) ? 0x3715u : 0x6240u;
                    const int chunk = 2 * q + (lane >> 4);
                    int8_t* const ylane = yblk + qd * 128 + 4 * ((lane >> 2) & 3);
                    for (int c0 = 32 * h; c0 < ncols; c0 += 128) {
                        int rr[32];
                        tmem_ld32(tbase + (uint32_t)c0, rr);
                        tmem_wait_ld();
                        const int vl0 = c0 >> 2;                    // first probe of the chunk
                        const int nv = a.V - (g * 64 + vl0);        // probes left (warp-uniform)
#pragma unroll
                        for (int p = 0; p < 8; ++p) {
                            const int vl = vl0 + p;
                            const int sh = __shfl_sync(0xffffffffu, vl < 32 ? shA : shB, vl & 31);
                            const long long T =
                                (((long long)rr[4 * p] * 128 + rr[4 * p + 1]) * 128 +
                                 rr[4 * p + 2]) * 128 + rr[4 * p + 3];
                            long long R;
                            if (sh >= 0) {
                                R = T << sh;
                            } else {
                                const int r = -sh;
                                R = (T + ((1LL << (r - 1)) - 1) + ((T >> r) & 1)) >> r;
                            }
                            // |R| < 2^28 (the bound fixed eY): with U = R + 63 (2^14 +
                            // 2^7 + 1) the low three base-128 digits of U are the
                            // balanced digits d1..d3 (in [-63, 64]) plus 63 and U >> 21
                            // is d0; the byte-wise subtraction of 63 from bytes 1..3
                            // (their top bits set first, so no byte borrows) leaves
                            // the word [d0, d1, d2, d3].
                            const int U = (int)R + 63 * (16384 + 128 + 1);
                            uint32_t w = (uint32_t)(U >> 21) & 0xFFu;
                            w |= ((uint32_t)(U >> 14) & 127u) << 8;
                            w |= ((uint32_t)(U >> 7) & 127u) << 16;
                            w |= ((uint32_t)U & 127u) << 24;
                            w = ((w | 0x80808000u) - 0x3F3F3F00u) ^ 0x80808000u;
                            // 4 x 4 byte transpose across the quad: lane 4a + t ends
                            // with digit t of samples 4a .. 4a + 3.
                            w = __byte_perm(w, __shfl_xor_sync(0xffffffffu, w, 2), selA);
                            w = __byte_perm(w, __shfl_xor_sync(0xffffffffu, w, 1), selB);
                            if (p < nv) {
                                const int v = g * 64 + vl;
                                *reinterpret_cast<uint32_t*>(
                                    ylane + v * 512 + ((chunk ^ (4 * (v & 1) + qd)) << 4)) = w;
                            }
                        }
                    }
                } else {
                for (int c0c = 16 * h; c0c < ncols; c0c += 64) {
                    int rr[16];
                    tmem_ld16(tbase + (uint32_t)c0c, rr);
                    tmem_wait_ld();
#pragma unroll
                    for (int p = 0; p < 4; ++p) {
                        const int vl = c0c / 4 + p;  // probe within the group (warp-uniform)
                        const int v = g * 64 + vl;
                        if (v >= a.V) continue;
                        const long long T =
                            (((long long)rr[4 * p] * 128 + rr[4 * p + 1]) * 128 + rr[4 * p + 2]) *
                                128 + rr[4 * p + 3];
                        const double sc = __shfl_sync(0xffffffffu, vl < 32 ? scA : scB, vl & 31);
                        a.Y[((int64_t)k * a.V + v) * a.N_pad + i] = sc * (double)T;
                    }
                }
                }
                tc_fence_before();
                __syncwarp();
                if (lane == 0) mbar_arrive(&acc_empty[b]);
            }
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

// Weight digits in the layout of p1_umma_kernel:
// Wq[((k*2 + part)*ncolp + 4 v + t)*Lmax + r], part 0 = W1, 1 = -W2.
// One CTA per (k, v); padding entries are left as zero (buffer cleared once).
__global__ void p1_weights4_kernel(P1UWeights w, const double* __restrict__ mean,
                                   const double* __restrict__ sdinv, const double* __restrict__ Z,
                                   int64_t z_ld) {
    __shared__ double red[32];
    const int k = blockIdx.x / w.V, v = blockIdx.x - (blockIdx.x / w.V) * w.V;
    const int64_t r0 = w.bin_off[k], nnzp = w.bin_off[k + 1] - r0;
    double amax = 0.0;
    for (int64_t r = threadIdx.x; r < nnzp; r += blockDim.x) {
        const double sc = w.sc[r0 + r];
        if (sc == 0.0) continue;
        const int64_t j = w.rowind[r0 + r];
        const double w1 = sdinv[j] * (sc * Z[(int64_t)v * z_ld + j]);
        amax = fmax(amax, fmax(fabs(w1), fabs(mean[j] * w1)));
    }
    for (int o = 16; o; o >>= 1) amax = fmax(amax, __shfl_xor_sync(0xffffffffu, amax, o));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = amax;
    __syncthreads();
    if (threadIdx.x < 32) {
        double x = (threadIdx.x < (blockDim.x >> 5)) ? red[threadIdx.x] : 0.0;
        for (int o = 16; o; o >>= 1) x = fmax(x, __shfl_xor_sync(0xffffffffu, x, o));
        if (threadIdx.x == 0) red[0] = x;
    }
    __syncthreads();
    amax = red[0];
    int e = 0;
    if (amax > 0.0 && isfinite(amax)) {
        e = ilogb(amax) + 1;
        if (ldexp(amax, 7 - e) > 127.0) e += 1;
    }
    int8_t* b1 = w.wq + ((int64_t)(k * 2 + 0) * w.ncolp + 4 * v) * w.lmax;
    int8_t* b2 = w.wq + ((int64_t)(k * 2 + 1) * w.ncolp + 4 * v) * w.lmax;
    for (int64_t r = threadIdx.x; r < nnzp; r += blockDim.x) {
        const double sc = w.sc[r0 + r];
        double t1 = 0.0, t2 = 0.0;
        if (sc != 0.0) {
            const int64_t j = w.rowind[r0 + r];
            const double w1 = sdinv[j] * (sc * Z[(int64_t)v * z_ld + j]);
            t1 = ldexp(w1, 7 - e);
            t2 = ldexp(-(mean[j] * w1), 7 - e);
        }
#pragma unroll
        for (int s = 0; s < 4; ++s) {
            const double q1 = rint(t1), q2 = rint(t2);
            b1[(int64_t)s * w.lmax + r] = (int8_t)q1;
            b2[(int64_t)s * w.lmax + r] = (int8_t)q2;
            t1 = (t1 - q1) * 128.0;
            t2 = (t2 - q2) * 128.0;
        }
    }
    if (threadIdx.x == 0) w.colscale[(int64_t)k * w.V + v] = ldexp(1.0, e - 7 - 21);
    if (w.ycolscale) {
        // Rigorous bound on |y_i| = |sum_j g_ij w1_j - o_ij w2_j| <= sum_j 2|w1_j| + |w2_j|
        // (inflated for the digit rounding of the weights), fixing the sketch's
        // digit exponent before phase 1 runs.
        double bsum = 0.0;
        for (int64_t r = threadIdx.x; r < nnzp; r += blockDim.x) {
            const double sc = w.sc[r0 + r];
            if (sc == 0.0) continue;
            const int64_t j = w.rowind[r0 + r];
            const double w1 = sdinv[j] * (sc * Z[(int64_t)v * z_ld + j]);
            bsum += 2.0 * fabs(w1) + fabs(mean[j] * w1);
        }
        __syncthreads();
        for (int o = 16; o; o >>= 1) bsum += __shfl_xor_sync(0xffffffffu, bsum, o);
        if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = bsum;
        __syncthreads();
        if (threadIdx.x == 0) {
            double tot = 0.0;
            for (int q = 0; q < (int)(blockDim.x >> 5); ++q) tot += red[q];
            // The weights enter as 4-digit values, each within 2^(e-29) of w1 and
            // of mu*w1: add that slack for every member, then the FP64 rounding
            // of the sum.
            tot = (tot + (double)nnzp * 3.0 * ldexp(1.0, e - 29)) * (1.0 + 1e-9);
            int ey = 0;
            if (tot > 0.0 && isfinite(tot)) {
                ey = ilogb(tot) + 1;
                if (ldexp(tot, 7 - ey) > 127.0) ey += 1;
            }
            w.ycolscale[(int64_t)k * w.V + v] = ldexp(1.0, ey - 28);
            // digit shift for the phase-1 epilogue: R = rint(T 2^(eW - eY))
            w.yshift[(int64_t)k * w.V + v] = e - ey;
        }
    }
}

void launch_p1_weights4(const P1UWeights& w, const double* mean, const double* sdinv,
                        const double* Z, int64_t z_ld, cudaStream_t st) {
    if (w.K * w.V == 0) return;
    p1_weights4_kernel<<<(unsigned)(w.K * w.V), 256, 0, st>>>(w, mean, sdinv, Z, z_ld);
    count_launch();
}

size_t p1_umma_smem_bytes() {
    return (size_t)p1::kStages * p1::kStageBytes + (size_t)p1::kRing * p1::kRingSlot + 1024 + 256;
}

void prepare_p1_umma() {
    cudaFuncSetAttribute(p1_umma_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)p1_umma_smem_bytes());
}

void launch_p1_umma(const CUtensorMap& tmW, const P1UArgs& a, int64_t N_pad, cudaStream_t st) {
    static std::atomic<unsigned long long> attr{0};
    once_per_device(attr, [] { prepare_p1_umma(); });
    const int spc = a.sb_per_cta > 0 ? a.sb_per_cta : 1;
    P1UArgs b = a;
    b.sb_per_cta = spc;
    dim3 grid((unsigned)(N_pad / p1::kBM), (unsigned)((a.K + spc - 1) / spc));
    p1_umma_kernel<<<grid, p1::kThreads, p1_umma_smem_bytes(), st>>>(tmW, b);
    count_launch();
}

}  // namespace umma
}  // namespace lds
