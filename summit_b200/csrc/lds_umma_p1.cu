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
// Roles (192 threads): warp 0 TMA producer for the digit tiles; warp 1 TMEM
// allocation and the single MMA-issuing thread; warps 2-5 gather the member
// SNPs' packed bytes from global memory (one row each, prefetched one stage
// ahead), decode them into the operand tiles, and run the epilogue.
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
constexpr int kThreads = 192;
constexpr uint32_t kTmemCols = 256;
}  // namespace p1

__global__ void __launch_bounds__(p1::kThreads, 1)
    p1_umma_kernel(const __grid_constant__ CUtensorMap tmW, P1UArgs a) {
    using namespace p1;
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>(
        (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem + kStages * kStageBytes);
    uint64_t* full_w = bars;
    uint64_t* full_dec = bars + kStages;
    uint64_t* empty = bars + 2 * kStages;
    uint64_t* acc_full = bars + 3 * kStages;
    uint64_t* acc_empty = bars + 3 * kStages + 1;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 3 * kStages + 2);
    volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int k = blockIdx.y;
    const int64_t i0 = (int64_t)blockIdx.x * kBM;
    const int64_t r0 = a.bin_off[k];
    const int nkt = (int)((a.bin_off[k + 1] - r0) / kBK);

    if (tid == 0) {
        for (int s = 0; s < kStages; ++s) {
            mbar_init(&full_w[s], 1);
            mbar_init(&full_dec[s], 128);
            mbar_init(&empty[s], 1);
        }
        mbar_init(acc_full, 1);
        mbar_init(acc_empty, 128);
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

    if (nkt > 0) {
        if (warp == 0) {
            if (lane == 0) {
                int it = 0;
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
        } else if (warp == 1) {
            if (lane == 0) {
                int it = 0;
                for (int g = 0; g < a.ngroups && !*abort_flag; ++g) {
                    const int ncols = min(256, a.ncolp - g * 256);
                    const uint32_t idesc = idesc_i8_amn(kBM, ncols);
                    if (g > 0 && !mbar_wait(acc_empty, (uint32_t)(g - 1) & 1u)) { fail(12); break; }
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
                            umma_i8(tmem, dG + 256 * kk, dW1 + 2 * kk, idesc, (kt | kk) ? 1u : 0u);
                            umma_i8(tmem, dO + 256 * kk, dW2 + 2 * kk, idesc, 1u);
                        }
                        umma_commit(&empty[s]);
                    }
                    umma_commit(acc_full);
                }
            }
        } else {
            // Decoders: thread t handles member row t of every stage.
            const int t = tid - 64;
            const int q = warp & 3;
            const uint8_t* codes = a.codes + i0 / 4;
            int it = 0;
            for (int g = 0; g < a.ngroups && !*abort_flag; ++g) {
                const int32_t* ri = a.rowind + r0;
                uint4 c0, c1;
                {
                    const uint4* src = reinterpret_cast<const uint4*>(codes + (int64_t)ri[t] * a.nbp);
                    c0 = __ldg(src);
                    c1 = __ldg(src + 1);
                }
                for (int kt = 0; kt < nkt; ++kt, ++it) {
                    const int s = it % kStages;
                    const uint32_t ph = (uint32_t)(it / kStages) & 1u;
                    uint4 n0 = c0, n1 = c1;
                    if (kt + 1 < nkt) {
                        const uint4* src = reinterpret_cast<const uint4*>(
                            codes + (int64_t)ri[(kt + 1) * kBK + t] * a.nbp);
                        n0 = __ldg(src);
                        n1 = __ldg(src + 1);
                    }
                    if (it >= kStages && !mbar_wait(&empty[s], ph ^ 1u)) { fail(14); break; }
                    if (*abort_flag) break;
                    uint8_t* st = smem + s * kStageBytes;
                    uint8_t* gRow = st + (t >> 3) * 1024 + (t & 7) * 128;
                    decode_row_sw128(c0, c1, gRow, gRow + kATile, t);
                    fence_async_smem();
                    mbar_arrive(&full_dec[s]);
                    c0 = n0;
                    c1 = n1;
                }
                if (*abort_flag) break;
                if (!mbar_wait(acc_full, (uint32_t)g & 1u)) { fail(15); break; }
                tc_fence_after();
                const int ncols = min(256, a.ncolp - g * 256);
                const uint32_t tbase = tmem + ((uint32_t)(q * 32) << 16);
                const int64_t i = i0 + q * 32 + lane;
                for (int c0c = 0; c0c < ncols; c0c += 32) {
                    int rr[32];
                    tmem_ld32(tbase + (uint32_t)c0c, rr);
                    tmem_wait_ld();
#pragma unroll
                    for (int p = 0; p < 8; ++p) {
                        const int v = g * 64 + c0c / 4 + p;
                        if (v >= a.V) continue;
                        const long long T =
                            (((long long)rr[4 * p] * 128 + rr[4 * p + 1]) * 128 + rr[4 * p + 2]) *
                                128 + rr[4 * p + 3];
                        a.Y[((int64_t)k * a.V + v) * a.N_pad + i] =
                            a.colscale[(int64_t)k * a.V + v] * (double)T;
                    }
                }
                tc_fence_before();
                mbar_arrive(acc_empty);
            }
        }
    } else if (warp >= 2) {
        // Bin without members: its sketch columns are zero (the reference's
        // untouched-bin zeroing, gw_ldscore.py:2017-2019).
        const int64_t i = i0 + (tid - 64);
        for (int v = 0; v < a.V; ++v) a.Y[((int64_t)k * a.V + v) * a.N_pad + i] = 0.0;
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
}

void launch_p1_weights4(const P1UWeights& w, const double* mean, const double* sdinv,
                        const double* Z, int64_t z_ld, cudaStream_t st) {
    if (w.K * w.V == 0) return;
    p1_weights4_kernel<<<(unsigned)(w.K * w.V), 256, 0, st>>>(w, mean, sdinv, Z, z_ld);
    count_launch();
}

size_t p1_umma_smem_bytes() { return (size_t)p1::kStages * p1::kStageBytes + 1024 + 256; }

void prepare_p1_umma() {
    cudaFuncSetAttribute(p1_umma_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)p1_umma_smem_bytes());
}

void launch_p1_umma(const CUtensorMap& tmW, const P1UArgs& a, int64_t N_pad, cudaStream_t st) {
    static bool attr = false;
    if (!attr) {
        cudaFuncSetAttribute(p1_umma_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)p1_umma_smem_bytes());
        attr = true;
    }
    dim3 grid((unsigned)(N_pad / p1::kBM), (unsigned)a.K);
    p1_umma_kernel<<<grid, p1::kThreads, p1_umma_smem_bytes(), st>>>(tmW, a);
    count_launch();
}

}  // namespace umma
}  // namespace lds
