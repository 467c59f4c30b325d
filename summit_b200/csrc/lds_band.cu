// Exact products of standardized genotypes between each SNP and its D nearest
// right-hand neighbours: xx[j][d] = x_j . x_{j+d}, d = 0..D, with
// x_ij = s_j (g_ij - mu_j) o_ij (the estimator's standardization; missing -> 0).
//
// The four integer sums behind it,
//   GG = sum_i g_ij g_ik, GO = sum_i g_ij o_ik, OG = sum_i o_ij g_ik, OO = sum_i o_ij o_ik,
// are bit counts over the packed 2-bit codes (PLINK: 00 -> g 0, 10 -> 1, 11 -> 2,
// 01 -> missing).  Each 32-bit code word (16 samples) becomes three planes with
// one 2-bit field per sample:
//   X  = a | b << 1   with a = (g >= 1), b = (g == 2)      (so popc(X & O2) = sum g o)
//   S  = b | a << 1   (X with its two bits swapped)
//   O2 = o | o << 1
// and, per word pair, GG = popc(Xj & Xk) + popc(Xj & Sk) (= sum (a_j + b_j)(a_k + b_k)),
// GO = popc(Xj & O2k), OG = popc(O2j & Xk), 2 OO = popc(O2j & O2k).  Integer and
// exact: this is HBM / ALU work, kept off the tensor cores.
//
// These products give the exact r^2 to nearby SNPs (the control variate's
// features and known means); they are the near-diagonal band of the X_w^T X_w
// that the exact windowed LD scores sum in full (compute_windowed_ld_chr_impl,
// winldcore.cpp:783).
#include <cstdint>

#include "lds_internal.h"

namespace lds {

namespace band {
constexpr int kTJ = 64;     // SNPs per CTA
constexpr int kWords = 64;  // 32-bit code words per row per chunk (1024 samples)
constexpr int kStride = kWords + 1;
}  // namespace band

__global__ void nn_band_counts_kernel(DevGeno g, int D, int32_t* __restrict__ counts) {
    using namespace band;
    extern __shared__ uint32_t planes[];
    const int rows = kTJ + D;
    uint32_t* PX = planes;
    uint32_t* PS = planes + rows * kStride;
    uint32_t* PO = planes + 2 * rows * kStride;
    const int64_t j0 = (int64_t)blockIdx.x * kTJ;
    const int jl = threadIdx.x % kTJ, d = threadIdx.x / kTJ;
    const int64_t nwords = g.nbp / 4;
    const uint32_t M5 = 0x55555555u;
    int gg = 0, go = 0, og = 0, oo2 = 0;
    for (int64_t w0 = 0; w0 < nwords; w0 += kWords) {
        __syncthreads();
        for (int idx = threadIdx.x; idx < rows * kWords; idx += blockDim.x) {
            const int r = idx / kWords, c = idx - (idx / kWords) * kWords;
            const int64_t row = j0 + r;
            uint32_t v = 0x55555555u;  // all missing
            if (row < g.M && w0 + c < nwords)
                v = *reinterpret_cast<const uint32_t*>(g.codes + row * g.nbp + (w0 + c) * 4);
            const uint32_t lo = v & M5, hi = (v >> 1) & M5;
            const uint32_t b = lo & hi;
            const uint32_t o = (~lo | hi) & M5;
            PX[r * kStride + c] = hi | (b << 1);
            PS[r * kStride + c] = b | (hi << 1);
            PO[r * kStride + c] = o | (o << 1);
        }
        __syncthreads();
        const uint32_t* xj = PX + jl * kStride;
        const uint32_t* oj = PO + jl * kStride;
        const uint32_t* xk = PX + (jl + d) * kStride;
        const uint32_t* sk = PS + (jl + d) * kStride;
        const uint32_t* ok = PO + (jl + d) * kStride;
#pragma unroll 8
        for (int c = 0; c < kWords; ++c) {
            const uint32_t a = xj[c], q = oj[c], x2 = xk[c];
            gg += __popc(a & x2) + __popc(a & sk[c]);
            go += __popc(a & ok[c]);
            og += __popc(q & x2);
            oo2 += __popc(q & ok[c]);
        }
    }
    const int64_t j = j0 + jl;
    if (j < g.M) {
        int32_t* o = counts + (j * (D + 1) + d) * 4;
        o[0] = gg;
        o[1] = go;
        o[2] = og;
        o[3] = oo2 >> 1;
    }
}

__global__ void nn_band_finish_kernel(int64_t M, int D, const int32_t* __restrict__ counts,
                                      const double* __restrict__ mean,
                                      const double* __restrict__ sdinv, double* __restrict__ xx) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= M * (D + 1)) return;
    const int64_t j = t / (D + 1);
    const int d = (int)(t - j * (D + 1));
    const int64_t k = j + d;
    double v = 0.0;
    if (k < M) {
        const int32_t* c = counts + t * 4;
        const double mj = mean[j], mk = mean[k];
        // sum_i (g_ij - mu_j) o_ij (g_ik - mu_k) o_ik from the exact integer sums
        const double s = (double)c[0] - mk * (double)c[1] - mj * (double)c[2] + mj * mk * (double)c[3];
        v = sdinv[j] * sdinv[k] * s;
    }
    xx[t] = v;
}

size_t nn_band_smem_bytes(int D) {
    return (size_t)3 * (band::kTJ + D) * band::kStride * sizeof(uint32_t);
}

void launch_nn_band(const DevGeno& g, int D, int32_t* counts, cudaStream_t st) {
    if (g.M == 0) return;
    const size_t smem = nn_band_smem_bytes(D);
    cudaFuncSetAttribute(nn_band_counts_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)smem);
    const unsigned grid = (unsigned)((g.M + band::kTJ - 1) / band::kTJ);
    nn_band_counts_kernel<<<grid, band::kTJ * (D + 1), smem, st>>>(g, D, counts);
    count_launch();
}

void launch_nn_band_finish(int64_t M, int D, const int32_t* counts, const double* mean,
                           const double* sdinv, double* xx, cudaStream_t st) {
    const int64_t n = M * (D + 1);
    if (n == 0) return;
    nn_band_finish_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(M, D, counts, mean, sdinv,
                                                                       xx);
    count_launch();
}

}  // namespace lds
