// Integrity check of the phase-2 tensor-core products (checksum vectors on the
// MMA outputs, verified on the host).
//
// The reference guards its GxE GEMMs with a Freivalds/ABFT checksum, (u^T A) B
// against u^T (A B) under a floating-point tolerance (gxeldcore.cpp:4674-4734).
// Here the products are exact integers, so the check is exact.  For SNP j of
// window w, with T_G(j, k, v) = sum_i g_ij y~_kv(i) and T_O(j, k, v) =
// sum_i o_ij y~_kv(i) the recombined digit products that the phase-2 epilogue
// turns into LD scores (y~ the sketch's 28-bit digit value), and h(k, v) an
// odd 64-bit weight per (bin, probe):
//   lhs_G[j] = sum_{k,v} h(k, v) T_G(j, k, v)       (phase-2 epilogue)
//   rhs_G[j] = sum_i g_ij u_w(i),  u_w(i) = sum_{k,v} h(k, v) y~_kv(i)
// both mod 2^64 (likewise O).  The right-hand side is formed here on the CUDA
// cores from the sketch digits and the packed genotype codes, independently
// of the tensor cores.  The two agree exactly unless a product is wrong; a
// single wrong product always shows, because h is odd.
#include <cstdint>

#include "lds_device.cuh"
#include "lds_internal.h"
#include "lds_umma.h"

namespace lds {

namespace {

constexpr int kUThreads = 256;     // 8 sample groups of 16 x 32 probe lanes
constexpr int kRhsChunk = 2048;    // samples of u staged in shared memory

// u[wl][i] = sum_{k < K, v < V} h(k, v0 + v) y~(super-bin wl*K + k, v, i) for
// the 128 samples of chunk blockIdx.x and window wl = blockIdx.y of the batch.
__global__ void __launch_bounds__(kUThreads)
    check_u_kernel(const int8_t* __restrict__ yq, int64_t yq_cols, int ncolp, int K, int V,
                   int v0, int64_t N_pad, unsigned long long* __restrict__ u) {
    __shared__ unsigned long long part[kUThreads / 8][128];
    const int t = threadIdx.x, sg = t & 7, lc = t >> 3;
    const int64_t kt = blockIdx.x, wl = blockIdx.y;
    unsigned long long acc[16];
#pragma unroll
    for (int s = 0; s < 16; ++s) acc[s] = 0ULL;
    for (int k = 0; k < K; ++k) {
        const int64_t col0 = (wl * K + k) * (int64_t)ncolp;
        for (int v = lc; v < V; v += kUThreads / 8) {
            const unsigned long long h = check_weight(k, v0 + v);
            int4 d[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int64_t col = col0 + 4 * v + q;
                d[q] = *reinterpret_cast<const int4*>(yq + (kt * yq_cols + col) * 128 +
                                                      ((sg ^ (int)(col & 7)) << 4));
            }
            const int* w0 = reinterpret_cast<const int*>(&d[0]);
            const int* w1 = reinterpret_cast<const int*>(&d[1]);
            const int* w2 = reinterpret_cast<const int*>(&d[2]);
            const int* w3 = reinterpret_cast<const int*>(&d[3]);
#pragma unroll
            for (int s = 0; s < 16; ++s) {
                const int sh = 8 * (s & 3);
                const int y = (int)(int8_t)(w0[s >> 2] >> sh) * (1 << 21) +
                              (int)(int8_t)(w1[s >> 2] >> sh) * (1 << 14) +
                              (int)(int8_t)(w2[s >> 2] >> sh) * (1 << 7) +
                              (int)(int8_t)(w3[s >> 2] >> sh);
                acc[s] += h * (unsigned long long)(long long)y;
            }
        }
    }
#pragma unroll
    for (int s = 0; s < 16; ++s) part[lc][sg * 16 + s] = acc[s];
    __syncthreads();
    if (t < 128) {
        unsigned long long tot = 0ULL;
        for (int l = 0; l < kUThreads / 8; ++l) tot += part[l][t];
        u[wl * N_pad + kt * 128 + t] = tot;
    }
}

// rhs[2j] += sum_i g_ij u_w(i), rhs[2j+1] += sum_i o_ij u_w(i) for the rows of
// tile blockIdx.x (one thread per SNP row; u staged in shared memory).
__global__ void __launch_bounds__(128)
    check_rhs_kernel(const uint8_t* __restrict__ codes, int64_t nbp, const int4* __restrict__ tiles,
                     int K, const unsigned long long* __restrict__ u, int64_t N_pad,
                     unsigned long long* __restrict__ rhs) {
    __shared__ unsigned long long us[kRhsChunk];
    const int4 tl = tiles[blockIdx.x];
    const int64_t j = (int64_t)tl.x + threadIdx.x;
    const bool live = j < tl.y;
    const unsigned long long* uw = u + (int64_t)(tl.z / K) * N_pad;
    const uint8_t* row = codes + (live ? j : (int64_t)tl.x) * nbp;
    unsigned long long sg = 0ULL, so = 0ULL;
    for (int64_t i0 = 0; i0 < N_pad; i0 += kRhsChunk) {
        const int n = N_pad - i0 < kRhsChunk ? (int)(N_pad - i0) : kRhsChunk;
        __syncthreads();
        for (int s = threadIdx.x; s < n; s += blockDim.x) us[s] = uw[i0 + s];
        __syncthreads();
        if (live) {
            for (int b = 0; b < n / 4; b += 16) {
                const uint4 p = *reinterpret_cast<const uint4*>(row + i0 / 4 + b);
                const uint32_t w[4] = {p.x, p.y, p.z, p.w};
#pragma unroll
                for (int q = 0; q < 4; ++q)
#pragma unroll
                    for (int c = 0; c < 16; ++c) {
                        const uint32_t code = (w[q] >> (2 * c)) & 3u;
                        const unsigned long long x = us[4 * (b + 4 * q) + c];
                        sg += (code >= 2u ? x : 0ULL) + (code == 3u ? x : 0ULL);
                        so += (code != 1u ? x : 0ULL);
                    }
            }
        }
    }
    if (live) {
        rhs[2 * j] += sg;
        rhs[2 * j + 1] += so;
    }
}

}  // namespace

void launch_check_u(const int8_t* yq, int64_t yq_cols, int ncolp, int K, int V, int v0,
                    int64_t n_windows, int64_t N_pad, unsigned long long* u, cudaStream_t st) {
    if (n_windows <= 0) return;
    check_u_kernel<<<dim3((unsigned)(N_pad / 128), (unsigned)n_windows), kUThreads, 0, st>>>(
        yq, yq_cols, ncolp, K, V, v0, N_pad, u);
    count_launch();
}

void launch_check_rhs(const uint8_t* codes, int64_t nbp, const int4* tiles, int64_t n_tiles, int K,
                      const unsigned long long* u, int64_t N_pad, unsigned long long* rhs,
                      cudaStream_t st) {
    if (n_tiles <= 0) return;
    check_rhs_kernel<<<(unsigned)n_tiles, 128, 0, st>>>(codes, nbp, tiles, K, u, N_pad, rhs);
    count_launch();
}

}  // namespace lds
