// Near-field control variate of the windowed stochastic LD scores.
//
// The plain estimator of SNP j's LD score in bin k uses, per probe v,
//   u_jv = sum_i c_ji sc_ik z_iv,   c_ji = x_j . x_i * sqrt(left_scale_j),
// over the SNPs i of j's window (E[u^2] = sum_i c_ji^2 sc_ik^2 is the score).
// Split the sum into the near field (|i - j| <= D, same window) a_jv and the rest
// f_jv.  a uses the same probes as u, and its mean is known exactly from the
// exact neighbour products:  E[a^2] = sum_near c_ji^2 sc_ik^2.  With independent
// probe entries, a and f are independent, so Cov(u^2, a^2) = Var(a^2) and the
// control variate u^2 - a^2 + E[a^2] keeps the mean with coefficient 1 (the
// optimal one) and removes the near field's share of the variance.
//
// cv_near_kernel accumulates C_jk += sum_v a_jkv^2 for one V-tile of probes and
// (first tile) writes mu_jk = E[a_jk^2].  Thread per (j, k).
#include <cstdint>

#include "lds_internal.h"

namespace lds {

template <int D>
__global__ void cv_near_kernel(CvNearArgs a) {
    const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int k = blockIdx.y;
    if (j >= a.M) return;
    const int wj = a.win_of[j];
    const double sj = a.sqrt_ls[j];
    double w[2 * D + 1];
    double mu = 0.0;
#pragma unroll
    for (int t = 0; t < 2 * D + 1; ++t) {
        const int64_t i = j + t - D;
        double c = 0.0;
        if (i >= 0 && i < a.M && a.win_of[i] == wj) {
            // x_j . x_i is stored once per unordered pair, at the lower index.
            const double xx = t >= D ? a.xx[j * (D + 1) + (t - D)] : a.xx[i * (D + 1) + (D - t)];
            c = xx * sj * a.annot[i * a.K + k];
        }
        w[t] = c;
        mu += c * c;
    }
    double acc = 0.0, acc2 = 0.0;
    for (int v = 0; v < a.V; ++v) {
        const double* z = a.z + (int64_t)v * a.z_ld;
        double s = 0.0;
#pragma unroll
        for (int t = 0; t < 2 * D + 1; ++t)
            if (w[t] != 0.0) s += w[t] * z[j + t - D];
        if (a.C2 && v >= a.split_v) acc2 += s * s;
        else acc += s * s;
    }
    a.C[j * a.K + k] += acc;
    if (a.C2) a.C2[j * a.K + k] += acc2;
    if (a.mu) a.mu[j * a.K + k] = mu;
}

void launch_cv_near(const CvNearArgs& a, int D, cudaStream_t st) {
    if (a.M == 0 || a.K == 0) return;
    dim3 grid((unsigned)((a.M + 127) / 128), (unsigned)a.K);
    switch (D) {
        case 4: cv_near_kernel<4><<<grid, 128, 0, st>>>(a); break;
        case 8: cv_near_kernel<8><<<grid, 128, 0, st>>>(a); break;
        case 15: cv_near_kernel<15><<<grid, 128, 0, st>>>(a); break;
        default: return;
    }
    count_launch();
}

// Finalize of a windowed estimate: meansq = sum of the probe slices and
// ld = meansq / nvecs - Mkw[window(j), k] / nd (gw_ldscore.py:2197, :2220-2222
// applied per window).
__global__ void win_finalize_kernel(const double* __restrict__ acc, int slices, int64_t MK, int K,
                                    double nvecs, double nd, const int32_t* __restrict__ win_of,
                                    const double* __restrict__ mkw, double* __restrict__ ld,
                                    double* __restrict__ meansq) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= MK) return;
    double s = acc[t];
    for (int q = 1; q < slices; ++q) s += acc[(int64_t)q * MK + t];
    const int64_t j = t / K;
    const int k = (int)(t - j * K);
    meansq[t] = s;
    ld[t] = s / nvecs - mkw[(int64_t)win_of[j] * K + k] / nd;
}

void launch_win_finalize(const double* acc, int slices, int64_t M, int K, double nvecs, double nd,
                         const int32_t* win_of, const double* mkw, double* ld, double* meansq,
                         cudaStream_t st) {
    const int64_t MK = M * K;
    if (MK == 0) return;
    win_finalize_kernel<<<(unsigned)((MK + 255) / 256), 256, 0, st>>>(acc, slices, MK, K, nvecs, nd,
                                                                      win_of, mkw, ld, meansq);
    count_launch();
}

}  // namespace lds
