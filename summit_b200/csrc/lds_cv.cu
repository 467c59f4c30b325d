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

}  // namespace lds
