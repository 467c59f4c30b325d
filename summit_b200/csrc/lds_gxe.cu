// SUMMIT-GxE directional LD-score products (MultiEnvironmentKernel,
// gxeldcore.cpp:10281-12557) on the B200: the elementwise and reduction
// kernels around the two tensor-core products, which reuse the phase-1 and
// phase-2 kernels.
//
// Source panel (source_block, gxeldcore.cpp:11008-11240).  Column
// c = ((e 2 + h) K + k) B + b of the panel holds
//   h = 0 (additive):     X [sqrt(a_k) o z_b o s_x,e]
//   h = 1 (interaction):  phi_e o (X [sqrt(a_k) o z_b o s_w,e])
// where X are the standardized genotypes of the block.  The product runs on
// p1_umma_kernel with one "super-bin" per (e, h, k); gxe_source_finalize
// applies phi_e and adds into the panel.
//
// Projection (project_sources, :11583-11729): P <- P - U (U^T P) with the
// common basis U, then per column the environment direction and the mean:
// P <- P - d_e (d_e^T P) - mean(P), both coefficients taken from the same
// values; the leakage onto the environment's fixed-effect basis must stay
// below 1e-9.  FP64 column reductions in a fixed order.
//
// Target (target_score_block, :11731-11936): out = X^T [P, w o P] on
// p2_umma_kernel with one "bin" per (pair half p, e, h, k) giving
// S = sum_b out^2 per SNP; gxe_target_finalize scales by s^2 / (N - rank_e)^2
// (s = s_x,e for p = 0, s_w,e for p = 1) into accum_{xx,xw,wx,ww}
// [(e total + block_start + j) K + k] (accumulator 2p + h).
//
// Probes (numpy_philox_rademacher_block, :10002-10113): NumPy's
// Philox4x64-10 stream per probe column (key from the caller), one 32-bit
// word per 4 rows, the high bit of each byte giving the sign; every row is
// independent given its counter, so the kernel is one thread per element.
#include <algorithm>
#include <cstdint>

#include "lds_internal.h"

namespace lds {

namespace {

__global__ void gxe_source_finalize_kernel(const double* __restrict__ Y, int64_t N, int64_t N_pad,
                                           int64_t C, int cols_half, const double* __restrict__ env,
                                           int64_t env_ld, int env_start, double* __restrict__ target,
                                           int64_t t_ld) {
    const int64_t n = N * C;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n;
         t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t c = t / N, i = t - c * N;
        const int64_t e = c / (2 * cols_half);
        const bool inter = ((c / cols_half) & 1) != 0;
        double v = Y[c * N_pad + i];
        if (inter) v *= env[(env_start + e) * env_ld + i];
        target[c * t_ld + i] += v;
    }
}

// out[c nb + a] = sum_i basis[a b_ld + i] panel[c p_ld + i] (basis may be null:
// a single all-ones column, i.e. the column sum).  One CTA per column, fixed
// reduction order.
constexpr int kDotThreads = 256;
constexpr int kMaxBasis = 32;

__global__ void __launch_bounds__(kDotThreads)
    col_dots_kernel(const double* __restrict__ panel, int64_t p_ld, int64_t N,
                    const double* __restrict__ basis, int64_t b_ld, int nb, int squares,
                    double* __restrict__ out) {
    __shared__ double red[kDotThreads / 32][kMaxBasis];
    const int64_t c = blockIdx.x;
    const double* v = panel + c * p_ld;
    double acc[kMaxBasis];
#pragma unroll
    for (int a = 0; a < kMaxBasis; ++a) acc[a] = 0.0;
    for (int64_t i = threadIdx.x; i < N; i += kDotThreads) {
        const double x = v[i];
        if (squares) {
            acc[0] += x * x;
            continue;
        }
#pragma unroll
        for (int a = 0; a < kMaxBasis; ++a)
            if (a < nb) acc[a] += (basis ? basis[a * b_ld + i] : 1.0) * x;
    }
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int nr = squares ? 1 : nb;
#pragma unroll
    for (int a = 0; a < kMaxBasis; ++a) {
        if (a >= nr) break;
        double s = acc[a];
        for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0) red[w][a] = s;
    }
    __syncthreads();
    if (threadIdx.x < nr) {
        double s = 0.0;
        for (int q = 0; q < kDotThreads / 32; ++q) s += red[q][threadIdx.x];
        out[c * nr + threadIdx.x] = s;
    }
}

// panel[c ld + i] -= sum_a basis[a b_ld + i] coef[c nb + a] scale_a, where a
// null basis column means all ones and scale multiplies coefficient a.
__global__ void sub_lowrank_kernel(double* __restrict__ panel, int64_t ld, int64_t N, int64_t C,
                                   const double* __restrict__ basis, int64_t b_ld, int nb,
                                   const double* __restrict__ coef, int ones_last, double last_scale) {
    const int64_t n = N * C;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n;
         t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t c = t / N, i = t - c * N;
        double s = 0.0;
        for (int a = 0; a < nb; ++a) {
            const bool ones = ones_last && a == nb - 1;
            const double b = ones ? 1.0 : basis[a * b_ld + i];
            s += b * (ones ? coef[c * nb + a] * last_scale : coef[c * nb + a]);
        }
        panel[c * ld + i] -= s;
    }
}

// Ypair[c N_pad + i] = S[c s_ld + i], Ypair[(C + c) N_pad + i] = w[g(c)] o S, rows
// N..N_pad zero; g(c) = c / cols_per_group.
__global__ void gxe_pair_kernel(const double* __restrict__ S, int64_t s_ld, int64_t N,
                                int64_t N_pad, int64_t C, int64_t cols_per_group,
                                const double* __restrict__ w, int64_t w_ld, int w_first,
                                double* __restrict__ Ypair) {
    const int64_t n = N_pad * C;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n;
         t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t c = t / N_pad, i = t - c * N_pad;
        double v = 0.0, vw = 0.0;
        if (i < N) {
            v = S[c * s_ld + i];
            vw = w[(w_first + c / cols_per_group) * w_ld + i] * v;
        }
        Ypair[c * N_pad + i] = v;
        Ypair[(C + c) * N_pad + i] = vw;
    }
}

__global__ void gxe_target_finalize_kernel(const double* __restrict__ S, int64_t L, int Kp, int K,
                                           int T, const double* __restrict__ sx,
                                           const double* __restrict__ sw, int64_t s_ld,
                                           const int32_t* __restrict__ ranks, int64_t N,
                                           int env_start, int64_t total, int64_t block_start,
                                           double* a0, double* a1, double* a2, double* a3) {
    const int64_t n = L * Kp;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n;
         t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t j = t / Kp;
        const int g = (int)(t - j * Kp);
        // g = ((p T + e) 2 + h) K + k
        const int k = g % K;
        const int h = (g / K) & 1;
        const int pe = g / (2 * K);
        const int e = pe % T, p = pe / T;
        const double s = p == 0 ? sx[(int64_t)e * s_ld + j] : sw[(int64_t)e * s_ld + j];
        const double df = (double)(N - ranks[env_start + e]);
        const double val = S[j * Kp + g] * (s * s) * (1.0 / (df * df));
        double* acc = (p == 0) ? (h == 0 ? a0 : a1) : (h == 0 ? a2 : a3);
        acc[((int64_t)(env_start + e) * total + block_start + j) * K + k] += val;
    }
}

__global__ void scale_kernel(double* __restrict__ x, int64_t n, double s) {
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n;
         t += (int64_t)gridDim.x * blockDim.x)
        x[t] *= s;
}

// Input checks of source/target (gxeldcore.cpp:11131-11158, :11817-11829):
// flag |= 1 for a non-finite probe, 2 for a non-finite or <= 0 scale, 4 for a
// negative or non-finite annotation (when given raw).
__global__ void gxe_check_kernel(const double* __restrict__ probes, int64_t np,
                                 const double* __restrict__ sx, const double* __restrict__ sw,
                                 int64_t ns, const double* __restrict__ annot, int64_t na,
                                 unsigned* flag) {
    unsigned f = 0;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < np;
         t += (int64_t)gridDim.x * blockDim.x)
        if (!isfinite(probes[t])) f |= 1u;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < ns;
         t += (int64_t)gridDim.x * blockDim.x) {
        const double a = sx[t], b = sw[t];
        if (!isfinite(a) || !isfinite(b) || a <= 0.0 || b <= 0.0) f |= 2u;
    }
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < na;
         t += (int64_t)gridDim.x * blockDim.x)
        if (!isfinite(annot[t]) || annot[t] < 0.0) f |= 4u;
    if (f) atomicOr(flag, f);
}

// ---- NumPy Philox4x64-10 (the published Random123 algorithm, NumPy's
// counter/buffer conventions as gxeldcore.cpp:10011-10068 uses them) ----
__device__ __forceinline__ void philox4x64_10(uint64_t c[4], uint64_t k0, uint64_t k1) {
    const uint64_t M0 = 0xD2E7470EE14C6C93ULL, M1 = 0xCA5A826395121157ULL;
    const uint64_t W0 = 0x9E3779B97F4A7C15ULL, W1 = 0xBB67AE8584CAA73BULL;
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        const uint64_t lo0 = M0 * c[0], hi0 = __umul64hi(M0, c[0]);
        const uint64_t lo1 = M1 * c[2], hi1 = __umul64hi(M1, c[2]);
        const uint64_t n0 = hi1 ^ c[1] ^ k0, n2 = hi0 ^ c[3] ^ k1;
        c[0] = n0;
        c[1] = lo1;
        c[2] = n2;
        c[3] = lo0;
        k0 += W0;
        k1 += W1;
    }
}

// Row r of column p: 32-bit word w = r / 4 of the stream (low half of 64-bit
// output w/2 first), 64-bit output q = w / 2 is word q % 4 of Philox block
// q / 4, generated from counter q / 4 + 1 (the counter is bumped before each
// block); the sign is the high bit of byte r % 4.
__global__ void philox_rademacher_kernel(const uint64_t* __restrict__ keys, int64_t P, int64_t rows,
                                         double* __restrict__ out) {
    const int64_t n = P * rows;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n;
         t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t p = t / rows, r = t - p * rows;
        const uint64_t w = (uint64_t)r >> 2, q = w >> 1, blk = q >> 2;
        uint64_t c[4] = {blk + 1, 0, 0, 0};
        if (c[0] == 0) c[1] = 1;  // 256-bit counter carry (blk + 1 overflowed)
        philox4x64_10(c, keys[2 * p], keys[2 * p + 1]);
        const int qi = (int)(q & 3);
        const uint64_t v = qi == 0 ? c[0] : qi == 1 ? c[1] : qi == 2 ? c[2] : c[3];
        const uint32_t word = (w & 1) ? (uint32_t)(v >> 32) : (uint32_t)v;
        const uint32_t byte = (word >> (8 * (r & 3))) & 0xFFu;
        out[p * rows + r] = (byte & 0x80u) ? 1.0 : -1.0;
    }
}

unsigned grid_for(int64_t n) {
    const int64_t b = (n + 255) / 256;
    return (unsigned)(b < 148 * 64 ? (b > 0 ? b : 1) : 148 * 64);
}

}  // namespace

void launch_gxe_source_finalize(const double* Y, int64_t N, int64_t N_pad, int64_t C, int cols_half,
                                const double* env, int64_t env_ld, int env_start, double* target,
                                int64_t t_ld, cudaStream_t st) {
    if (N * C == 0) return;
    gxe_source_finalize_kernel<<<grid_for(N * C), 256, 0, st>>>(Y, N, N_pad, C, cols_half, env,
                                                                 env_ld, env_start, target, t_ld);
    count_launch();
}

void launch_col_dots(const double* panel, int64_t p_ld, int64_t N, int64_t C, const double* basis,
                     int64_t b_ld, int nb, int squares, double* out, cudaStream_t st) {
    if (C == 0) return;
    col_dots_kernel<<<(unsigned)C, kDotThreads, 0, st>>>(panel, p_ld, N, basis, b_ld, nb, squares, out);
    count_launch();
}

int col_dots_max_basis() { return kMaxBasis; }

void launch_sub_lowrank(double* panel, int64_t ld, int64_t N, int64_t C, const double* basis,
                        int64_t b_ld, int nb, const double* coef, int ones_last, double last_scale,
                        cudaStream_t st) {
    if (N * C == 0 || nb == 0) return;
    sub_lowrank_kernel<<<grid_for(N * C), 256, 0, st>>>(panel, ld, N, C, basis, b_ld, nb, coef,
                                                         ones_last, last_scale);
    count_launch();
}

void launch_gxe_pair(const double* S, int64_t s_ld, int64_t N, int64_t N_pad, int64_t C,
                     int64_t cols_per_group, const double* w, int64_t w_ld, int w_first,
                     double* Ypair, cudaStream_t st) {
    if (N_pad * C == 0) return;
    gxe_pair_kernel<<<grid_for(N_pad * C), 256, 0, st>>>(S, s_ld, N, N_pad, C, cols_per_group, w,
                                                          w_ld, w_first, Ypair);
    count_launch();
}

void launch_gxe_target_finalize(const double* S, int64_t L, int Kp, int K, int T, const double* sx,
                                const double* sw, int64_t s_ld, const int32_t* ranks, int64_t N,
                                int env_start, int64_t total, int64_t block_start, double* a0,
                                double* a1, double* a2, double* a3, cudaStream_t st) {
    if (L * Kp == 0) return;
    gxe_target_finalize_kernel<<<grid_for(L * Kp), 256, 0, st>>>(
        S, L, Kp, K, T, sx, sw, s_ld, ranks, N, env_start, total, block_start, a0, a1, a2, a3);
    count_launch();
}

void launch_scale(double* x, int64_t n, double s, cudaStream_t st) {
    if (n == 0) return;
    scale_kernel<<<grid_for(n), 256, 0, st>>>(x, n, s);
    count_launch();
}

void launch_gxe_check(const double* probes, int64_t np, const double* sx, const double* sw,
                      int64_t ns, const double* annot, int64_t na, unsigned* flag, cudaStream_t st) {
    gxe_check_kernel<<<grid_for(std::max(std::max(np, ns), na)), 256, 0, st>>>(probes, np, sx, sw, ns,
                                                                              annot, na, flag);
    count_launch();
}

void launch_philox_rademacher(const uint64_t* keys, int64_t P, int64_t rows, double* out,
                              cudaStream_t st) {
    if (P * rows == 0) return;
    philox_rademacher_kernel<<<grid_for(P * rows), 256, 0, st>>>(keys, P, rows, out);
    count_launch();
}

}  // namespace lds
