// Dense FP64 work of the gwldcore boundary: the entries that take a dense
// genotype matrix instead of a BED file (phase1_compute_Xz_geno_chunk,
// phase2_accum_XtXz_geno, gwldcore.cpp:1896-1923 and :2624-2649), the
// covariate projections of genotype blocks (:1643-1657, :2376-2390), the
// mu22 moments of the residual-variance pass (:3421-3547) and the
// block corrections of binary annotations (:3569-3627).
//
// sm_100a has no FP64 kind of tcgen05.mma and its FP64 rate is the same on
// the CUDA cores, so the FP64 products here are a shared-memory tiled SIMT
// GEMM (64 x 64 output tile per CTA, 4 x 4 per thread).  The LD-score hot
// path (BED codes) stays on the int8 tensor-core kernels.
#include <cstdint>

#include "lds_internal.h"

namespace lds {

namespace {

constexpr int kBM = 64, kBN = 64, kBK = 16, kGemmThreads = 256;

__global__ void __launch_bounds__(kGemmThreads) dgemm_kernel(DGemmArgs a) {
    __shared__ double As[kBK][kBM + 1];
    __shared__ double Bs[kBK][kBN + 1];
    const int t = threadIdx.x;
    const int tx = t & 15, ty = t >> 4;
    const int64_t m0 = (int64_t)blockIdx.x * kBM, n0 = (int64_t)blockIdx.y * kBN;
    const bool a_mc = a.a_ms == 1 || a.a_kidx != nullptr;  // m contiguous in A
    const bool b_kc = a.b_ks == 1;                          // k contiguous in B
    double acc[4][4];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = 0.0;
    for (int64_t k0 = 0; k0 < a.K; k0 += kBK) {
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            const int e = t + r * kGemmThreads;
            const int mm = a_mc ? (e & 63) : (e >> 4);
            const int kk = a_mc ? (e >> 6) : (e & 15);
            const int64_t m = m0 + mm, k = k0 + kk;
            double v = 0.0;
            if (m < a.M && k < a.K) {
                const int64_t kc = a.a_kidx ? (int64_t)a.a_kidx[k] : k;
                v = a.A[m * a.a_ms + kc * a.a_ks];
                if (a.a_square) v *= v;
            }
            As[kk][mm] = v;
        }
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            const int e = t + r * kGemmThreads;
            const int kk = b_kc ? (e & 15) : (e >> 6);
            const int nn = b_kc ? (e >> 4) : (e & 63);
            const int64_t k = k0 + kk, n = n0 + nn;
            Bs[kk][nn] = (k < a.K && n < a.N) ? a.B[k * a.b_ks + n * a.b_ns] : 0.0;
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < kBK; ++kk) {
            double av[4], bv[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) av[i] = As[kk][tx + 16 * i];
#pragma unroll
            for (int j = 0; j < 4; ++j) bv[j] = Bs[kk][ty + 16 * j];
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) acc[i][j] = fma(av[i], bv[j], acc[i][j]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int64_t m = m0 + tx + 16 * i, n = n0 + ty + 16 * j;
            if (m >= a.M || n >= a.N) continue;
            double* c = a.C + m * a.c_ms + n * a.c_ns;
            const double v = a.alpha * acc[i][j];
            *c = a.beta == 0.0 ? v : v + a.beta * *c;
        }
}

// Per (SNP j, bin k): the guarded update of the phase-2 reduction
// (gwldcore.cpp:2520-2568) from the FP64 product panel W (L x K*V,
// column-major, column k*V + v).
__global__ void dense_p2_epilogue_kernel(const double* __restrict__ W, int64_t L, int K, int V,
                                         const double* __restrict__ ls, double* __restrict__ accum,
                                         double* __restrict__ mc,
                                         unsigned long long* __restrict__ guards,
                                         double extreme_warn, int drop_extreme) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= L * K) return;
    const int64_t j = t % L;
    const int k = (int)(t / L);
    double s2 = 0.0, s4 = 0.0;
    for (int v = 0; v < V; ++v) {
        const double w = W[((int64_t)k * V + v) * L + j];
        const double w2 = w * w;
        s2 += w2;
        s4 += w2 * w2;
    }
    const double scale = ls[j];
    double upd = s2 * scale;
    const double seg = (double)V;
    const bool nonfinite = !isfinite(upd);
    const bool extreme = !nonfinite && isfinite(extreme_warn) && seg > 0.0 && upd > extreme_warn * seg;
    if (nonfinite) atomicAdd(&guards[0], 1ULL);
    else if (extreme) atomicAdd(&guards[1], 1ULL);
    if (nonfinite || (extreme && drop_extreme)) return;
    if (upd < 0.0) upd = 0.0;
    accum[j * K + k] += upd;
    if (mc) mc[j * K + k] += s4 * scale * scale;
}

// Standardized genotypes of SNPs [j0, j0 + L) of the image as a dense
// column-major N x L block: x = s_j (g - mu_j) for observed calls, 0 else.
__global__ void decode_standardized_kernel(DevGeno g, int64_t j0, int64_t L,
                                           const double* __restrict__ mean,
                                           const double* __restrict__ sdinv,
                                           double* __restrict__ X, int64_t ldx) {
    const int64_t nq = (g.N + 3) / 4;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < nq * L;
         t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t j = t / nq, q = t - j * nq;
        const uint8_t b = g.codes[(j0 + j) * g.nbp + q];
        const double mu = mean[j0 + j], s = sdinv[j0 + j];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int64_t i = 4 * q + u;
            if (i >= g.N) break;
            const unsigned c = (b >> (2 * u)) & 3u;
            // 00 -> 0, 10 -> 1, 11 -> 2, 01 -> missing
            const double x = c == 1u ? 0.0 : s * ((c == 0u ? 0.0 : (c == 2u ? 1.0 : 2.0)) - mu);
            X[j * ldx + i] = x;
        }
    }
}

// ss[j] = sum_i X[i, j]^2, rows in order (one thread per column).
__global__ void col_sumsq_kernel(const double* __restrict__ X, int64_t N, int64_t ld, int64_t L,
                                 double* __restrict__ ss) {
    const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= L) return;
    const double* x = X + j * ld;
    double s = 0.0;
    for (int64_t i = 0; i < N; ++i) s += x[i] * x[i];
    ss[j] = s;
}

// compute_block_corrections_binary (gwldcore.cpp:3569-3627): one thread per
// (a, b); rows in order, so the sums match the reference's loop.
template <typename Tann>
__global__ void block_corrections_kernel(const double* __restrict__ meansq,
                                         const double* __restrict__ mu22,
                                         const Tann* __restrict__ annot, int64_t M, int B, double N,
                                         double d, double* __restrict__ R2, double* __restrict__ rho2,
                                         double* __restrict__ bias, double* __restrict__ delta) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (int64_t)B * B) return;
    const int a = (int)(t / B), b = (int)(t % B);
    double Ma = 0.0, Mb = 0.0, S = 0.0;
    for (int64_t i = 0; i < M; ++i) {
        const bool ia = annot[i * B + a] != (Tann)0;
        if (ia) {
            Ma += 1.0;
            S += meansq[i * B + b];
        }
        if (annot[i * B + b] != (Tann)0) Mb += 1.0;
    }
    double r2 = 0.0, rh = 0.0, bi = 0.0, de = 0.0;
    if (Ma > 0.0 && Mb > 0.0 && S != 0.0) {
        r2 = S / (Ma * Mb);
        const double mu = mu22[(int64_t)a * B + b];
        rh = (d * d * r2 - N * mu) / (N * (N - 1.0));
        bi = S - Ma * Mb * rh;
        de = mu - (1.0 + 2.0 * rh);
    }
    R2[t] = r2;
    rho2[t] = rh;
    bias[t] = bi;
    delta[t] = de;
}

// Column restandardization over N rows with ddof 0 (restandardize_cols_inplace,
// winldcore.cpp:215-267): x <- (x - mean) / sd, sd = 1 when the column has
// no spread.  One thread per column, rows in order.
__global__ void restandardize_cols_kernel(double* __restrict__ X, int64_t N, int64_t ld,
                                          int64_t L) {
    const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= L) return;
    double* col = X + j * ld;
    double sum = 0.0, sumsq = 0.0;
    for (int64_t i = 0; i < N; ++i) {
        const double x = col[i];
        sum += x;
        sumsq += x * x;
    }
    const double mean = sum / (double)N;
    double ss = sumsq - (sum * sum) / (double)N;
    if (ss < 0.0 && ss > -1e-12) ss = 0.0;
    double inv_sd = 1.0;
    if (ss > 0.0 && isfinite(ss)) {
        const double var = ss / (double)N;
        if (var > 0.0 && isfinite(var)) inv_sd = 1.0 / sqrt(var);
    }
    for (int64_t i = 0; i < N; ++i) col[i] = (col[i] - mean) * inv_sd;
}

// Windowed LD of a row chunk from its FP64 Gram panel S (rows x P,
// column-major, column i - p0): out[r, k] += sum_{i in [lo_r, hi_r)} f(r_ri)
// annot[i, k] with r = S / N and f = r^2 or the unbiased r^2 - (1 - r^2) / (d - 1).
// One warp per row; lane partial sums in shared memory, summed in lane order.
constexpr int kWinWarps = 4;
__global__ void __launch_bounds__(kWinWarps * 32)
    window_cov_epilogue_kernel(const double* __restrict__ S, int64_t rows, int64_t p0,
                               const int64_t* __restrict__ lo, const int64_t* __restrict__ hi,
                               const double* __restrict__ annot, int64_t annot_row0, int K,
                               double invN, double corr_den, double* __restrict__ out) {
    extern __shared__ double acc[];  // [warp][k][lane]
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t r = (int64_t)blockIdx.x * kWinWarps + w;
    if (r >= rows) return;
    double* a = acc + (int64_t)w * K * 32;
    for (int k = 0; k < K; ++k) a[k * 32 + lane] = 0.0;
    for (int64_t i = lo[r] + lane; i < hi[r]; i += 32) {
        const double rr = S[r + (i - p0) * rows] * invN;
        const double r2 = rr * rr;
        const double f = corr_den > 0.0 ? r2 - (1.0 - r2) * corr_den : r2;
        const double* an = annot + (i - annot_row0) * K;
        for (int k = 0; k < K; ++k) a[k * 32 + lane] += f * an[k];
    }
    __syncwarp();
    for (int k = lane; k < K; k += 32) {
        double t = 0.0;
        for (int l = 0; l < 32; ++l) t += a[k * 32 + l];
        out[r * K + k] += t;
    }
}

unsigned grid_for_n(int64_t n, int threads) {
    const int64_t b = (n + threads - 1) / threads;
    return (unsigned)(b < 148 * 32 ? (b > 0 ? b : 1) : 148 * 32);
}

}  // namespace

void launch_dgemm(const DGemmArgs& a, cudaStream_t st) {
    if (a.M <= 0 || a.N <= 0) return;
    if (a.K <= 0 && a.beta == 1.0) return;
    dim3 grid((unsigned)((a.M + kBM - 1) / kBM), (unsigned)((a.N + kBN - 1) / kBN));
    dgemm_kernel<<<grid, kGemmThreads, 0, st>>>(a);
    count_launch();
}

void launch_dense_p2_epilogue(const double* W, int64_t L, int K, int V, const double* ls,
                              double* accum, double* mc, unsigned long long* guards,
                              double extreme_warn, int drop_extreme, cudaStream_t st) {
    if (L * K == 0) return;
    dense_p2_epilogue_kernel<<<(unsigned)((L * K + 255) / 256), 256, 0, st>>>(
        W, L, K, V, ls, accum, mc, guards, extreme_warn, drop_extreme);
    count_launch();
}

void launch_decode_standardized(const DevGeno& g, int64_t j0, int64_t L, const double* mean,
                                const double* sdinv, double* X, int64_t ldx, cudaStream_t st) {
    if (L <= 0) return;
    decode_standardized_kernel<<<grid_for_n(((g.N + 3) / 4) * L, 256), 256, 0, st>>>(
        g, j0, L, mean, sdinv, X, ldx);
    count_launch();
}

void launch_col_sumsq(const double* X, int64_t N, int64_t ld, int64_t L, double* ss,
                      cudaStream_t st) {
    if (L <= 0) return;
    col_sumsq_kernel<<<(unsigned)((L + 127) / 128), 128, 0, st>>>(X, N, ld, L, ss);
    count_launch();
}

void launch_restandardize_cols(double* X, int64_t N, int64_t ld, int64_t L, cudaStream_t st) {
    if (L <= 0) return;
    restandardize_cols_kernel<<<(unsigned)((L + 127) / 128), 128, 0, st>>>(X, N, ld, L);
    count_launch();
}

int window_cov_max_bins() { return (int)(200 * 1024 / (kWinWarps * 32 * sizeof(double))); }

void launch_window_cov_epilogue(const double* S, int64_t rows, int64_t p0, const int64_t* lo,
                                const int64_t* hi, const double* annot, int64_t annot_row0, int K,
                                double invN, double corr_den, double* out, cudaStream_t st) {
    if (rows <= 0 || K <= 0) return;
    const size_t smem = (size_t)kWinWarps * K * 32 * sizeof(double);
    static std::atomic<unsigned long long> attr{0};
    once_per_device(attr, [] {
        cudaFuncSetAttribute(window_cov_epilogue_kernel,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    });
    window_cov_epilogue_kernel<<<(unsigned)((rows + kWinWarps - 1) / kWinWarps), kWinWarps * 32,
                                 smem, st>>>(S, rows, p0, lo, hi, annot, annot_row0, K, invN,
                                             corr_den, out);
    count_launch();
}

template <typename Tann>
void launch_block_corrections(const double* meansq, const double* mu22, const Tann* annot,
                              int64_t M, int B, double N, double d, double* R2, double* rho2,
                              double* bias, double* delta, cudaStream_t st) {
    if (B <= 0) return;
    const int64_t n = (int64_t)B * B;
    block_corrections_kernel<Tann><<<(unsigned)((n + 127) / 128), 128, 0, st>>>(
        meansq, mu22, annot, M, B, N, d, R2, rho2, bias, delta);
    count_launch();
}
template void launch_block_corrections<float>(const double*, const double*, const float*, int64_t,
                                              int, double, double, double*, double*, double*,
                                              double*, cudaStream_t);
template void launch_block_corrections<double>(const double*, const double*, const double*,
                                               int64_t, int, double, double, double*, double*,
                                               double*, double*, cudaStream_t);

}  // namespace lds
