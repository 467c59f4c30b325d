// Device pieces of the generalized per-variant GxE two-pass estimator
// (ldscore/generalized_gxe_pass1.py, generalized_gxe_pass2.py): the global
// variant x probe Rademacher stream and the component-kernel diagonals.
// The genotype products of both passes run on the tensor-core kernels
// (lds_umma_p1.cu, lds_umma.cu) through lds_geno_source_product /
// lds_geno_target_product.
#include <algorithm>
#include <cstdint>

#include "lds_device.cuh"
#include "lds_internal.h"

namespace lds {

namespace {

// splitmix64 with the increment applied first (generalized_gxe_variant.py
// _splitmix64), and the addressable sign of global_probe_sign.
__device__ __forceinline__ uint64_t splitmix64_step(uint64_t v) {
    v += 0x9E3779B97F4A7C15ULL;
    v = (v ^ (v >> 30)) * 0xBF58476D1CE4E5B9ULL;
    v = (v ^ (v >> 27)) * 0x94D049BB133111EBULL;
    return v ^ (v >> 31);
}

// out[b * L + j] = sign(root, variant v0 + j, probe p0 + b) (column-major L x B).
__global__ void global_probes_kernel(uint64_t root_state, int64_t v0, int64_t L, int64_t p0,
                                     int64_t B, double* __restrict__ out) {
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= L * B) return;
    const int64_t j = idx % L, b = idx / L;
    uint64_t s = root_state;
    s ^= splitmix64_step((uint64_t)(v0 + j) + 0xD2B74407B1CE6E93ULL);
    s ^= splitmix64_step((uint64_t)(p0 + b) + 0xCA5A826395121157ULL);
    out[idx] = (splitmix64_step(s) >> 63) ? 1.0 : -1.0;
}

constexpr int kDiagThreads = 128;
constexpr int kDiagComp = 16;      // components per thread (registers)

// num[c * N + i] += sum_j a[j, k] kf(p) f_q(i, j) f_r(i, j) for the components
// c = k * P + p of this CTA's chunk, with the projected contextual features
// f_q(i, j) = phi_q(i) x_ij - sum_r F(i, r) coef[j, q, r] (pass-2 feature
// tiles, generalized_gxe_pass2.py:528-562) and x_ij the image's standardized
// genotype (0 on a missing call).  One thread per sample.
__global__ void __launch_bounds__(kDiagThreads)
    component_diag_kernel(const uint8_t* __restrict__ codes, int64_t nbp,
                          const double* __restrict__ mean, const double* __restrict__ sdinv,
                          int64_t j0, int64_t L, int64_t N, const double* __restrict__ annot,
                          int K, const double* __restrict__ basis, int Q,
                          const double* __restrict__ fixed, int R,
                          const double* __restrict__ coef, const int* __restrict__ pq,
                          const int* __restrict__ pr, const double* __restrict__ kf, int P,
                          double* __restrict__ num) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int c0 = blockIdx.y * kDiagComp;
    const int C = K * P;
    if (i >= N) return;
    double phi[kGenMaxQ], frow[kGenMaxR], acc[kDiagComp];
    for (int q = 0; q < Q; ++q) phi[q] = basis[(int64_t)q * N + i];
    for (int r = 0; r < R; ++r) frow[r] = fixed[(int64_t)r * N + i];
#pragma unroll
    for (int t = 0; t < kDiagComp; ++t) acc[t] = 0.0;
    const int shift = 2 * (int)(i & 3);
    for (int64_t jl = 0; jl < L; ++jl) {
        const int64_t j = j0 + jl;
        const uint32_t code = (codes[j * nbp + (i >> 2)] >> shift) & 3u;
        const double g = (double)((code >> 1) + (code == 3u));
        const double x = code == 1u ? 0.0 : sdinv[j] * (g - mean[j]);
        double f[kGenMaxQ];
        for (int q = 0; q < Q; ++q) {
            double v = phi[q] * x;
            const double* cj = coef + (jl * Q + q) * R;
            for (int r = 0; r < R; ++r) v -= frow[r] * cj[r];
            f[q] = v;
        }
#pragma unroll
        for (int t = 0; t < kDiagComp; ++t) {
            const int c = c0 + t;
            if (c >= C) break;
            const int k = c / P, p = c - k * P;
            const double a = annot[jl * K + k];
            if (a != 0.0) acc[t] += a * (kf[p] * f[pq[p]] * f[pr[p]]);
        }
    }
#pragma unroll
    for (int t = 0; t < kDiagComp; ++t) {
        const int c = c0 + t;
        if (c < C) num[(int64_t)c * N + i] += acc[t];
    }
}

// Pass-2 scores of one variant block, one CTA per variant row jl: the row's
// cross sketches cross[c] = s_j cs[c] (G^T y_c - mu_j O^T y_c) / rr from the
// exact raw digit products (column c = (k * B + b) * F + f of the
// right-hand side, raw row stride raw_ld), then
//   out[jl][tp][k * P + sp] = (1 / B) sum over the orientation terms (f1, f2)
//   of (tp, sp) of sum_b cross[(k B + b) F + f1] cross[(k B + b) F + f2]
// (generalized_gxe_pass2.py:600-676).
__global__ void gen_rows_kernel(const long long* __restrict__ raw_g,
                                const long long* __restrict__ raw_o, int64_t raw_ld,
                                const double* __restrict__ cs, const double* __restrict__ mean,
                                const double* __restrict__ sdinv, int64_t j0, double inv_rr, int K,
                                int B, int F, int P, const int* __restrict__ term_off,
                                const int* __restrict__ term_f1, const int* __restrict__ term_f2,
                                double* __restrict__ out) {
    extern __shared__ double cross[];
    const int64_t jl = blockIdx.x, j = j0 + jl;
    const int cols = K * B * F, C = K * P, nout = P * C;
    const double mu = mean[j], sd = sdinv[j];
    for (int c = threadIdx.x; c < cols; c += blockDim.x) {
        const int64_t q = jl * raw_ld + c;
        cross[c] = sd * cs[c] * ((double)raw_g[q] - mu * (double)raw_o[q]) * inv_rr;
    }
    __syncthreads();
    for (int o = threadIdx.x; o < nout; o += blockDim.x) {
        const int tp = o / C, c = o - tp * C, k = c / P, sp = c - k * P;
        double acc = 0.0;
        for (int t = term_off[tp * P + sp]; t < term_off[tp * P + sp + 1]; ++t) {
            const double* x1 = cross + (int64_t)k * B * F + term_f1[t];
            const double* x2 = cross + (int64_t)k * B * F + term_f2[t];
            double s = 0.0;
            for (int b = 0; b < B; ++b) s += x1[b * F] * x2[b * F];
            acc += s;
        }
        out[jl * nout + o] = acc / (double)B;
    }
}

// directed[c1][c2] += sum_jl a[j0 + jl][k1] rows[jl][p1][c2], c1 = k1 P + p1.
__global__ void gen_directed_kernel(const double* __restrict__ rows, int64_t L,
                                    const double* __restrict__ annot, int64_t j0, int K, int P,
                                    double* __restrict__ directed) {
    const int C = K * P;
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= C * C) return;
    const int c1 = idx / C, c2 = idx - c1 * C, k1 = c1 / P, p1 = c1 - k1 * P;
    double s = 0.0;
    for (int64_t jl = 0; jl < L; ++jl)
        s += annot[(j0 + jl) * K + k1] * rows[(jl * P + p1) * C + c2];
    directed[idx] += s;
}

// Pass 2's right-hand side from the contextual sources
// (GeneralizedGxEPass2Executor's family columns, generalized_gxe_pass2.py):
// column (k B + b) F + f = phi_t o sources[k, s][:, b] for family f = (t, s).
// S holds the sources as K Q B rows of N_pad samples, basis is N x Q
// row-major; Y gets one column of N_pad samples per (k, b, f), rows N and
// beyond left as they are (zero).
__global__ void gen_assemble_rhs_kernel(const double* __restrict__ S, int64_t Np,
                                        const double* __restrict__ basis, int Q,
                                        const int* __restrict__ fam_t,
                                        const int* __restrict__ fam_s, int B, int F, int64_t N,
                                        double* __restrict__ Y) {
    const int col = blockIdx.y;
    const int f = col % F, kb = col / F;
    const int b = kb % B, k = kb / B;
    const int t = fam_t[f], s = fam_s[f];
    const double* src = S + ((int64_t)(k * Q + s) * B + b) * Np;
    double* dst = Y + (int64_t)col * Np;
    for (int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; n < N;
         n += (int64_t)gridDim.x * blockDim.x)
        dst[n] = src[n] * basis[n * Q + t];
}

// Pass 1's projection of the contextual sources off the fixed effects
// (GeneralizedGxEPass1Executor, generalized_gxe_pass1.py:718-757), one CTA per
// (annotation k, basis coordinate q, probe b): with w = basis[:, q] o
// base[k, b], coef = fixed^T w, the row is p = w - fixed coef, written to out;
// leak = fixed^T p (R values) and p^T p are reduced in a fixed order for the
// host's leakage check.  base is K B rows of N samples, basis N x Q and fixed
// N x R row-major.
constexpr int kProjThreads = 256;

// Sums v[0..n) over the CTA (warp trees, then warps in order); the totals
// land in tot[0..n) for every thread.
template <int kMax>
__device__ __forceinline__ void block_sum(double (&v)[kMax], int n, double (*red)[kMax],
                                          double* tot) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int r = 0; r < kMax; ++r) {
        if (r >= n) break;
        double x = v[r];
        for (int o = 16; o; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
        if (lane == 0) red[w][r] = x;
    }
    __syncthreads();
    if (threadIdx.x < n) {
        double t = 0.0;
        for (int i = 0; i < (int)(blockDim.x >> 5); ++i) t += red[i][threadIdx.x];
        tot[threadIdx.x] = t;
    }
    __syncthreads();
}

__global__ void __launch_bounds__(kProjThreads)
    gen_project_kernel(const double* __restrict__ base, const double* __restrict__ basis, int Q,
                       const double* __restrict__ fixed, int R, int B, int64_t N,
                       double* __restrict__ out, double* __restrict__ leak,
                       double* __restrict__ pn2) {
    constexpr int kM = kGenMaxR + 1;
    __shared__ double red[kProjThreads / 32][kM];
    __shared__ double coef[kM];
    const int row = blockIdx.x;  // (k Q + q) B + b
    const int b = row % B, kq = row / B, q = kq % Q, k = kq / Q;
    const double* src = base + ((int64_t)k * B + b) * N;
    double* dst = out + (int64_t)row * N;
    double acc[kM];
#pragma unroll
    for (int r = 0; r < kM; ++r) acc[r] = 0.0;
    for (int64_t n = threadIdx.x; n < N; n += blockDim.x) {
        const double w = src[n] * basis[n * Q + q];
#pragma unroll
        for (int r = 0; r < kGenMaxR; ++r)
            if (r < R) acc[r] += w * fixed[n * R + r];
    }
    block_sum<kM>(acc, R, red, coef);
#pragma unroll
    for (int r = 0; r < kM; ++r) acc[r] = 0.0;  // leak[0..R), p^T p at R
    for (int64_t n = threadIdx.x; n < N; n += blockDim.x) {
        const double w = src[n] * basis[n * Q + q];
        double fc = 0.0;
#pragma unroll
        for (int r = 0; r < kGenMaxR; ++r)
            if (r < R) fc += fixed[n * R + r] * coef[r];
        const double p = w - fc;
        dst[n] = p;
#pragma unroll
        for (int r = 0; r < kGenMaxR; ++r)
            if (r < R) acc[r] += p * fixed[n * R + r];
        acc[R < kGenMaxR ? R : kGenMaxR] += p * p;
    }
    block_sum<kM>(acc, R + 1, red, coef);
    if (threadIdx.x < R) leak[(int64_t)row * R + threadIdx.x] = coef[threadIdx.x];
    if (threadIdx.x == 0) pn2[row] = coef[R];
}

}  // namespace

void launch_gen_project(const double* base, const double* basis, int Q, const double* fixed,
                        int R, int K, int B, int64_t N, double* out, double* leak, double* pn2,
                        cudaStream_t st) {
    const int rows = K * Q * B;
    if (rows <= 0 || N <= 0) return;
    gen_project_kernel<<<(unsigned)rows, kProjThreads, 0, st>>>(base, basis, Q, fixed, R, B, N, out,
                                                               leak, pn2);
    count_launch();
}

void launch_gen_assemble_rhs(const double* S, int64_t Np, const double* basis, int Q,
                             const int* fam_t, const int* fam_s, int K, int B, int F, int64_t N,
                             double* Y, cudaStream_t st) {
    const int cols = K * B * F;
    if (cols <= 0 || N <= 0) return;
    const unsigned bx = (unsigned)std::min<int64_t>((N + 255) / 256, 64);
    gen_assemble_rhs_kernel<<<dim3(bx, (unsigned)cols), 256, 0, st>>>(S, Np, basis, Q, fam_t, fam_s,
                                                                     B, F, N, Y);
    count_launch();
}

size_t gen_rows_smem_bytes(int cols) { return (size_t)cols * sizeof(double); }

void launch_gen_rows(const long long* raw_g, const long long* raw_o, int64_t raw_ld,
                     const double* cs, const double* mean, const double* sdinv, int64_t j0,
                     int64_t L, double inv_rr, int K, int B, int F, int P, const int* term_off,
                     const int* term_f1, const int* term_f2, double* out, cudaStream_t st) {
    if (L <= 0) return;
    const size_t smem = gen_rows_smem_bytes(K * B * F);
    static std::atomic<unsigned long long> attr{0};
    once_per_device(attr, [] {
        cudaFuncSetAttribute(gen_rows_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)kGenRowsMaxSmem);
    });
    gen_rows_kernel<<<(unsigned)L, 256, smem, st>>>(raw_g, raw_o, raw_ld, cs, mean, sdinv, j0,
                                                     inv_rr, K, B, F, P, term_off, term_f1,
                                                     term_f2, out);
    count_launch();
}

void launch_gen_directed(const double* rows, int64_t L, const double* annot, int64_t j0, int K,
                         int P, double* directed, cudaStream_t st) {
    const int C = K * P;
    if (L <= 0 || C <= 0) return;
    gen_directed_kernel<<<(unsigned)((C * C + 255) / 256), 256, 0, st>>>(rows, L, annot, j0, K, P,
                                                                          directed);
    count_launch();
}

void launch_global_probes(uint64_t root_state, int64_t v0, int64_t L, int64_t p0, int64_t B,
                          double* out, cudaStream_t st) {
    const int64_t n = L * B;
    if (n <= 0) return;
    global_probes_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(root_state, v0, L, p0, B,
                                                                      out);
    count_launch();
}

void launch_component_diag(const uint8_t* codes, int64_t nbp, const double* mean,
                           const double* sdinv, int64_t j0, int64_t L, int64_t N,
                           const double* annot, int K, const double* basis, int Q,
                           const double* fixed, int R, const double* coef, const int* pq,
                           const int* pr, const double* kf, int P, double* num, cudaStream_t st) {
    const int C = K * P;
    if (N <= 0 || L <= 0 || C <= 0) return;
    dim3 grid((unsigned)((N + kDiagThreads - 1) / kDiagThreads),
              (unsigned)((C + kDiagComp - 1) / kDiagComp));
    component_diag_kernel<<<grid, kDiagThreads, 0, st>>>(codes, nbp, mean, sdinv, j0, L, N, annot,
                                                         K, basis, Q, fixed, R, coef, pq, pr, kf,
                                                         P, num);
    count_launch();
}

}  // namespace lds
