// SNP-block jackknife of normal equations and their rank-revealing symmetric
// solve, in FP64 on the device (inference/jackknife.py:109-214,
// context/fit.py:435-525, the replicate SE of inference/gxe.py:2052-2057).
//
// Per-SNP contributions t_j = [vec(A_j) (K*K, row-major), b_j (K)] are summed
// per contiguous SNP block (fixed order, deterministic), the delete-one systems
// are total - block, and every system is solved by the reference's spectral
// rule: symmetrize, eigendecompose (cyclic Jacobi, one CTA per system),
// retain |lambda| > max(100 eps scale, rtol max|lambda|), and form
// x = sum_retained v (v^T b) / (v^T A v).
#include <cstdint>

#include "lds_internal.h"

namespace lds {

namespace {

constexpr int kMaxK = 96;       // largest system (three K x (K+1) FP64 tiles in shared memory)
constexpr int kSolveThreads = 128;

__global__ void block_sums_kernel(const double* __restrict__ X, int64_t P,
                                  const int64_t* __restrict__ starts,
                                  const int64_t* __restrict__ ends, double* __restrict__ out) {
    const int64_t b = blockIdx.x;
    const int64_t c = (int64_t)blockIdx.y * blockDim.x + threadIdx.x;
    if (c >= P) return;
    double s = 0.0;
    for (int64_t j = starts[b]; j < ends[b]; ++j) s += X[j * P + c];
    out[b * P + c] = s;
}

// total[c] = sum_b blocks[b, c] in block order; sys[0] = total, sys[1 + b] = total - block b.
__global__ void delete_one_kernel(const double* __restrict__ blocks, int64_t B, int64_t P,
                                  double* __restrict__ sys) {
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= P) return;
    double tot = 0.0;
    for (int64_t b = 0; b < B; ++b) tot += blocks[b * P + c];
    sys[c] = tot;
    for (int64_t b = 0; b < B; ++b) sys[(1 + b) * P + c] = tot - blocks[b * P + c];
}

// One CTA per system (row-major K x K matrix then K rhs, stride K*K + K).
// status[s] bits: 1 asymmetric input, 2 rank deficient under require_full_rank,
// 4 non-finite input.
// Optional outputs (ex, any pointer may be null): eigenvectors (K x K per
// system, column p the eigenvector of the p-th smallest eigenvalue), the solve
// residual S x - b, the symmetry error max|A - A^T| and the retention
// tolerance.
__global__ void __launch_bounds__(kSolveThreads)
    sym_solve_kernel(const double* __restrict__ sys, int K, double rtol, int require_full_rank,
                     double* __restrict__ x, int* __restrict__ rank_out,
                     double* __restrict__ eig_out, int* __restrict__ status, SymSolveExtras ex) {
    extern __shared__ double sm[];
    const int ld = K + 1;
    auto A = [&](int i, int j) -> double& { return sm[i * ld + j]; };
    auto S = [&](int i, int j) -> double& { return sm[K * ld + i * ld + j]; };
    auto V = [&](int i, int j) -> double& { return sm[2 * K * ld + i * ld + j]; };
    __shared__ double bvec[kMaxK], lam[kMaxK], xs[kMaxK], red[kSolveThreads];
    __shared__ double rot[2];
    __shared__ int flag;
    const int s = blockIdx.x, t = threadIdx.x;
    const double* src = sys + (int64_t)s * (K * K + K);
    if (t == 0) flag = 0;
    if (t < K) {
        for (int j = 0; j < K; ++j) A(t, j) = src[t * K + j];
        bvec[t] = src[K * K + t];
    }
    __syncthreads();
    // scale and asymmetry (fit.py:440-443); symmetrize
    double mx = 0.0, asym = 0.0;
    bool finite = true;
    if (t < K)
        for (int j = 0; j < K; ++j) {
            finite = finite && isfinite(A(t, j));
            mx = fmax(mx, fabs(A(t, j)));
            asym = fmax(asym, fabs(A(t, j) - A(j, t)));
        }
    if (t < K && !isfinite(bvec[t])) finite = false;
    if (!finite) atomicOr(&flag, 4);
    red[t] = mx;
    __syncthreads();
    for (int o = kSolveThreads / 2; o; o >>= 1) {
        if (t < o) red[t] = fmax(red[t], red[t + o]);
        __syncthreads();
    }
    const double scale = fmax(red[0], 1.0);
    __syncthreads();
    red[t] = asym;
    __syncthreads();
    for (int o = kSolveThreads / 2; o; o >>= 1) {
        if (t < o) red[t] = fmax(red[t], red[t + o]);
        __syncthreads();
    }
    if (t == 0 && red[0] > 2.0e-10 * scale) atomicOr(&flag, 1);
    if (t == 0 && ex.asym) ex.asym[s] = red[0];
    if (t < K)
        for (int j = 0; j < K; ++j) {
            S(t, j) = 0.5 * (A(t, j) + A(j, t));
            V(t, j) = (t == j) ? 1.0 : 0.0;
        }
    __syncthreads();
    for (int j = 0; j < K; ++j) {
        if (t < K) A(t, j) = S(t, j);
    }
    __syncthreads();
    // cyclic Jacobi sweeps on A (a copy of S)
    for (int sweep = 0; sweep < 60; ++sweep) {
        // off-diagonal magnitude
        double off = 0.0;
        if (t < K)
            for (int j = 0; j < K; ++j)
                if (j != t) off = fmax(off, fabs(A(t, j)));
        red[t] = off;
        __syncthreads();
        for (int o = kSolveThreads / 2; o; o >>= 1) {
            if (t < o) red[t] = fmax(red[t], red[t + o]);
            __syncthreads();
        }
        const double offmax = red[0];
        __syncthreads();
        if (!(offmax > 1e-300) || offmax <= 1e-16 * scale) break;
        for (int p = 0; p < K - 1; ++p)
            for (int q = p + 1; q < K; ++q) {
                if (t == 0) {
                    const double apq = A(p, q);
                    double c = 1.0, sn = 0.0;
                    if (fabs(apq) > 1e-300) {
                        const double theta = (A(q, q) - A(p, p)) / (2.0 * apq);
                        const double tt = (theta >= 0.0 ? 1.0 : -1.0) /
                                          (fabs(theta) + sqrt(theta * theta + 1.0));
                        c = 1.0 / sqrt(tt * tt + 1.0);
                        sn = tt * c;
                    }
                    rot[0] = c;
                    rot[1] = sn;
                }
                __syncthreads();
                const double c = rot[0], sn = rot[1];
                if (sn != 0.0) {
                    // columns p, q of A and V
                    if (t < K) {
                        const double akp = A(t, p), akq = A(t, q);
                        A(t, p) = c * akp - sn * akq;
                        A(t, q) = sn * akp + c * akq;
                        const double vkp = V(t, p), vkq = V(t, q);
                        V(t, p) = c * vkp - sn * vkq;
                        V(t, q) = sn * vkp + c * vkq;
                    }
                    __syncthreads();
                    // rows p, q of A
                    if (t < K) {
                        const double apk = A(p, t), aqk = A(q, t);
                        A(p, t) = c * apk - sn * aqk;
                        A(q, t) = sn * apk + c * aqk;
                    }
                }
                __syncthreads();
            }
    }
    // eigenvalues, tolerance (fit.py:445-451)
    if (t < K) lam[t] = A(t, t);
    __syncthreads();
    red[t] = (t < K) ? fabs(lam[t]) : 0.0;
    __syncthreads();
    for (int o = kSolveThreads / 2; o; o >>= 1) {
        if (t < o) red[t] = fmax(red[t], red[t + o]);
        __syncthreads();
    }
    const double leading = red[0];
    const double abs_tol = 100.0 * 2.220446049250313e-16 * scale;
    const double tol = fmax(abs_tol, rtol * leading);
    if (t == 0 && ex.tol) ex.tol[s] = tol;
    __syncthreads();
    // retained Rayleigh quotients and the solution (fit.py:496-506)
    // proj[t] = v_t^T b / (v_t^T S v_t) for retained t
    double coef = 0.0;
    int keep = 0;
    if (t < K && fabs(lam[t]) > tol) {
        keep = 1;
        double vb = 0.0, vsv = 0.0;
        for (int i = 0; i < K; ++i) {
            vb += V(i, t) * bvec[i];
            double sv = 0.0;
            for (int j = 0; j < K; ++j) sv += S(i, j) * V(j, t);
            vsv += V(i, t) * sv;
        }
        coef = vb / vsv;
    }
    red[t] = coef;
    __syncthreads();
    if (t < K) {
        double xi = 0.0;
        for (int r = 0; r < K; ++r) xi += V(t, r) * red[r];
        x[(int64_t)s * K + t] = xi;
        xs[t] = xi;
    }
    __syncthreads();
    if (ex.resid && t < K) {
        double r = 0.0;
        for (int j = 0; j < K; ++j) r += S(t, j) * xs[j];
        ex.resid[(int64_t)s * K + t] = r - bvec[t];
    }
    red[t] = keep;
    __syncthreads();
    for (int o = kSolveThreads / 2; o; o >>= 1) {
        if (t < o) red[t] += red[t + o];
        __syncthreads();
    }
    if (t == 0) {
        const int rank = (int)red[0];
        rank_out[s] = rank;
        int f = flag;
        if (require_full_rank && rank != K) f |= 2;
        status[s] = f;
    }
    // eigenvalues ascending (for diagnostics): simple rank sort
    if (t < K) {
        int pos = 0;
        for (int j = 0; j < K; ++j)
            if (lam[j] < lam[t] || (lam[j] == lam[t] && j < t)) ++pos;
        eig_out[(int64_t)s * K + pos] = lam[t];
        if (ex.evec)
            for (int i = 0; i < K; ++i) ex.evec[(int64_t)s * K * K + (int64_t)i * K + pos] = V(i, t);
    }
}

// replicates (R x K): mean, se = sqrt((R-1)/R sum (r - mean)^2) and the
// covariance (R-1)/R sum (r - mean)(r - mean)^T (gxe.py:2052-2057).
__global__ void jackknife_stats_kernel(const double* __restrict__ reps, int64_t R, int K,
                                       double* __restrict__ mean, double* __restrict__ se,
                                       double* __restrict__ cov) {
    const int a = blockIdx.x, b = threadIdx.x;
    if (b >= K) return;
    double ma = 0.0, mb = 0.0;
    for (int64_t r = 0; r < R; ++r) {
        ma += reps[r * K + a];
        mb += reps[r * K + b];
    }
    ma /= (double)R;
    mb /= (double)R;
    double s = 0.0;
    for (int64_t r = 0; r < R; ++r) s += (reps[r * K + a] - ma) * (reps[r * K + b] - mb);
    const double c = ((double)R - 1.0) / (double)R * s;
    cov[(int64_t)a * K + b] = c;
    if (a == b) {
        mean[a] = ma;
        se[a] = sqrt(c);
    }
}

}  // namespace

int sym_solve_max_k() { return kMaxK; }

void launch_block_sums(const double* X, int64_t P, const int64_t* starts, const int64_t* ends,
                       int64_t B, double* out, cudaStream_t st) {
    if (B == 0 || P == 0) return;
    block_sums_kernel<<<dim3((unsigned)B, (unsigned)((P + 127) / 128)), 128, 0, st>>>(X, P, starts,
                                                                                    ends, out);
    count_launch();
}

void launch_delete_one(const double* blocks, int64_t B, int64_t P, double* sys, cudaStream_t st) {
    if (P == 0) return;
    delete_one_kernel<<<(unsigned)((P + 127) / 128), 128, 0, st>>>(blocks, B, P, sys);
    count_launch();
}

void launch_sym_solve(const double* sys, int64_t nsys, int K, double rtol, int require_full_rank,
                      double* x, int* rank, double* eig, int* status, cudaStream_t st,
                      const SymSolveExtras& ex) {
    if (nsys == 0) return;
    const size_t smem = (size_t)3 * K * (K + 1) * sizeof(double);
    static std::atomic<unsigned long long> attr{0};
    once_per_device(attr, [] {
        cudaFuncSetAttribute(sym_solve_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)((size_t)3 * kMaxK * (kMaxK + 1) * sizeof(double)));
    });
    sym_solve_kernel<<<(unsigned)nsys, kSolveThreads, smem, st>>>(sys, K, rtol, require_full_rank, x,
                                                                   rank, eig, status, ex);
    count_launch();
}

void launch_jackknife_stats(const double* reps, int64_t R, int K, double* mean, double* se,
                            double* cov, cudaStream_t st) {
    if (K == 0) return;
    jackknife_stats_kernel<<<(unsigned)K, kSolveThreads, 0, st>>>(reps, R, K, mean, se, cov);
    count_launch();
}

}  // namespace lds
