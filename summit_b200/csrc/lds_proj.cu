// Sketch-panel utilities of the gwldcore boundary: column sums of a row-major
// sketch (compute_col_sums_rowmajor_core, gwldcore.cpp:710-726), layout
// conversions for the row-major entry points, and in-place standardization of
// dense dosages (standardize_dosage_inplace_impl, :1511-1580).
//
// Column sums and dosage statistics run one thread per column over the rows
// in order, the reference's summation order, so they match it bit for bit.
#include <cstdint>

#include "lds_internal.h"

namespace lds {

namespace {

template <typename T>
__global__ void col_sums_rowmajor_kernel(const T* __restrict__ X, int64_t N, int64_t Q,
                                         double* __restrict__ out) {
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= Q) return;
    double acc = 0.0;
    for (int64_t i = 0; i < N; ++i) acc += (double)X[i * Q + c];
    out[c] = acc;
}

template <typename T>
__global__ void rowmajor_to_colmajor_kernel(const T* __restrict__ in, int64_t N, int64_t Q,
                                            double* __restrict__ out) {
    const int64_t n = N * Q;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n;
         t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = t / Q, c = t - i * Q;
        out[c * N + i] = (double)in[t];
    }
}

template <typename T>
__global__ void colmajor_to_rowmajor_kernel(const double* __restrict__ in, int64_t N, int64_t Q,
                                            T* __restrict__ out) {
    const int64_t n = N * Q;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n;
         t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = t / Q, c = t - i * Q;
        out[t] = (T)in[c * N + i];
    }
}

template <typename T>
__global__ void convert_kernel(const T* __restrict__ in, int64_t n, double* __restrict__ out) {
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n;
         t += (int64_t)gridDim.x * blockDim.x)
        out[t] = (double)in[t];
}

template <typename T>
__global__ void convert_back_kernel(const double* __restrict__ in, int64_t n, T* __restrict__ out) {
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n;
         t += (int64_t)gridDim.x * blockDim.x)
        out[t] = (T)in[t];
}

// One thread per column: observed mean and inverse sd (nobs - ddof), then
// x <- (x - mu) inv_sd for valid calls in [0, 2] and 0 for missing or invalid
// ones; counts[0] += missing calls, counts[1] += invalid calls.
template <typename T>
__global__ void standardize_dosage_kernel(T* __restrict__ G, int64_t N, int64_t L, int ddof,
                                          double missing, unsigned long long* counts) {
    const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= L) return;
    T* col = G + j * N;
    long long nobs = 0, nmiss = 0, ninv = 0;
    double sum = 0.0, sumsq = 0.0;
    for (int64_t i = 0; i < N; ++i) {
        const double x = (double)col[i];
        if (x == missing) {
            ++nmiss;
            continue;
        }
        if (!isfinite(x) || x < 0.0 || x > 2.0) {
            ++ninv;
            continue;
        }
        ++nobs;
        sum += x;
        sumsq += x * x;
    }
    const double mu = nobs > 0 ? sum / (double)nobs : 0.0;
    double m2 = nobs > 0 ? sumsq - sum * sum / (double)nobs : 0.0;
    if (m2 < 0.0 && m2 > -1e-12) m2 = 0.0;
    const long long denom = nobs - (long long)ddof;
    double inv_sd = 1.0;
    if (denom > 0 && m2 > 0.0) {
        const double var = m2 / (double)denom;
        if (isfinite(var) && var > 0.0) inv_sd = 1.0 / sqrt(var);
    }
    for (int64_t i = 0; i < N; ++i) {
        const double x = (double)col[i];
        col[i] = (x == missing || !isfinite(x) || x < 0.0 || x > 2.0) ? T(0) : (T)((x - mu) * inv_sd);
    }
    if (nmiss) atomicAdd(&counts[0], (unsigned long long)nmiss);
    if (ninv) atomicAdd(&counts[1], (unsigned long long)ninv);
}

unsigned grid_n(int64_t n) {
    const int64_t b = (n + 255) / 256;
    return (unsigned)(b < 148 * 64 ? (b > 0 ? b : 1) : 148 * 64);
}

}  // namespace

template <typename T>
void launch_col_sums_rowmajor(const T* X, int64_t N, int64_t Q, double* out, cudaStream_t st) {
    if (Q <= 0) return;
    col_sums_rowmajor_kernel<T><<<(unsigned)((Q + 127) / 128), 128, 0, st>>>(X, N, Q, out);
    count_launch();
}

template <typename T>
void launch_rowmajor_to_colmajor(const T* in, int64_t N, int64_t Q, double* out, cudaStream_t st) {
    if (N * Q == 0) return;
    rowmajor_to_colmajor_kernel<T><<<grid_n(N * Q), 256, 0, st>>>(in, N, Q, out);
    count_launch();
}

template <typename T>
void launch_colmajor_to_rowmajor(const double* in, int64_t N, int64_t Q, T* out, cudaStream_t st) {
    if (N * Q == 0) return;
    colmajor_to_rowmajor_kernel<T><<<grid_n(N * Q), 256, 0, st>>>(in, N, Q, out);
    count_launch();
}

template <typename T>
void launch_convert(const T* in, int64_t n, double* out, cudaStream_t st) {
    if (n == 0) return;
    convert_kernel<T><<<grid_n(n), 256, 0, st>>>(in, n, out);
    count_launch();
}

template <typename T>
void launch_convert_back(const double* in, int64_t n, T* out, cudaStream_t st) {
    if (n == 0) return;
    convert_back_kernel<T><<<grid_n(n), 256, 0, st>>>(in, n, out);
    count_launch();
}

template <typename T>
void launch_standardize_dosage(T* G, int64_t N, int64_t L, int ddof, double missing,
                               unsigned long long* counts, cudaStream_t st) {
    if (L <= 0) return;
    standardize_dosage_kernel<T><<<(unsigned)((L + 127) / 128), 128, 0, st>>>(G, N, L, ddof, missing,
                                                                             counts);
    count_launch();
}

#define LDS_PROJ_INST(T)                                                                          \
    template void launch_col_sums_rowmajor<T>(const T*, int64_t, int64_t, double*, cudaStream_t); \
    template void launch_rowmajor_to_colmajor<T>(const T*, int64_t, int64_t, double*,             \
                                                 cudaStream_t);                                   \
    template void launch_colmajor_to_rowmajor<T>(const double*, int64_t, int64_t, T*,             \
                                                 cudaStream_t);                                   \
    template void launch_convert<T>(const T*, int64_t, double*, cudaStream_t);                    \
    template void launch_convert_back<T>(const double*, int64_t, T*, cudaStream_t);               \
    template void launch_standardize_dosage<T>(T*, int64_t, int64_t, int, double,                 \
                                               unsigned long long*, cudaStream_t);
LDS_PROJ_INST(float)
LDS_PROJ_INST(double)

}  // namespace lds
