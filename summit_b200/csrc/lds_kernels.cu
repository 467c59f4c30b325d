// LD-score kernels for sm_100a.
//
// Exactness scheme.  Genotype operands are the exact integers G (value, 0 for
// missing) and O (observed mask) decoded from 2-bit BED codes.  Floating
// operands (probe weights in phase 1, the sketch Y in phase 2) are split per
// column into S signed int8 digits with a power-of-two scale
//     y ~= 2^(e-7) * (d0 + d1/128 + ... + d_{S-1}/128^(S-1)),
// d0 in [-127,127], d_k in [-64,64], all round-to-nearest (unbiased).  Every
// digit product is an exact int32 tensor-core accumulation; digits are
// recombined exactly in int64 and converted to FP64 once.  The only error is
// the representation error of the floating operand, |dy| <= 2^(e-8-7(S-1)).
#include <cfloat>
#include <cstdint>
#include <cstdio>

#include "lds_device.cuh"
#include "lds_internal.h"

namespace lds {

// ===========================================================================
// Genotype image preparation
// ===========================================================================
__global__ void repack_kernel(const uint8_t* __restrict__ src, int64_t src_bytes,
                              int64_t n_total, const int32_t* __restrict__ rows, int64_t N,
                              int64_t nbp, int64_t M, int64_t M_pad,
                              uint8_t* __restrict__ dst) {
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= M_pad * nbp) return;
    const int64_t j = idx / nbp;
    const int64_t b = idx - j * nbp;
    if (j >= M) {
        dst[idx] = 0x55;
        return;
    }
    const uint8_t* row = src + j * src_bytes;
    const int64_t i0 = b * 4;
    if (!rows && i0 + 4 <= N) {
        dst[idx] = row[b];
        return;
    }
    uint32_t out = 0;
    for (int t = 0; t < 4; ++t) {
        const int64_t i = i0 + t;
        uint32_t code = 1u;  // missing
        if (i < N) {
            const int64_t r = rows ? (int64_t)rows[i] : i;
            code = (row[r >> 2] >> (2 * (r & 3))) & 3u;
        }
        out |= code << (2 * t);
    }
    dst[idx] = (uint8_t)out;
}

void launch_repack(const uint8_t* src, int64_t src_bytes, int64_t n_total, const int32_t* rows,
                   const DevGeno& g, cudaStream_t st) {
    const int64_t total = g.M_pad * g.nbp;
    const int tpb = 256;
    repack_kernel<<<(unsigned)((total + tpb - 1) / tpb), tpb, 0, st>>>(
        src, src_bytes, n_total, rows, g.N, g.nbp, g.M, g.M_pad, g.codes);
    count_launch();
}

// One warp per SNP: counts of codes 00, 10, 11 and 01 over the real samples.
__global__ void counts_kernel(const uint8_t* __restrict__ codes, int64_t nbp, int64_t N,
                              int64_t N_pad, int64_t M, SnpCounts* __restrict__ out) {
    const int64_t j = (int64_t)blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (j >= M) return;
    const uint32_t* row = reinterpret_cast<const uint32_t*>(codes + j * nbp);
    const int64_t nw = nbp / 4;
    int c10 = 0, c11 = 0, c01 = 0;
    for (int64_t w = lane; w < nw; w += 32) {
        const uint32_t x = row[w];
        const uint32_t hi = (x >> 1) & 0x55555555u;
        const uint32_t lo = x & 0x55555555u;
        c11 += __popc(hi & lo);
        c10 += __popc(hi & ~lo);
        c01 += __popc(lo & ~hi);
    }
    for (int o = 16; o; o >>= 1) {
        c10 += __shfl_xor_sync(0xffffffffu, c10, o);
        c11 += __shfl_xor_sync(0xffffffffu, c11, o);
        c01 += __shfl_xor_sync(0xffffffffu, c01, o);
    }
    if (lane == 0) {
        const int miss = c01 - (int)(N_pad - N);
        SnpCounts c;
        c.n[1] = c10;
        c.n[2] = c11;
        c.n[3] = miss;
        c.n[0] = (int)N - c10 - c11 - miss;
        out[j] = c;
    }
}

void launch_counts(const DevGeno& g, SnpCounts* out, cudaStream_t st) {
    const int warps = 8;
    counts_kernel<<<(unsigned)((g.M + warps - 1) / warps), warps * 32, 0, st>>>(
        g.codes, g.nbp, g.N, g.N_pad, g.M, out);
    count_launch();
}

// HWE imputation of missing calls, genotype.cpp:146-184 (hwe_impute_value_prepared).
__device__ __forceinline__ uint32_t hwe_code(double q0, double q01, uint64_t seed_base,
                                             int global_row) {
    int v;
    if (q0 >= 1.0) {
        v = 0;
    } else if (q01 <= 0.0) {
        v = 2;
    } else {
        uint64_t h = seed_base;
        h ^= mix64((uint64_t)(uint32_t)global_row + 0x9e3779b97f4a7c15ULL);
        const uint64_t x = mix64(h);
        const double u = (double)((x >> 11) & ((1ULL << 53) - 1)) * (1.0 / 9007199254740992.0);
        v = (u < q0) ? 0 : (u < q01) ? 1 : 2;
    }
    return v == 0 ? 0u : v == 1 ? 2u : 3u;
}

__global__ void hwe_impute_kernel(uint8_t* __restrict__ codes, int64_t nbp, int64_t N, int64_t M,
                                  const double* __restrict__ q0, const double* __restrict__ q01,
                                  const uint64_t* __restrict__ seed_base,
                                  const int32_t* __restrict__ global_rows) {
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= M * nbp) return;
    const int64_t j = idx / nbp;
    const int64_t b = idx - j * nbp;
    const int64_t i0 = b * 4;
    if (i0 >= N) return;
    uint32_t byte = codes[idx];
    bool any = false;
    for (int t = 0; t < 4; ++t) any |= (((byte >> (2 * t)) & 3u) == 1u);
    if (!any) return;
    for (int t = 0; t < 4; ++t) {
        const int64_t i = i0 + t;
        if (i >= N) break;
        if (((byte >> (2 * t)) & 3u) != 1u) continue;
        const int gr = global_rows ? global_rows[i] : (int)i;
        const uint32_t c = hwe_code(q0[j], q01[j], seed_base[j], gr);
        byte = (byte & ~(3u << (2 * t))) | (c << (2 * t));
    }
    codes[idx] = (uint8_t)byte;
}

void launch_hwe_impute(const DevGeno& g, const double* q0, const double* q01,
                       const uint64_t* seed_base, const int32_t* global_rows, cudaStream_t st) {
    const int64_t total = g.M * g.nbp;
    hwe_impute_kernel<<<(unsigned)((total + 255) / 256), 256, 0, st>>>(
        g.codes, g.nbp, g.N, g.M, q0, q01, seed_base, global_rows);
    count_launch();
}

// ===========================================================================
// Digit splitting of floating operands
// ===========================================================================
// Exponent e with amax * 2^(7-e) <= 127 (so the leading digit fits in s8).
__device__ __forceinline__ int digit_exponent(double amax) {
    if (!(amax > 0.0) || !isfinite(amax)) return 0;
    int e = ilogb(amax) + 1;
    if (ldexp(amax, 7 - e) > 127.0) e += 1;
    return e;
}

template <int S>
__device__ __forceinline__ void split_digits(double y, int e, int8_t (&d)[S]) {
    double t = ldexp(y, 7 - e);
    double r = rint(t);
    d[0] = (int8_t)r;
    t -= r;
#pragma unroll
    for (int k = 1; k < S; ++k) {
        t *= 128.0;
        r = rint(t);
        d[k] = (int8_t)r;
        t -= r;
    }
}

__device__ __forceinline__ double block_max(double v, double* red) {
    for (int o = 16; o; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    __syncthreads();
    if (lane == 0) red[warp] = v;
    __syncthreads();
    if (warp == 0) {
        v = (lane < (int)(blockDim.x >> 5)) ? red[lane] : 0.0;
        for (int o = 16; o; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
        if (lane == 0) red[0] = v;
    }
    __syncthreads();
    return red[0];
}

// Phase-1 weights: one CTA per padded column (k, v).
template <int S>
__global__ void p1_weights_kernel(P1Weights w, const double* __restrict__ mean,
                                  const double* __restrict__ sdinv, const double* __restrict__ Z,
                                  int64_t z_ld, int64_t z_row0) {
    __shared__ double red[32];
    const int col = blockIdx.x;
    const int k = col / w.Vp, v = col - k * w.Vp;
    const int64_t r0 = w.bin_off[k], nnzp = w.bin_off[k + 1] - r0;
    int8_t* base = w.wq + w.wq_off[k];
    if (v >= w.V) {
        for (int64_t r = threadIdx.x; r < nnzp; r += blockDim.x)
            for (int t = 0; t < S; ++t)
                for (int p = 0; p < 2; ++p) base[(((int64_t)t * 2 + p) * w.Vp + v) * nnzp + r] = 0;
        if (threadIdx.x == 0) w.colscale[col] = 0.0;
        return;
    }
    double amax = 0.0;
    for (int64_t r = threadIdx.x; r < nnzp; r += blockDim.x) {
        const double sc = w.sc[r0 + r];
        if (sc == 0.0) continue;
        const int64_t j = w.rowind[r0 + r];
        const double w1 = sdinv[j] * (sc * Z[(int64_t)v * z_ld + (j - z_row0)]);
        amax = fmax(amax, fmax(fabs(w1), fabs(mean[j] * w1)));
    }
    amax = block_max(amax, red);
    const int e = digit_exponent(amax);
    for (int64_t r = threadIdx.x; r < nnzp; r += blockDim.x) {
        const double sc = w.sc[r0 + r];
        int8_t d1[S], d2[S];
        if (sc == 0.0) {
            for (int t = 0; t < S; ++t) d1[t] = d2[t] = 0;
        } else {
            const int64_t j = w.rowind[r0 + r];
            const double w1 = sdinv[j] * (sc * Z[(int64_t)v * z_ld + (j - z_row0)]);
            split_digits<S>(w1, e, d1);
            split_digits<S>(-(mean[j] * w1), e, d2);
        }
        for (int t = 0; t < S; ++t) {
            base[(((int64_t)t * 2 + 0) * w.Vp + v) * nnzp + r] = d1[t];
            base[(((int64_t)t * 2 + 1) * w.Vp + v) * nnzp + r] = d2[t];
        }
    }
    if (threadIdx.x == 0) w.colscale[col] = ldexp(1.0, e - 7 - 7 * (S - 1));
}

void launch_p1_weights(const P1Weights& w, const double* mean, const double* sdinv,
                       const double* Z, int64_t z_ld, int64_t z_row0, cudaStream_t st) {
    const unsigned grid = (unsigned)(w.K * w.Vp);
    if (grid == 0) return;
    switch (w.S) {
        case 3: p1_weights_kernel<3><<<grid, 256, 0, st>>>(w, mean, sdinv, Z, z_ld, z_row0); break;
        case 4: p1_weights_kernel<4><<<grid, 256, 0, st>>>(w, mean, sdinv, Z, z_ld, z_row0); break;
        case 5: p1_weights_kernel<5><<<grid, 256, 0, st>>>(w, mean, sdinv, Z, z_ld, z_row0); break;
        default: p1_weights_kernel<6><<<grid, 256, 0, st>>>(w, mean, sdinv, Z, z_ld, z_row0); break;
    }
    count_launch();
}

// Sketch quantization: one CTA per padded column.
template <int S>
__global__ void quantize_y_kernel(const double* __restrict__ Y, int64_t N, int64_t N_pad, int K,
                                  int V, int Vp, int8_t* __restrict__ Yq,
                                  double* __restrict__ colscale) {
    __shared__ double red[32];
    const int col = blockIdx.x;
    const int k = col / Vp, v = col - k * Vp;
    const int64_t KVp = (int64_t)K * Vp;
    if (v >= V) {
        for (int64_t i = threadIdx.x; i < N_pad; i += blockDim.x)
            for (int t = 0; t < S; ++t) Yq[((int64_t)t * KVp + col) * N_pad + i] = 0;
        if (threadIdx.x == 0) colscale[col] = 0.0;
        return;
    }
    const double* y = Y + ((int64_t)k * V + v) * N_pad;
    double amax = 0.0;
    int bad = 0;
    for (int64_t i = threadIdx.x; i < N; i += blockDim.x) {
        const double a = fabs(y[i]);
        bad |= !(a <= DBL_MAX);  // NaN or infinite
        amax = fmax(amax, a);
    }
    // A non-finite sketch value makes every product with this column
    // non-finite in the reference's GEMM; a NaN scale does the same here, so
    // the phase-2 guards drop those updates just as the reference does.
    bad = __syncthreads_or(bad);
    amax = block_max(bad ? 0.0 : amax, red);
    const int e = digit_exponent(amax);
    for (int64_t i = threadIdx.x; i < N_pad; i += blockDim.x) {
        int8_t d[S];
        if (i < N && !bad) {
            split_digits<S>(y[i], e, d);
        } else {
            for (int t = 0; t < S; ++t) d[t] = 0;
        }
        for (int t = 0; t < S; ++t) Yq[((int64_t)t * KVp + col) * N_pad + i] = d[t];
    }
    if (threadIdx.x == 0) colscale[col] = bad ? (double)NAN : ldexp(1.0, e - 7 - 7 * (S - 1));
}

void launch_quantize_y(const double* Y, int64_t N, int64_t N_pad, int K, int V, int Vp, int S,
                       int8_t* Yq, double* colscale, cudaStream_t st) {
    const unsigned grid = (unsigned)(K * Vp);
    switch (S) {
        case 3: quantize_y_kernel<3><<<grid, 256, 0, st>>>(Y, N, N_pad, K, V, Vp, Yq, colscale); break;
        case 4: quantize_y_kernel<4><<<grid, 256, 0, st>>>(Y, N, N_pad, K, V, Vp, Yq, colscale); break;
        case 5: quantize_y_kernel<5><<<grid, 256, 0, st>>>(Y, N, N_pad, K, V, Vp, Yq, colscale); break;
        default: quantize_y_kernel<6><<<grid, 256, 0, st>>>(Y, N, N_pad, K, V, Vp, Yq, colscale); break;
    }
    count_launch();
}

// ===========================================================================
// Phase 1: Y = X W (reduction over SNPs), int8 tensor cores.
// CTA: 128 samples x 16 probe columns (x S digits) of one bin; 8 warps as
// 4 (samples) x 2 (column halves).  K-step: 32 SNPs of the bin's member list.
// The packed SNP rows are decoded and transposed to sample-major in smem.
// ===========================================================================
template <int S>
__global__ void __launch_bounds__(256) p1_kernel(DevGeno g, P1Weights w, double* __restrict__ Y) {
    constexpr int BM = 128, BK = 32, ROWA = 48, ROWB = 48;
    constexpr int NB = 2 * S * 8;
    __shared__ __align__(16) uint8_t sG[BM * ROWA];
    __shared__ __align__(16) uint8_t sO[BM * ROWA];
    __shared__ __align__(16) uint8_t sW[2][2][NB * ROWB];
    __shared__ __align__(16) uint8_t sP[2][BK * 32];

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int wm = warp & 3, wn = warp >> 2;
    const int nct = w.Vp / 16;
    const int k = blockIdx.y / nct, ct = blockIdx.y - k * nct;
    const int64_t i0 = (int64_t)blockIdx.x * BM;
    const int64_t r0 = w.bin_off[k], nnzp = w.bin_off[k + 1] - r0;
    const int nkt = (int)(nnzp / BK);
    const int8_t* wbase = w.wq + w.wq_off[k];

    int acc[2][S][4];
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
        for (int t = 0; t < S; ++t)
#pragma unroll
            for (int q = 0; q < 4; ++q) acc[a][t][q] = 0;

    auto load_stage = [&](int kt, int st) {
        if (tid < 64) {
            const int row = tid >> 1, hf = tid & 1;
            const int64_t j = w.rowind[r0 + (int64_t)kt * BK + row];
            cp_async16(&sP[st][row * 32 + hf * 16], g.codes + j * g.nbp + i0 / 4 + hf * 16);
        }
        for (int c = tid; c < 4 * NB; c += 256) {
            const int p = c / (2 * NB);
            const int rem = c - p * 2 * NB;
            const int sr = rem >> 1, hf = rem & 1;
            const int half = sr / (S * 8), t = (sr >> 3) % S, cc = sr & 7;
            const int v = ct * 16 + half * 8 + cc;
            const int8_t* src =
                wbase + (((int64_t)t * 2 + p) * w.Vp + v) * nnzp + (int64_t)kt * BK + hf * 16;
            cp_async16(&sW[st][p][sr * ROWB + hf * 16], src);
        }
        cp_async_commit();
    };

    if (nkt > 0) load_stage(0, 0);
    for (int kt = 0; kt < nkt; ++kt) {
        const int st = kt & 1;
        cp_async_wait_all();
        __syncthreads();
        if (kt + 1 < nkt) load_stage(kt + 1, st ^ 1);
        {
            const int sq = tid & 7, sqd = tid >> 3;
            uint32_t g4[4], o4[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) decode4(sP[st][(sq * 4 + i) * 32 + sqd], g4[i], o4[i]);
            uint32_t c[4];
            transpose4x4(g4[0], g4[1], g4[2], g4[3], c[0], c[1], c[2], c[3]);
#pragma unroll
            for (int s = 0; s < 4; ++s)
                *reinterpret_cast<uint32_t*>(&sG[(sqd * 4 + s) * ROWA + sq * 4]) = c[s];
            transpose4x4(o4[0], o4[1], o4[2], o4[3], c[0], c[1], c[2], c[3]);
#pragma unroll
            for (int s = 0; s < 4; ++s)
                *reinterpret_cast<uint32_t*>(&sO[(sqd * 4 + s) * ROWA + sq * 4]) = c[s];
        }
        __syncthreads();
        uint32_t aG[2][4], aO[2][4];
#pragma unroll
        for (int mt = 0; mt < 2; ++mt) {
            const int row = wm * 32 + mt * 16 + (lane & 15);
            const int col = (lane >> 4) * 16;
            ldsm_x4(smem_u32(&sG[row * ROWA + col]), aG[mt][0], aG[mt][1], aG[mt][2], aG[mt][3]);
            ldsm_x4(smem_u32(&sO[row * ROWA + col]), aO[mt][0], aO[mt][1], aO[mt][2], aO[mt][3]);
        }
#pragma unroll
        for (int t = 0; t < S; ++t) {
            const int sr = (wn * S + t) * 8 + (lane & 7);
            const int col = ((lane >> 3) & 1) * 16;
            uint32_t b0, b1, c0, c1;
            ldsm_x2(smem_u32(&sW[st][0][sr * ROWB + col]), b0, b1);
            ldsm_x2(smem_u32(&sW[st][1][sr * ROWB + col]), c0, c1);
#pragma unroll
            for (int mt = 0; mt < 2; ++mt) {
                mma_s8(acc[mt][t], aG[mt], b0, b1);
                mma_s8(acc[mt][t], aO[mt], c0, c1);
            }
        }
    }

#pragma unroll
    for (int mt = 0; mt < 2; ++mt)
#pragma unroll
        for (int h = 0; h < 2; ++h)
#pragma unroll
            for (int e = 0; e < 2; ++e) {
                const int64_t i = i0 + wm * 32 + mt * 16 + h * 8 + (lane >> 2);
                const int v = ct * 16 + wn * 8 + (lane & 3) * 2 + e;
                if (v >= w.V) continue;
                long long T = 0;
#pragma unroll
                for (int t = 0; t < S; ++t) T = T * 128 + (long long)acc[mt][t][h * 2 + e];
                Y[((int64_t)k * w.V + v) * g.N_pad + i] = w.colscale[k * w.Vp + v] * (double)T;
            }
}

void launch_p1(const DevGeno& g, const P1Weights& w, const int64_t* h_bin_off, double* Y,
               cudaStream_t st) {
    (void)h_bin_off;
    dim3 grid((unsigned)(g.N_pad / 128), (unsigned)(w.K * (w.Vp / 16)));
    switch (w.S) {
        case 3: p1_kernel<3><<<grid, 256, 0, st>>>(g, w, Y); break;
        case 4: p1_kernel<4><<<grid, 256, 0, st>>>(g, w, Y); break;
        case 5: p1_kernel<5><<<grid, 256, 0, st>>>(g, w, Y); break;
        default: p1_kernel<6><<<grid, 256, 0, st>>>(g, w, Y); break;
    }
    count_launch();
}

// ===========================================================================
// Phase 2: Work = X^T Y (reduction over samples) with the LD-score epilogue.
// CTA: 128 SNPs x one bin; loops over the bin's 16-column tiles; 8 warps as
// 4 (SNPs) x 2 (column halves).  K-step: 64 samples.  Per row the squared
// (and fourth-power) sums over the bin's probes are accumulated in FP64 in a
// fixed order, then guarded and added to accum — one writer per (SNP, bin).
// ===========================================================================
template <int S, bool RAW>
__global__ void __launch_bounds__(256) p2_kernel(DevGeno g, P2Args a) {
    constexpr int BM = 128, BK = 64, ROWB = 80;
    constexpr int NB = 2 * S * 8;
    __shared__ __align__(16) uint8_t sG[BM * ROWB];
    __shared__ __align__(16) uint8_t sO[BM * ROWB];
    __shared__ __align__(16) uint8_t sB[2][NB * ROWB];
    __shared__ __align__(16) uint8_t sP[2][BM * 16];
    __shared__ double sPart[2][2][BM];

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int wm = warp & 3, wn = warp >> 2;
    const int k = blockIdx.y;
    const int64_t jt0 = a.j0 + (int64_t)blockIdx.x * BM;
    const int64_t KVp = (int64_t)a.K * a.Vp;
    const int nct = a.Vp / 16;
    const int nkt = (int)(g.N_pad / BK);
    double run2 = 0.0, run4 = 0.0;

    for (int ct = 0; ct < nct; ++ct) {
        int accG[2][S][4], accO[2][S][4];
#pragma unroll
        for (int m = 0; m < 2; ++m)
#pragma unroll
            for (int t = 0; t < S; ++t)
#pragma unroll
                for (int q = 0; q < 4; ++q) accG[m][t][q] = accO[m][t][q] = 0;

        auto load_stage = [&](int kt, int st) {
            if (tid < BM)
                cp_async16(&sP[st][tid * 16], g.codes + (jt0 + tid) * g.nbp + (int64_t)kt * (BK / 4));
            for (int c = tid; c < NB * 4; c += 256) {
                const int sr = c >> 2, part = c & 3;
                const int half = sr / (S * 8), t = (sr >> 3) % S, cc = sr & 7;
                const int64_t q = (int64_t)k * a.Vp + ct * 16 + half * 8 + cc;
                const int8_t* src = a.Yq + ((int64_t)t * KVp + q) * g.N_pad + (int64_t)kt * BK + part * 16;
                cp_async16(&sB[st][sr * ROWB + part * 16], src);
            }
            cp_async_commit();
        };

        load_stage(0, 0);
        for (int kt = 0; kt < nkt; ++kt) {
            const int st = kt & 1;
            cp_async_wait_all();
            __syncthreads();
            if (kt + 1 < nkt) load_stage(kt + 1, st ^ 1);
            {
                const int r = tid >> 1, h = tid & 1;
                const uint2 pk = *reinterpret_cast<const uint2*>(&sP[st][r * 16 + h * 8]);
                uint32_t gw[8], ow[8];
                decode8(pk.x & 0xFFFFu, gw[0], gw[1], ow[0], ow[1]);
                decode8(pk.x >> 16, gw[2], gw[3], ow[2], ow[3]);
                decode8(pk.y & 0xFFFFu, gw[4], gw[5], ow[4], ow[5]);
                decode8(pk.y >> 16, gw[6], gw[7], ow[6], ow[7]);
                uint4* dG = reinterpret_cast<uint4*>(&sG[r * ROWB + h * 32]);
                uint4* dO = reinterpret_cast<uint4*>(&sO[r * ROWB + h * 32]);
                dG[0] = make_uint4(gw[0], gw[1], gw[2], gw[3]);
                dG[1] = make_uint4(gw[4], gw[5], gw[6], gw[7]);
                dO[0] = make_uint4(ow[0], ow[1], ow[2], ow[3]);
                dO[1] = make_uint4(ow[4], ow[5], ow[6], ow[7]);
            }
            __syncthreads();
#pragma unroll
            for (int kk = 0; kk < 2; ++kk) {
                uint32_t aG[2][4], aO[2][4];
#pragma unroll
                for (int mt = 0; mt < 2; ++mt) {
                    const int row = wm * 32 + mt * 16 + (lane & 15);
                    const int col = kk * 32 + (lane >> 4) * 16;
                    ldsm_x4(smem_u32(&sG[row * ROWB + col]), aG[mt][0], aG[mt][1], aG[mt][2], aG[mt][3]);
                    ldsm_x4(smem_u32(&sO[row * ROWB + col]), aO[mt][0], aO[mt][1], aO[mt][2], aO[mt][3]);
                }
#pragma unroll
                for (int t = 0; t < S; ++t) {
                    const int sr = (wn * S + t) * 8 + (lane & 7);
                    const int col = kk * 32 + ((lane >> 3) & 1) * 16;
                    uint32_t b0, b1;
                    ldsm_x2(smem_u32(&sB[st][sr * ROWB + col]), b0, b1);
#pragma unroll
                    for (int mt = 0; mt < 2; ++mt) {
                        mma_s8(accG[mt][t], aG[mt], b0, b1);
                        mma_s8(accO[mt][t], aO[mt], b0, b1);
                    }
                }
            }
        }

        if constexpr (RAW) {
            // Verification mode: exact recombined integer products G^T y and
            // O^T y per (SNP, column), no scaling.
#pragma unroll
            for (int mt = 0; mt < 2; ++mt)
#pragma unroll
                for (int h = 0; h < 2; ++h)
#pragma unroll
                    for (int e = 0; e < 2; ++e) {
                        const int64_t j = jt0 + wm * 32 + mt * 16 + h * 8 + (lane >> 2);
                        const int v = ct * 16 + wn * 8 + (lane & 3) * 2 + e;
                        if (v >= a.V || j >= a.j1) continue;
                        long long TG = 0, TO = 0;
#pragma unroll
                        for (int t = 0; t < S; ++t) {
                            TG = TG * 128 + (long long)accG[mt][t][h * 2 + e];
                            TO = TO * 128 + (long long)accO[mt][t][h * 2 + e];
                        }
                        a.raw_g[(j - a.out_row0) * a.V + v] = TG;
                        a.raw_o[(j - a.out_row0) * a.V + v] = TO;
                    }
            __syncthreads();
            continue;
        }
        // Epilogue of this column tile.
        double p2[2][2], p4[2][2];
#pragma unroll
        for (int mt = 0; mt < 2; ++mt)
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                p2[mt][h] = 0.0;
                p4[mt][h] = 0.0;
                const int r = wm * 32 + mt * 16 + h * 8 + (lane >> 2);
                const int64_t j = jt0 + r;
                const double mu = (j < g.M) ? a.mean[j] : 0.0;
                const double sd = (j < g.M) ? a.sdinv[j] : 0.0;
#pragma unroll
                for (int e = 0; e < 2; ++e) {
                    const int v = ct * 16 + wn * 8 + (lane & 3) * 2 + e;
                    if (v >= a.V) continue;
                    long long TG = 0, TO = 0;
#pragma unroll
                    for (int t = 0; t < S; ++t) {
                        TG = TG * 128 + (long long)accG[mt][t][h * 2 + e];
                        TO = TO * 128 + (long long)accO[mt][t][h * 2 + e];
                    }
                    const double cs = a.colscale[(int64_t)k * a.Vp + v];
                    const double wv = sd * cs * ((double)TG - mu * (double)TO);
                    const double w2 = wv * wv;
                    p2[mt][h] += w2;
                    p4[mt][h] += w2 * w2;
                }
                p2[mt][h] += __shfl_xor_sync(0xffffffffu, p2[mt][h], 1);
                p2[mt][h] += __shfl_xor_sync(0xffffffffu, p2[mt][h], 2);
                p4[mt][h] += __shfl_xor_sync(0xffffffffu, p4[mt][h], 1);
                p4[mt][h] += __shfl_xor_sync(0xffffffffu, p4[mt][h], 2);
                if ((lane & 3) == 0) {
                    sPart[0][wn][r] = p2[mt][h];
                    sPart[1][wn][r] = p4[mt][h];
                }
            }
        __syncthreads();
        if (tid < BM) {
            run2 += sPart[0][0][tid] + sPart[0][1][tid];
            run4 += sPart[1][0][tid] + sPart[1][1][tid];
        }
        __syncthreads();
    }

    if (RAW) return;
    if (tid < BM) {
        const int64_t j = jt0 + tid;
        if (j < a.j1) {
            const double ls = a.left_scale[j];
            double upd = run2 * ls;
            const double seg = (double)a.V;
            const bool nonfinite = !isfinite(upd);
            const bool extreme = !nonfinite && isfinite(a.extreme_warn) && seg > 0.0 &&
                                 upd > a.extreme_warn * seg;
            if (a.guard_counts) {
                if (nonfinite) atomicAdd(&a.guard_counts[0], 1ULL);
                else if (extreme) atomicAdd(&a.guard_counts[1], 1ULL);
            }
            if (!(nonfinite || (extreme && a.drop_extreme))) {
                if (upd < 0.0) upd = 0.0;
                const int64_t o = (j - a.out_row0) * a.K + k;
                a.accum[o] += upd;
                if (a.mc) a.mc[o] += run4 * ls * ls;
            }
        }
    }
}

void launch_p2(const DevGeno& g, const P2Args& a, cudaStream_t st) {
    const int64_t rows = a.j1 - a.j0;
    if (rows <= 0 || a.K <= 0) return;
    dim3 grid((unsigned)((rows + 127) / 128), (unsigned)a.K);
    if (a.raw_g) {
        if (a.S != 1) return;
        p2_kernel<1, true><<<grid, 256, 0, st>>>(g, a);
        count_launch();
        return;
    }
    switch (a.S) {
        case 3: p2_kernel<3, false><<<grid, 256, 0, st>>>(g, a); break;
        case 4: p2_kernel<4, false><<<grid, 256, 0, st>>>(g, a); break;
        case 5: p2_kernel<5, false><<<grid, 256, 0, st>>>(g, a); break;
        default: p2_kernel<6, false><<<grid, 256, 0, st>>>(g, a); break;
    }
    count_launch();
}

// ===========================================================================
// Synthetic genotypes (bedfile.py): one thread per packed byte column.
// ===========================================================================
__device__ __forceinline__ uint64_t synth_draw(uint64_t key, uint64_t i, uint64_t j) {
    return mix64(key ^ mix64((j << 32) | i));
}

// Rows of `ld` bytes; with pad_missing the samples past n (and the bytes past
// ceil(n/4)) carry the missing code 01, as the padded genotype image needs.
__global__ void synth_kernel(int64_t n, int64_t M, uint64_t k2, uint64_t k3,
                             const int64_t* __restrict__ t0, const int64_t* __restrict__ t1,
                             int missing, uint8_t* __restrict__ out, int64_t ld,
                             int pad_missing) {
    const int64_t nb = (n + 3) / 4;
    const int64_t b = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= ld) return;
    if (b >= nb) {
        for (int64_t j = 0; j < M; ++j) out[j * ld + b] = 0x55;
        return;
    }
    long long u[4] = {0, 0, 0, 0};
    for (int64_t j = 0; j < M; ++j) {
        const long long a0 = t0[j], a1 = t1[j];
        uint32_t byte = 0;
        for (int t = 0; t < 4; ++t) {
            const int64_t i = b * 4 + t;
            if (i >= n) {
                if (pad_missing) byte |= 1u << (2 * t);
                continue;
            }
            const uint64_t r = synth_draw(k2, (uint64_t)i, (uint64_t)j);
            const long long e = (long long)(r & 0xFFFFULL) + (long long)((r >> 16) & 0xFFFFULL) +
                                (long long)((r >> 32) & 0xFFFFULL) + (long long)(r >> 48) - 131070LL;
            u[t] = (j == 0) ? e : ((58982LL * u[t] + 28567LL * e) >> 16);
            uint32_t code = (u[t] < a0) ? 0u : (u[t] < a1) ? 2u : 3u;
            if (missing && (synth_draw(k3, (uint64_t)i, (uint64_t)j) >> 32) < 42949673ULL) code = 1u;
            byte |= code << (2 * t);
        }
        out[j * ld + b] = (uint8_t)byte;
    }
}

void launch_synth(int64_t n, int64_t M, uint64_t seed, const int64_t* t0, const int64_t* t1,
                  int missing, uint8_t* out, cudaStream_t st, int64_t ld, int pad_missing) {
    const uint64_t k2 = mix64(seed ^ mix64(2ULL));
    const uint64_t k3 = mix64(seed ^ mix64(3ULL));
    const int64_t nb = (n + 3) / 4;
    if (ld <= 0) ld = nb;
    synth_kernel<<<(unsigned)((ld + 127) / 128), 128, 0, st>>>(n, M, k2, k3, t0, t1, missing, out,
                                                              ld, pad_missing);
    count_launch();
}

}  // namespace lds
