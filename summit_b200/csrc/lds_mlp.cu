// Surrogate network of the learned control variate: in -> 128 -> 128 -> 128 -> out,
// GELU (erf form) after each hidden layer, trained by mean squared error.
//
// Weights are kept in FP32 (Adam's master copy) and enter every product
// rounded to BF16; hidden activations are rounded to BF16 where they feed the
// next product; all sums accumulate in FP32.  Four kernels make one training
// step over a mini-batch of gathered rows:
//   mlp_forward_kernel      32 rows per CTA, all four layers in shared memory
//                           (weights transposed, BF16); stores pre-activations
//                           z1..z3 and the loss gradient of the outputs;
//   mlp_backward_data_kernel  dZ_l = (dZ_{l+1} W_{l+1}) * gelu'(z_l), l = 3, 2, 1;
//   mlp_backward_weight_kernel dW_l = dZ_l^T H_{l-1}, db_l = sum dZ_l over rows
//                           (row-split, FP32 atomics into the gradient);
//   mlp_adam_kernel         Adam with bias correction on the FP32 master weights.
// The batch is small next to the genotype products (a few GFLOP per epoch), so
// these run on the CUDA cores with register tiles.
#include <cuda_bf16.h>

#include <cstdint>

#include "lds_internal.h"

namespace lds {
namespace mlp {

constexpr int kR = 32;         // rows per CTA
constexpr int kThreads = 256;

__device__ __forceinline__ float bf16r(float x) { return __bfloat162float(__float2bfloat16_rn(x)); }
__device__ __forceinline__ float gelu(float z) {
    return 0.5f * z * (1.0f + erff(z * 0.70710678118654752f));
}
__device__ __forceinline__ float gelu_grad(float z) {
    return 0.5f * (1.0f + erff(z * 0.70710678118654752f)) +
           z * 0.39894228040143268f * expf(-0.5f * z * z);
}

// acc[i][j] = sum_k A[(r0+i) lda + k] * B[k ldb + c0 + j] for this thread's
// 4 x 4 tile (rows r0 = 4 (tid / 32), columns c0 = 4 (tid % 32)).  A is FP32 in
// shared memory (a warp reads one row group: broadcast), B is BF16 in shared
// memory with columns contiguous (a warp reads 256 contiguous bytes).
__device__ __forceinline__ void tile_product(const float* A, int lda, const __nv_bfloat16* B,
                                             int ldb, int K, float (&acc)[4][4]) {
    const int t = threadIdx.x, c0 = 4 * (t & 31), r0 = 4 * (t >> 5);
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = 0.0f;
    if (c0 >= ldb) return;
#pragma unroll 4
    for (int k = 0; k < K; ++k) {
        const uint2 wv = *reinterpret_cast<const uint2*>(B + (int64_t)k * ldb + c0);
        const __nv_bfloat162 w01 = *reinterpret_cast<const __nv_bfloat162*>(&wv.x);
        const __nv_bfloat162 w23 = *reinterpret_cast<const __nv_bfloat162*>(&wv.y);
        const float w[4] = {__low2float(w01), __high2float(w01), __low2float(w23),
                            __high2float(w23)};
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const float a = A[(r0 + i) * lda + k];
#pragma unroll
            for (int j = 0; j < 4; ++j) acc[i][j] = fmaf(a, w[j], acc[i][j]);
        }
    }
}

// Copy `bytes` (a multiple of 16) from global to shared memory.
__device__ __forceinline__ void copy16(void* dst, const void* src, int bytes) {
    const uint4* s = reinterpret_cast<const uint4*>(src);
    uint4* d = reinterpret_cast<uint4*>(dst);
    for (int i = threadIdx.x; i < bytes / 16; i += blockDim.x) d[i] = s[i];
}

}  // namespace mlp

using namespace mlp;

// BF16 copies of the weights, made once per step: pack_t = W1^T | W2^T | W3^T |
// W4^T (column-contiguous, W4^T padded to out_pad columns) for the forward
// products, pack_n = W4 | W3 | W2 as stored (W4 padded to out_pad rows) for the
// backward ones.
__global__ void mlp_pack_kernel(MlpArgs a, __nv_bfloat16* __restrict__ pack_t,
                                __nv_bfloat16* __restrict__ pack_n) {
    const MlpLayout L = mlp_layout(a.in, a.out);
    const int op = mlp_out_pad(a.out), H = kMlpHidden;
    const int64_t nt = (int64_t)a.in * H + 2 * H * H + (int64_t)H * op;
    const int64_t nn = (int64_t)op * H + 2 * H * H;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nt + nn;
         i += (int64_t)gridDim.x * blockDim.x) {
        if (i < nt) {
            // transposed: element (k, c) of W^T = W[c][k]
            float v = 0.0f;
            int64_t r = i;
            if (r < (int64_t)a.in * H) {
                const int k = (int)(r / H), c = (int)(r % H);
                v = a.params[L.W1 + (int64_t)c * a.in + k];
            } else if ((r -= (int64_t)a.in * H) < H * H) {
                v = a.params[L.W2 + (r % H) * H + r / H];
            } else if ((r -= H * H) < H * H) {
                v = a.params[L.W3 + (r % H) * H + r / H];
            } else {
                r -= H * H;
                const int k = (int)(r / op), c = (int)(r % op);
                v = c < a.out ? a.params[L.W4 + (int64_t)c * H + k] : 0.0f;
            }
            pack_t[i] = __float2bfloat16_rn(v);
        } else {
            int64_t r = i - nt;
            float v = 0.0f;
            if (r < (int64_t)op * H) {
                const int c = (int)(r / H);
                v = c < a.out ? a.params[L.W4 + r] : 0.0f;
            } else if ((r -= (int64_t)op * H) < H * H) {
                v = a.params[L.W3 + r];
            } else {
                v = a.params[L.W2 + (r - H * H)];
            }
            pack_n[i - nt] = __float2bfloat16_rn(v);
        }
    }
}

__global__ void __launch_bounds__(kThreads)
    mlp_forward_kernel(MlpArgs a, const __nv_bfloat16* __restrict__ pack_t,
                       const float* __restrict__ x, const int32_t* __restrict__ rows, int64_t n,
                       const float* __restrict__ target, float* __restrict__ out,
                       float* __restrict__ zs, float* __restrict__ dout, double* __restrict__ loss,
                       float gscale) {
    extern __shared__ __align__(16) uint8_t smem[];
    const MlpLayout L = mlp_layout(a.in, a.out);
    const int op = mlp_out_pad(a.out);
    __nv_bfloat16* T1 = reinterpret_cast<__nv_bfloat16*>(smem);    // [in][128]
    __nv_bfloat16* T2 = T1 + a.in * kMlpHidden;                     // [128][128]
    __nv_bfloat16* T3 = T2 + kMlpHidden * kMlpHidden;               // [128][128]
    __nv_bfloat16* T4 = T3 + kMlpHidden * kMlpHidden;               // [128][op]
    float* X = reinterpret_cast<float*>(T4 + kMlpHidden * op);      // [kR][in]
    float* H1 = X + kR * a.in;                                      // [kR][128]
    float* H2 = H1 + kR * kMlpHidden;                               // [kR][128]
    __shared__ float red[kThreads / 32];

    copy16(T1, pack_t, (a.in * kMlpHidden + 2 * kMlpHidden * kMlpHidden + kMlpHidden * op) * 2);
    const int64_t r_base = (int64_t)blockIdx.x * kR;
    for (int idx = threadIdx.x; idx < kR * a.in; idx += blockDim.x) {
        const int r = idx / a.in, k = idx - (idx / a.in) * a.in;
        const int64_t rr = r_base + r;
        float v = 0.0f;
        if (rr < n) v = bf16r(x[(int64_t)(rows ? rows[rr] : rr) * a.in + k]);
        X[idx] = v;
    }
    __syncthreads();

    const int t = threadIdx.x, c0 = 4 * (t & 31), r0 = 4 * (t >> 5);
    float acc[4][4];
    const float* bias[3] = {a.params + L.b1, a.params + L.b2, a.params + L.b3};
    const __nv_bfloat16* Ts[3] = {T1, T2, T3};
    const float* in_act[3] = {X, H1, H2};
    float* out_act[3] = {H1, H2, H1};
    const int kin[3] = {a.in, kMlpHidden, kMlpHidden};
    for (int l = 0; l < 3; ++l) {
        tile_product(in_act[l], kin[l], Ts[l], kMlpHidden, kin[l], acc);
        __syncthreads();  // layer 3 writes H1, which layer 2 read
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const int64_t rr = r_base + r0 + i;
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const float z = acc[i][j] + bias[l][c0 + j];
                if (zs && rr < n) zs[(rr * 3 + l) * kMlpHidden + c0 + j] = z;
                out_act[l][(r0 + i) * kMlpHidden + c0 + j] = bf16r(gelu(z));
            }
        }
        __syncthreads();
    }
    tile_product(H1, kMlpHidden, T4, op, kMlpHidden, acc);
    float lsum = 0.0f;
    if (c0 < op) {
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const int64_t rr = r_base + r0 + i;
            if (rr >= n) continue;
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const int c = c0 + j;
                if (c >= a.out) continue;
                const float o = acc[i][j] + a.params[L.b4 + c];
                if (out) out[rr * a.out + c] = o;
                if (target) {
                    const float d = o - target[(int64_t)(rows ? rows[rr] : rr) * a.out + c];
                    if (dout) dout[rr * op + c] = 2.0f * d * gscale;
                    lsum += d * d;
                }
            }
        }
    }
    if (dout && c0 < op) {  // padding columns of dout read as zero in backward
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const int64_t rr = r_base + r0 + i;
            if (rr >= n) continue;
            for (int j = 0; j < 4; ++j)
                if (c0 + j >= a.out) dout[rr * op + c0 + j] = 0.0f;
        }
    }
    if (loss) {
        for (int o = 16; o; o >>= 1) lsum += __shfl_xor_sync(0xffffffffu, lsum, o);
        if ((t & 31) == 0) red[t >> 5] = lsum;
        __syncthreads();
        if (t == 0) {
            double s = 0.0;
            for (int w = 0; w < kThreads / 32; ++w) s += red[w];
            atomicAdd(loss, s * (double)gscale);
        }
    }
}

__global__ void __launch_bounds__(kThreads)
    mlp_backward_data_kernel(MlpArgs a, const __nv_bfloat16* __restrict__ pack_n, int64_t n,
                             const float* __restrict__ zs, const float* __restrict__ dout,
                             float* __restrict__ dzs) {
    extern __shared__ __align__(16) uint8_t smem[];
    const int op = mlp_out_pad(a.out);
    __nv_bfloat16* N4 = reinterpret_cast<__nv_bfloat16*>(smem);     // [op][128] (W4 as stored)
    __nv_bfloat16* N3 = N4 + op * kMlpHidden;                       // [128][128]
    __nv_bfloat16* N2 = N3 + kMlpHidden * kMlpHidden;               // [128][128]
    float* G = reinterpret_cast<float*>(N2 + kMlpHidden * kMlpHidden);  // [kR][128] grad in
    float* D = G + kR * kMlpHidden;                                     // [kR][128] grad out
    copy16(N4, pack_n, (op * kMlpHidden + 2 * kMlpHidden * kMlpHidden) * 2);
    const int64_t r_base = (int64_t)blockIdx.x * kR;
    for (int idx = threadIdx.x; idx < kR * op; idx += blockDim.x) {
        const int r = idx / op;
        const int64_t rr = r_base + r;
        G[idx] = rr < n ? dout[rr * op + (idx - r * op)] : 0.0f;
    }
    __syncthreads();
    const int t = threadIdx.x, c0 = 4 * (t & 31), r0 = 4 * (t >> 5);
    const __nv_bfloat16* Ns[3] = {N4, N3, N2};
    float acc[4][4];
    int kred = op;
    for (int s = 0; s < 3; ++s) {
        const int l = 2 - s;  // hidden layer index of z being differentiated
        const float* src = (s & 1) ? D : G;
        float* dst = (s & 1) ? G : D;
        tile_product(src, (s == 0) ? op : kMlpHidden, Ns[s], kMlpHidden, kred, acc);
        __syncthreads();
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const int64_t rr = r_base + r0 + i;
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                float g = 0.0f;
                if (rr < n) {
                    g = acc[i][j] * gelu_grad(zs[(rr * 3 + l) * kMlpHidden + c0 + j]);
                    dzs[(rr * 3 + l) * kMlpHidden + c0 + j] = g;
                }
                dst[(r0 + i) * kMlpHidden + c0 + j] = g;
            }
        }
        __syncthreads();
        kred = kMlpHidden;
    }
}

// Work item (blockIdx.y): layer l (0..3) and a chunk of 16 output units; the
// rows of the batch are split over blockIdx.x.
__global__ void __launch_bounds__(kThreads)
    mlp_backward_weight_kernel(MlpArgs a, const float* __restrict__ x,
                               const int32_t* __restrict__ rows, int64_t n,
                               const float* __restrict__ zs, const float* __restrict__ dzs,
                               const float* __restrict__ dout, float* __restrict__ grad,
                               int rows_per_split) {
    __shared__ float Hs[kR][kMlpHidden + 1];
    __shared__ float Ds[kR][17];
    const MlpLayout L = mlp_layout(a.in, a.out);
    const int op = mlp_out_pad(a.out);
    const int nch_h = kMlpHidden / 16;
    int item = blockIdx.y, l, ch;
    if (item < 3 * nch_h) { l = item / nch_h; ch = item - l * nch_h; }
    else { l = 3; ch = item - 3 * nch_h; }
    const int nout = l < 3 ? kMlpHidden : a.out;
    const int kin = l == 0 ? a.in : kMlpHidden;
    const int c_lo = ch * 16;
    const int t = threadIdx.x, cl = t >> 4, k0 = (t & 15) * 8;
    float acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    float bacc = 0.0f;
    const int64_t r_begin = (int64_t)blockIdx.x * rows_per_split;
    const int64_t r_end = min(n, r_begin + rows_per_split);
    for (int64_t rb = r_begin; rb < r_end; rb += kR) {
        __syncthreads();
        for (int idx = t; idx < kR * kin; idx += kThreads) {
            const int r = idx / kin, k = idx - (idx / kin) * kin;
            const int64_t rr = rb + r;
            float h = 0.0f;
            if (rr < r_end) {
                if (l == 0) h = bf16r(x[(int64_t)(rows ? rows[rr] : rr) * a.in + k]);
                else h = bf16r(gelu(zs[(rr * 3 + (l - 1)) * kMlpHidden + k]));
            }
            Hs[r][k] = h;
        }
        for (int idx = t; idx < kR * 16; idx += kThreads) {
            const int r = idx >> 4, c = c_lo + (idx & 15);
            const int64_t rr = rb + r;
            float d = 0.0f;
            if (rr < r_end && c < nout)
                d = l < 3 ? dzs[(rr * 3 + l) * kMlpHidden + c] : dout[rr * op + c];
            Ds[r][idx & 15] = d;
        }
        __syncthreads();
        for (int r = 0; r < kR; ++r) {
            const float d = Ds[r][cl];
#pragma unroll
            for (int q = 0; q < 8; ++q) acc[q] = fmaf(d, Hs[r][(k0 + q) % kMlpHidden], acc[q]);
            bacc += d;
        }
    }
    const int c = c_lo + cl;
    if (c >= nout) return;
    const int64_t wofs = l == 0 ? L.W1 : l == 1 ? L.W2 : l == 2 ? L.W3 : L.W4;
    const int64_t bofs = l == 0 ? L.b1 : l == 1 ? L.b2 : l == 2 ? L.b3 : L.b4;
#pragma unroll
    for (int q = 0; q < 8; ++q)
        if (k0 + q < kin) atomicAdd(&grad[wofs + (int64_t)c * kin + k0 + q], acc[q]);
    if ((t & 15) == 0) atomicAdd(&grad[bofs + c], bacc);
}

__global__ void mlp_adam_kernel(float* __restrict__ p, float* __restrict__ m, float* __restrict__ v,
                                const float* __restrict__ g, int64_t P, float lr, float b1, float b2,
                                float eps, float bc1, float bc2) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P) return;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.0f - b1) * gi;
    const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi / bc1) / (sqrtf(vi / bc2) + eps);
}

size_t mlp_forward_smem(int in, int out) {
    const int op = mlp_out_pad(out);
    return (size_t)(in * kMlpHidden + 2 * kMlpHidden * kMlpHidden + kMlpHidden * op) * 2 +
           (size_t)(kR * in + 2 * kR * kMlpHidden) * 4;
}
size_t mlp_backward_smem(int out) {
    const int op = mlp_out_pad(out);
    return (size_t)(op * kMlpHidden + 2 * kMlpHidden * kMlpHidden) * 2 +
           (size_t)(2 * kR * kMlpHidden) * 4;
}

size_t mlp_pack_elems(int in, int out) {
    const int op = mlp_out_pad(out);
    return (size_t)in * kMlpHidden + 2 * kMlpHidden * kMlpHidden + (size_t)kMlpHidden * op +
           (size_t)op * kMlpHidden + 2 * kMlpHidden * kMlpHidden;
}

void launch_mlp_pack(const MlpArgs& a, void* pack, cudaStream_t st) {
    __nv_bfloat16* pt = static_cast<__nv_bfloat16*>(pack);
    __nv_bfloat16* pn = pt + (size_t)a.in * kMlpHidden + 2 * kMlpHidden * kMlpHidden +
                        (size_t)kMlpHidden * mlp_out_pad(a.out);
    mlp_pack_kernel<<<148, 256, 0, st>>>(a, pt, pn);
    count_launch();
}

static void set_smem_attrs(int in, int out) {
    static int done_in = -1, done_out = -1;
    if (done_in == in && done_out == out) return;
    cudaFuncSetAttribute(mlp_forward_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)mlp_forward_smem(in, out));
    cudaFuncSetAttribute(mlp_backward_data_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)mlp_backward_smem(out));
    done_in = in;
    done_out = out;
}

void launch_mlp_forward(const MlpArgs& a, const void* pack, const float* x, const int32_t* rows,
                        int64_t n, const float* target, float* out, float* zs, float* dout,
                        double* loss, float gscale, cudaStream_t st) {
    if (n <= 0) return;
    set_smem_attrs(a.in, a.out);
    mlp_forward_kernel<<<(unsigned)((n + kR - 1) / kR), kThreads, mlp_forward_smem(a.in, a.out), st>>>(
        a, static_cast<const __nv_bfloat16*>(pack), x, rows, n, target, out, zs, dout, loss, gscale);
    count_launch();
}

void launch_mlp_backward(const MlpArgs& a, const void* pack, const float* x, const int32_t* rows,
                         int64_t n, const float* zs, const float* dout, float* dzs, float* grad,
                         cudaStream_t st) {
    if (n <= 0) return;
    set_smem_attrs(a.in, a.out);
    const __nv_bfloat16* pn = static_cast<const __nv_bfloat16*>(pack) +
                              (size_t)a.in * kMlpHidden + 2 * kMlpHidden * kMlpHidden +
                              (size_t)kMlpHidden * mlp_out_pad(a.out);
    mlp_backward_data_kernel<<<(unsigned)((n + kR - 1) / kR), kThreads, mlp_backward_smem(a.out),
                               st>>>(a, pn, n, zs, dout, dzs);
    count_launch();
    const int items = 3 * (kMlpHidden / 16) + (a.out + 15) / 16;
    const int rps = 512;
    dim3 grid((unsigned)((n + rps - 1) / rps), (unsigned)items);
    mlp_backward_weight_kernel<<<grid, kThreads, 0, st>>>(a, x, rows, n, zs, dzs, dout, grad, rps);
    count_launch();
}

void launch_mlp_adam(float* p, float* m, float* v, const float* g, int64_t P, float lr, float b1,
                     float b2, float eps, float bc1, float bc2, cudaStream_t st) {
    mlp_adam_kernel<<<(unsigned)((P + 255) / 256), 256, 0, st>>>(p, m, v, g, P, lr, b1, b2, eps,
                                                                 bc1, bc2);
    count_launch();
}

}  // namespace lds
