// Surrogate network of the learned control variate: in -> 128 -> 128 -> 128 -> out,
// GELU (erf form) after each hidden layer, trained by mean squared error.
//
// Weights are kept in FP32 (Adam's master copy) and enter every product
// rounded to BF16; hidden activations are rounded to BF16 where they feed the
// next product; all sums accumulate in FP32.  Four kernels make one training
// step over a mini-batch of gathered rows:
//   mlp_forward_kernel      32 rows per CTA, all four layers in shared memory;
//                           the products run on the tensor cores
//                           (mma.sync m16n8k16, BF16 x BF16 -> FP32), one
//                           16 x 32 output tile per warp; stores the
//                           pre-activations z1..z3 and the loss gradient of the
//                           outputs;
//   mlp_backward_data_kernel  dZ_l = (dZ_{l+1} W_{l+1}) * gelu'(z_l), l = 3, 2, 1,
//                           on the tensor cores too: the FP32 gradients enter as
//                           a BF16 pair hi + lo (two products), so they keep
//                           16 significant bits against the BF16 weights;
//   mlp_backward_weight_kernel dW_l = dZ_l^T H_{l-1}, db_l = sum dZ_l over rows
//                           (row-split, FP32 atomics into the gradient);
//   mlp_adam_kernel         Adam with bias correction on the FP32 master weights.
// Shared-memory operand rows carry 8 BF16 of padding, so the fragment loads of
// the 8 rows a quad group touches fall in distinct banks.
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

constexpr int kPad = 8;              // BF16 of padding per shared-memory operand row
constexpr int kLdH = kMlpHidden + kPad;  // row stride of 128-wide operands

__host__ __device__ inline int round16(int x) { return (x + 15) & ~15; }
__host__ __device__ inline int ld_in(int in) { return round16(in) + kPad; }
__host__ __device__ inline int ld_out(int out) { return round16(out) + kPad; }

__device__ __forceinline__ uint32_t ld32(const __nv_bfloat16* p) {
    return *reinterpret_cast<const uint32_t*>(p);
}

__device__ __forceinline__ void mma_bf16(float (&d)[4], const uint32_t (&a)[4], uint32_t b0,
                                         uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
        "{%8,%9}, {%0,%1,%2,%3};"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// acc[nt] (+)= the warp's 16 x 8 tiles (rows row0.., columns col0 + 8 nt..) of
// A B over K (a multiple of 16): A row-major BF16 [rows][lda], B stored per
// output column with K contiguous, BF16 [cols][ldb]; tiles at or beyond ncols
// are skipped.  With A2 (the low halves of a split FP32 operand) both halves
// are multiplied into the same accumulators.
__device__ __forceinline__ void warp_mma4(const __nv_bfloat16* A, const __nv_bfloat16* A2, int lda,
                                          int row0, const __nv_bfloat16* B, int ldb, int col0,
                                          int ncols, int K, float (&acc)[4][4]) {
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
#pragma unroll
    for (int nt = 0; nt < 4; ++nt)
#pragma unroll
        for (int e = 0; e < 4; ++e) acc[nt][e] = 0.0f;
    for (int k = 0; k < K; k += 16) {
        const int ao = (row0 + g) * lda + k + 2 * t;
        const uint32_t a[4] = {ld32(A + ao), ld32(A + ao + 8 * lda), ld32(A + ao + 8),
                               ld32(A + ao + 8 * lda + 8)};
        uint32_t a2[4] = {0, 0, 0, 0};
        if (A2) {
            a2[0] = ld32(A2 + ao);
            a2[1] = ld32(A2 + ao + 8 * lda);
            a2[2] = ld32(A2 + ao + 8);
            a2[3] = ld32(A2 + ao + 8 * lda + 8);
        }
#pragma unroll
        for (int nt = 0; nt < 4; ++nt) {
            const int n = col0 + 8 * nt;
            if (n >= ncols) continue;
            const __nv_bfloat16* br = B + (n + g) * ldb + k + 2 * t;
            const uint32_t b0 = ld32(br), b1 = ld32(br + 8);
            mma_bf16(acc[nt], a, b0, b1);
            if (A2) mma_bf16(acc[nt], a2, b0, b1);
        }
    }
}

// Element e (0..3) of the warp's fragment nt: row and column of C.
__device__ __forceinline__ int frag_row(int row0, int e) {
    return row0 + ((threadIdx.x & 31) >> 2) + 8 * (e >> 1);
}
__device__ __forceinline__ int frag_col(int col0, int nt, int e) {
    return col0 + 8 * nt + 2 * (threadIdx.x & 3) + (e & 1);
}

// A FP32 value as a BF16 pair hi + lo (hi + lo within 2^-16 relative of v).
__device__ __forceinline__ void split_bf16(float v, __nv_bfloat16& hi, __nv_bfloat16& lo) {
    hi = __float2bfloat16_rn(v);
    lo = __float2bfloat16_rn(v - __bfloat162float(hi));
}

// Copy `bytes` (a multiple of 16) from global to shared memory.
__device__ __forceinline__ void copy16(void* dst, const void* src, int bytes) {
    const uint4* s = reinterpret_cast<const uint4*>(src);
    uint4* d = reinterpret_cast<uint4*>(dst);
    for (int i = threadIdx.x; i < bytes / 16; i += blockDim.x) d[i] = s[i];
}

}  // namespace mlp

using namespace mlp;

// BF16 copies of the weights in the operand layouts of the products, made
// once per step (rows padded to the shared-memory strides, padding zero):
//   forward  F1 [128][ld_in] = W1, F2, F3 [128][kLdH] = W2, W3,
//            F4 [round16(out)][kLdH] = W4 (rows >= out zero);
//   backward B4 [128][ld_out] = W4^T, B3, B2 [128][kLdH] = W3^T, W2^T.
__global__ void mlp_pack_kernel(MlpArgs a, __nv_bfloat16* __restrict__ pack) {
    const MlpLayout L = mlp_layout(a.in, a.out);
    const int H = kMlpHidden, li = ld_in(a.in), lo = ld_out(a.out), o16 = round16(a.out);
    const int64_t nF1 = (int64_t)H * li, nH = (int64_t)H * kLdH, nF4 = (int64_t)o16 * kLdH;
    const int64_t nB4 = (int64_t)H * lo;
    const int64_t total = nF1 + 2 * nH + nF4 + nB4 + 2 * nH;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
         i += (int64_t)gridDim.x * blockDim.x) {
        int64_t r = i;
        float v = 0.0f;
        if (r < nF1) {
            const int c = (int)(r / li), k = (int)(r % li);
            if (k < a.in) v = a.params[L.W1 + (int64_t)c * a.in + k];
        } else if ((r -= nF1) < 2 * nH) {
            const int64_t base = r < nH ? L.W2 : L.W3;
            const int64_t q = r % nH;
            const int c = (int)(q / kLdH), k = (int)(q % kLdH);
            if (k < H) v = a.params[base + (int64_t)c * H + k];
        } else if ((r -= 2 * nH) < nF4) {
            const int c = (int)(r / kLdH), k = (int)(r % kLdH);
            if (c < a.out && k < H) v = a.params[L.W4 + (int64_t)c * H + k];
        } else if ((r -= nF4) < nB4) {
            const int n = (int)(r / lo), k = (int)(r % lo);  // B4[n][k] = W4[k][n]
            if (k < a.out) v = a.params[L.W4 + (int64_t)k * H + n];
        } else {
            r -= nB4;
            const int64_t base = r < nH ? L.W3 : L.W2;
            const int64_t q = r % nH;
            const int n = (int)(q / kLdH), k = (int)(q % kLdH);  // W^T[n][k] = W[k][n]
            if (k < H) v = a.params[base + (int64_t)k * H + n];
        }
        pack[i] = __float2bfloat16_rn(v);
    }
}

__global__ void __launch_bounds__(kThreads)
    mlp_forward_kernel(MlpArgs a, const __nv_bfloat16* __restrict__ pack,
                       const float* __restrict__ x, const int32_t* __restrict__ rows, int64_t n,
                       const float* __restrict__ target, float* __restrict__ out,
                       float* __restrict__ zs, float* __restrict__ dout, double* __restrict__ loss,
                       float gscale) {
    extern __shared__ __align__(16) uint8_t smem[];
    const MlpLayout L = mlp_layout(a.in, a.out);
    const int op = mlp_out_pad(a.out), li = ld_in(a.in), o16 = round16(a.out);
    __nv_bfloat16* F1 = reinterpret_cast<__nv_bfloat16*>(smem);    // [128][li]
    __nv_bfloat16* F2 = F1 + kMlpHidden * li;                       // [128][kLdH]
    __nv_bfloat16* F3 = F2 + kMlpHidden * kLdH;                     // [128][kLdH]
    __nv_bfloat16* F4 = F3 + kMlpHidden * kLdH;                     // [o16][kLdH]
    __nv_bfloat16* X = F4 + o16 * kLdH;                             // [kR][li]
    __nv_bfloat16* H1 = X + kR * li;                                // [kR][kLdH]
    __nv_bfloat16* H2 = H1 + kR * kLdH;                             // [kR][kLdH]
    __shared__ float red[kThreads / 32];

    copy16(F1, pack, (kMlpHidden * li + 2 * kMlpHidden * kLdH + o16 * kLdH) * 2);
    const int64_t r_base = (int64_t)blockIdx.x * kR;
    for (int idx = threadIdx.x; idx < kR * li; idx += blockDim.x) {
        const int r = idx / li, k = idx - (idx / li) * li;
        const int64_t rr = r_base + r;
        float v = 0.0f;
        if (rr < n && k < a.in) v = x[(int64_t)(rows ? rows[rr] : rr) * a.in + k];
        X[idx] = __float2bfloat16_rn(v);
    }
    __syncthreads();

    const int t = threadIdx.x, w = t >> 5;
    const int row0 = 16 * (w & 1), col0 = 32 * (w >> 1);
    float acc[4][4];
    const float* bias[3] = {a.params + L.b1, a.params + L.b2, a.params + L.b3};
    const __nv_bfloat16* Ws[3] = {F1, F2, F3};
    const __nv_bfloat16* in_act[3] = {X, H1, H2};
    __nv_bfloat16* out_act[3] = {H1, H2, H1};
    const int lda[3] = {li, kLdH, kLdH};
    const int kin[3] = {round16(a.in), kMlpHidden, kMlpHidden};
    for (int l = 0; l < 3; ++l) {
        warp_mma4(in_act[l], nullptr, lda[l], row0, Ws[l], lda[l], col0, kMlpHidden, kin[l], acc);
        __syncthreads();  // layer 3 writes H1, which layer 2 read
#pragma unroll
        for (int nt = 0; nt < 4; ++nt)
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                const int r = frag_row(row0, e), c = frag_col(col0, nt, e);
                const int64_t rr = r_base + r;
                const float z = acc[nt][e] + bias[l][c];
                if (zs && rr < n) zs[(rr * 3 + l) * kMlpHidden + c] = z;
                out_act[l][r * kLdH + c] = __float2bfloat16_rn(gelu(z));
            }
        __syncthreads();
    }
    warp_mma4(H1, nullptr, kLdH, row0, F4, kLdH, col0, o16, kMlpHidden, acc);
    float lsum = 0.0f;
#pragma unroll
    for (int nt = 0; nt < 4; ++nt)
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            const int r = frag_row(row0, e), c = frag_col(col0, nt, e);
            const int64_t rr = r_base + r;
            if (rr >= n || c >= op) continue;
            if (c >= a.out) {  // padding columns of dout read as zero in backward
                if (dout) dout[rr * op + c] = 0.0f;
                continue;
            }
            const float o = acc[nt][e] + a.params[L.b4 + c];
            if (out) out[rr * a.out + c] = o;
            if (target) {
                const float d = o - target[(int64_t)(rows ? rows[rr] : rr) * a.out + c];
                if (dout) dout[rr * op + c] = 2.0f * d * gscale;
                lsum += d * d;
            }
        }
    if (loss) {
        for (int o = 16; o; o >>= 1) lsum += __shfl_xor_sync(0xffffffffu, lsum, o);
        if ((t & 31) == 0) red[t >> 5] = lsum;
        __syncthreads();
        if (t == 0) {
            double sum = 0.0;
            for (int q = 0; q < kThreads / 32; ++q) sum += red[q];
            atomicAdd(loss, sum * (double)gscale);
        }
    }
}

__global__ void __launch_bounds__(kThreads)
    mlp_backward_data_kernel(MlpArgs a, const __nv_bfloat16* __restrict__ pack_b, int64_t n,
                             const float* __restrict__ zs, const float* __restrict__ dout,
                             float* __restrict__ dzs) {
    extern __shared__ __align__(16) uint8_t smem[];
    const int op = mlp_out_pad(a.out), lo = ld_out(a.out);
    __nv_bfloat16* B4 = reinterpret_cast<__nv_bfloat16*>(smem);     // [128][lo] = W4^T
    __nv_bfloat16* B3 = B4 + kMlpHidden * lo;                       // [128][kLdH] = W3^T
    __nv_bfloat16* B2 = B3 + kMlpHidden * kLdH;                     // [128][kLdH] = W2^T
    __nv_bfloat16* A0 = B2 + kMlpHidden * kLdH;                     // [2][kR][kLdH] hi | lo
    __nv_bfloat16* A1 = A0 + 2 * kR * kLdH;                         // [2][kR][kLdH] hi | lo
    copy16(B4, pack_b, (kMlpHidden * lo + 2 * kMlpHidden * kLdH) * 2);
    const int64_t r_base = (int64_t)blockIdx.x * kR;
    for (int idx = threadIdx.x; idx < kR * lo; idx += blockDim.x) {
        const int r = idx / lo, k = idx - r * lo;
        const int64_t rr = r_base + r;
        const float g = (rr < n && k < op) ? dout[rr * op + k] : 0.0f;
        split_bf16(g, A0[r * lo + k], A0[kR * kLdH + r * lo + k]);
    }
    __syncthreads();
    const int t = threadIdx.x, w = t >> 5;
    const int row0 = 16 * (w & 1), col0 = 32 * (w >> 1);
    const __nv_bfloat16* Bs[3] = {B4, B3, B2};
    float acc[4][4];
    for (int s = 0; s < 3; ++s) {
        const int l = 2 - s;  // hidden layer index of z being differentiated
        __nv_bfloat16* src = (s & 1) ? A1 : A0;
        __nv_bfloat16* dst = (s & 1) ? A0 : A1;
        const int ld = s == 0 ? lo : kLdH;
        warp_mma4(src, src + kR * kLdH, ld, row0, Bs[s], ld, col0, kMlpHidden,
                  s == 0 ? round16(a.out) : kMlpHidden, acc);
        __syncthreads();
#pragma unroll
        for (int nt = 0; nt < 4; ++nt)
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                const int r = frag_row(row0, e), c = frag_col(col0, nt, e);
                const int64_t rr = r_base + r;
                float g = 0.0f;
                if (rr < n) {
                    g = acc[nt][e] * gelu_grad(zs[(rr * 3 + l) * kMlpHidden + c]);
                    dzs[(rr * 3 + l) * kMlpHidden + c] = g;
                }
                if (s < 2) split_bf16(g, dst[r * kLdH + c], dst[kR * kLdH + r * kLdH + c]);
            }
        __syncthreads();
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
    return (size_t)(kMlpHidden * ld_in(in) + 2 * kMlpHidden * kLdH + round16(out) * kLdH +
                    kR * ld_in(in) + 2 * kR * kLdH) * 2;
}
size_t mlp_backward_smem(int out) {
    return (size_t)(kMlpHidden * ld_out(out) + 2 * kMlpHidden * kLdH + 4 * kR * kLdH) * 2;
}

static size_t pack_forward_elems(int in, int out) {
    return (size_t)kMlpHidden * ld_in(in) + 2 * kMlpHidden * kLdH + (size_t)round16(out) * kLdH;
}

size_t mlp_pack_elems(int in, int out) {
    return pack_forward_elems(in, out) + (size_t)kMlpHidden * ld_out(out) +
           2 * kMlpHidden * kLdH;
}

void launch_mlp_pack(const MlpArgs& a, void* pack, cudaStream_t st) {
    mlp_pack_kernel<<<148, 256, 0, st>>>(a, static_cast<__nv_bfloat16*>(pack));
    count_launch();
}

// The kernels' shared-memory limits, set once per device for the largest
// network the C ABI admits (LDS_MLP_MAX_IN inputs, LDS_MLP_MAX_OUT outputs).
static void set_smem_attrs(int, int) {
    static std::atomic<unsigned long long> done{0};
    once_per_device(done, [] {
        cudaFuncSetAttribute(mlp_forward_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)mlp_forward_smem(128, 64));
        cudaFuncSetAttribute(mlp_backward_data_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)mlp_backward_smem(64));
    });
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
    const __nv_bfloat16* pn =
        static_cast<const __nv_bfloat16*>(pack) + pack_forward_elems(a.in, a.out);
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
