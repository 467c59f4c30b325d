// Device helpers shared by the LD-score kernels: 2-bit BED decode, int8
// tensor-core fragments, hashing.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace lds {

// ---------------------------------------------------------------------------
// BED 2-bit decode (PLINK SNP-major; genotype.cpp:135-140).  Code -> value:
// 00 -> 0, 01 -> missing, 10 -> 1, 11 -> 2.  We produce two int8 planes per
// call: G (value, missing -> 0) and O (observed mask).  Both are exact
// integers, so tensor-core products of them with int8 operands are exact.
//
// The 8 codes in the low 16 bits of `w` are spread to one nibble each, then
// `prmt` uses the nibble as an index into a 4-byte lookup table.
// ---------------------------------------------------------------------------
constexpr uint32_t kLutG = 0x02010000u;  // bytes: g(00)=0 g(01)=0 g(10)=1 g(11)=2
constexpr uint32_t kLutO = 0x01010001u;  // bytes: o(00)=1 o(01)=0 o(10)=1 o(11)=1

__device__ __forceinline__ uint32_t spread_codes8(uint32_t w16) {
    uint32_t y = (w16 | (w16 << 8)) & 0x00FF00FFu;
    y = (y | (y << 4)) & 0x0F0F0F0Fu;
    return (y | (y << 2)) & 0x33333333u;
}

// Decode 8 codes (2 packed bytes) -> 8 G bytes (g0: samples 0-3, g1: 4-7)
// and 8 O bytes.
__device__ __forceinline__ void decode8(uint32_t w16, uint32_t& g0, uint32_t& g1,
                                        uint32_t& o0, uint32_t& o1) {
    const uint32_t y = spread_codes8(w16);
    g0 = __byte_perm(kLutG, 0u, y);
    g1 = __byte_perm(kLutG, 0u, y >> 16);
    o0 = __byte_perm(kLutO, 0u, y);
    o1 = __byte_perm(kLutO, 0u, y >> 16);
}

// Decode one packed byte (4 codes) -> 4 G bytes and 4 O bytes.
__device__ __forceinline__ void decode4(uint32_t b8, uint32_t& g, uint32_t& o) {
    const uint32_t y = spread_codes8(b8 & 0xFFu);
    g = __byte_perm(kLutG, 0u, y);
    o = __byte_perm(kLutO, 0u, y);
}

// 4x4 byte transpose: rows a,b,c,d (4 bytes each) -> columns.
__device__ __forceinline__ void transpose4x4(uint32_t a, uint32_t b, uint32_t c, uint32_t d,
                                             uint32_t& c0, uint32_t& c1, uint32_t& c2,
                                             uint32_t& c3) {
    const uint32_t t0 = __byte_perm(a, b, 0x5140);
    const uint32_t t1 = __byte_perm(a, b, 0x7362);
    const uint32_t t2 = __byte_perm(c, d, 0x5140);
    const uint32_t t3 = __byte_perm(c, d, 0x7362);
    c0 = __byte_perm(t0, t2, 0x5410);
    c1 = __byte_perm(t0, t2, 0x7632);
    c2 = __byte_perm(t1, t3, 0x5410);
    c3 = __byte_perm(t1, t3, 0x7632);
}

// ---------------------------------------------------------------------------
// Warp-level int8 MMA (m16n8k32, s8 x s8 -> s32) and ldmatrix fragment loads.
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void ldsm_x4(uint32_t addr, uint32_t& r0, uint32_t& r1, uint32_t& r2,
                                        uint32_t& r3) {
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];\n"
                 : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3)
                 : "r"(addr));
}

__device__ __forceinline__ void ldsm_x2(uint32_t addr, uint32_t& r0, uint32_t& r1) {
    asm volatile("ldmatrix.sync.aligned.m8n8.x2.shared.b16 {%0,%1}, [%2];\n"
                 : "=r"(r0), "=r"(r1)
                 : "r"(addr));
}

__device__ __forceinline__ void mma_s8(int (&d)[4], const uint32_t (&a)[4], uint32_t b0,
                                       uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k32.row.col.s32.s8.s8.s32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
        "{%8,%9}, {%0,%1,%2,%3};\n"
        : "+r"(d[0]), "+r"(d[1]), "+r"(d[2]), "+r"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// cp.async 16 bytes global -> shared; `bytes` < 16 zero-fills the rest.
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem, int bytes = 16) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(smem_u32(smem)),
                 "l"(gmem), "r"(bytes));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n"); }

// ---------------------------------------------------------------------------
// splitmix64 finaliser (genotype.cpp:106-112) and the synthetic generator's
// counter-based draws (bedfile.py).
// ---------------------------------------------------------------------------
__host__ __device__ __forceinline__ uint64_t mix64(uint64_t x) {
    x += 0x9e3779b97f4a7c15ULL;
    x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ULL;
    x = (x ^ (x >> 27)) * 0x94d049bb133111ebULL;
    return x ^ (x >> 31);
}

// Odd 64-bit weight of (bin k, probe v) in the phase-2 product checksums.
__host__ __device__ __forceinline__ uint64_t check_weight(int k, int v) {
    return mix64(((uint64_t)(uint32_t)k << 32) | (uint64_t)(uint32_t)v) | 1ULL;
}

}  // namespace lds
