// tcgen05 / TMA / mbarrier helpers shared by the tensor-core kernels
// (inline PTX for sm_100a).
#pragma once
#include <cstdint>
#include <cuda.h>
#include <cuda_runtime.h>

#include "lds_device.cuh"
#include "lds_internal.h"

namespace lds {
namespace umma {

// Each try_wait suspends the thread for at most kSuspendNs (it returns as
// soon as the phase completes), so a wait gives up after at most about
// kWaitLimit * kSuspendNs = 6.7 s.
constexpr long long kWaitLimit = 1LL << 25;
#ifndef LDS_SUSPEND_NS
#define LDS_SUSPEND_NS 200
#endif
constexpr uint32_t kSuspendNs = LDS_SUSPEND_NS;

// The iteration limit in force: one copy per translation unit and device,
// kWaitLimit unless lds_set_wait_limit() changed it.  Each file that includes
// this header registers a setter for its copy (WaitLimitRegistrar below).
static __constant__ long long c_wait_limit = kWaitLimit;

__device__ __forceinline__ long long wait_limit() { return c_wait_limit; }

// Host side: set this translation unit's copy on the current device.
static inline cudaError_t set_wait_limit_here(long long iters) {
    return cudaMemcpyToSymbol(c_wait_limit, &iters, sizeof iters);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.shared::cta.b64 st, [%0];\n\t}" ::"r"(
        smem_u32(bar)));
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile(
        "{\n\t.reg .b64 st;\n\tmbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n\t}" ::"r"(
            smem_u32(bar)),
        "r"(bytes));
}
// Bounded wait for the phase with the given parity.  Returns false on timeout.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
    const uint32_t addr = smem_u32(bar);
    const long long limit = wait_limit();
    for (long long i = 0; i < limit; ++i) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(addr), "r"(parity), "n"(kSuspendNs)
            : "memory");
        if (done) return true;
    }
    return false;
}

__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int x, int y,
                                            uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes "
        "[%0], [%1, {%2, %3}], [%4];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_u32(bar))
        : "memory");
}

// Bulk copy of `bytes` contiguous bytes (16-byte aligned, a multiple of 16)
// into this CTA's shared memory, completing on `bar`.
__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes,
                                          uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
            "r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(src)), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

// UMMA shared-memory descriptor: K-major, SWIZZLE_128B, 8-row groups 1024 B
// apart (SBO), version 1 (sm100), base offset 0 (tiles are 1024-aligned).
__device__ __forceinline__ uint64_t sw128_desc(const void* smem) {
    const uint64_t a = (uint64_t)((smem_u32(smem) >> 4) & 0x3FFF);
    return a | (1ULL << 16) | ((uint64_t)(1024 >> 4) << 32) | (1ULL << 46) | (2ULL << 61);
}

// Instruction descriptor: kind::i8, D = s32, A = s8, B = s8, both K-major.
__host__ __device__ constexpr uint32_t idesc_i8(int M, int N) {
    return (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) |
           ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void umma_i8(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc,
                                        uint32_t idesc, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate));
}

__device__ __forceinline__ void umma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, int (&r)[32]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,"
        "%14,%15,%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
          "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]),
          "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
          "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]),
          "=r"(r[31])
        : "r"(taddr));
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, int (&r)[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,"
        "%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
          "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
}

__device__ __forceinline__ void tmem_wait_ld() {
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_before() {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void fence_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// MN-major SWIZZLE_128B descriptor: 128-byte rows run along M (one M block of
// 128 int8 elements), 8-row groups along K are 1024 B apart (SBO).
__device__ __forceinline__ uint64_t sw128_desc_mn(const void* smem) {
    const uint64_t a = (uint64_t)((smem_u32(smem) >> 4) & 0x3FFF);
    return a | ((uint64_t)(8192 >> 4) << 16) | ((uint64_t)(1024 >> 4) << 32) | (1ULL << 46) |
           (2ULL << 61);
}

// Instruction descriptor, kind::i8 with A MN-major (bit 15) and B K-major.
__host__ __device__ constexpr uint32_t idesc_i8_amn(int M, int N) {
    return idesc_i8(M, N) | (1u << 15);
}

// Decode 32 packed bytes (128 codes) of one operand row into the G and O
// rows of two SWIZZLE_128B tiles (row r of the tile, chunk c at c ^ (r & 7)).
__device__ __forceinline__ void decode_row_sw128(uint4 p0, uint4 p1, uint8_t* gRow, uint8_t* oRow,
                                                 int r) {
    const uint32_t words[8] = {p0.x, p0.y, p0.z, p0.w, p1.x, p1.y, p1.z, p1.w};
#pragma unroll
    for (int c = 0; c < 8; ++c) {
        uint32_t g0, g1, g2, g3, o0, o1, o2, o3;
        decode8(words[c] & 0xFFFFu, g0, g1, o0, o1);
        decode8(words[c] >> 16, g2, g3, o2, o3);
        const int off = ((c ^ (r & 7)) << 4);
        *reinterpret_cast<uint4*>(gRow + off) = make_uint4(g0, g1, g2, g3);
        *reinterpret_cast<uint4*>(oRow + off) = make_uint4(o0, o1, o2, o3);
    }
}

// Index checks of the bounds-checked build (-DLDS_CHECKED): a failed check
// records its code in the library's device error word (first failure wins)
// and evaluates false, and the caller skips the access instead of trapping.
// In ordinary builds in_range is true and the checks compile away.
#ifdef LDS_CHECKED
static __constant__ unsigned* c_checked_err = nullptr;
__device__ __forceinline__ bool in_range(bool ok, unsigned code) {
    if (!ok && c_checked_err) atomicCAS(c_checked_err, 0u, code);
    return ok;
}
static inline cudaError_t set_checked_err_here(unsigned* p) {
    return cudaMemcpyToSymbol(c_checked_err, &p, sizeof p);
}
struct CheckedErrRegistrar {
    CheckedErrRegistrar() { register_checked_err_setter(&set_checked_err_here); }
};
static CheckedErrRegistrar g_checked_err_registrar;
#else
__device__ __forceinline__ bool in_range(bool, unsigned) { return true; }
#endif

// Registers set_wait_limit_here of the including file with the library, so
// that lds_set_wait_limit reaches every copy of c_wait_limit.
struct WaitLimitRegistrar {
    WaitLimitRegistrar() { register_wait_limit_setter(&set_wait_limit_here); }
};
static WaitLimitRegistrar g_wait_limit_registrar;

// The G row only (tiles whose O plane is not needed).
__device__ __forceinline__ void decode_row_sw128_g(uint4 p0, uint4 p1, uint8_t* gRow, int r) {
    const uint32_t words[8] = {p0.x, p0.y, p0.z, p0.w, p1.x, p1.y, p1.z, p1.w};
#pragma unroll
    for (int c = 0; c < 8; ++c) {
        uint32_t g0, g1, g2, g3, o0, o1, o2, o3;
        decode8(words[c] & 0xFFFFu, g0, g1, o0, o1);
        decode8(words[c] >> 16, g2, g3, o2, o3);
        *reinterpret_cast<uint4*>(gRow + ((c ^ (r & 7)) << 4)) = make_uint4(g0, g1, g2, g3);
    }
}

}  // namespace umma
}  // namespace lds
