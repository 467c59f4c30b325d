// Rademacher probe streams on the device, bit-identical to the host streams:
// each unit (a SNP block of a V-tile) is one std::mt19937_64 stream seeded
// per (root, block start, V-tile start) (make_seed, gwldcore.cpp:452-458),
// whose draws fill the unit's L x V column-major probe block in order,
// z = (draw & 1) ? +1 : -1 (gwldcore.cpp:1702-1706).
//
// The generator is the Mersenne Twister of the C++ standard ([rand.eng.mers]:
// w = 64, n = 312, m = 156, r = 31, a = 0xB5026F5AA96619E9, u = 29,
// d = 0x5555555555555555, s = 17, b = 0x71D67FFFEDA60000, t = 37,
// c = 0xFFF7EEE000000000, l = 43, f = 6364136223846793005).  One CTA runs one
// stream: the 312-word state lives in shared memory, each twist is computed by
// 312 threads in the three dependency phases of the sequential recurrence
// (words 0..155 read only old words; 156..310 read the new words 0..154;
// 311 reads the new words 0 and 155), and each thread tempers one word, so a
// block of 312 consecutive draws is written per round.
#include <cstdint>

#include "lds_internal.h"

namespace lds {

namespace {

constexpr int kN = 312, kM = 156;
constexpr uint64_t kA = 0xB5026F5AA96619E9ULL;
constexpr uint64_t kUpper = 0xFFFFFFFF80000000ULL, kLower = 0x7FFFFFFFULL;
constexpr int kGenThreads = 320;

__device__ __forceinline__ uint64_t twist_word(uint64_t cur, uint64_t next, uint64_t far) {
    const uint64_t y = (cur & kUpper) | (next & kLower);
    return far ^ (y >> 1) ^ ((y & 1ULL) ? kA : 0ULL);
}

__device__ __forceinline__ uint64_t temper(uint64_t y) {
    y ^= (y >> 29) & 0x5555555555555555ULL;
    y ^= (y << 17) & 0x71D67FFFEDA60000ULL;
    y ^= (y << 37) & 0xFFF7EEE000000000ULL;
    y ^= y >> 43;
    return y;
}

__global__ void __launch_bounds__(kGenThreads)
    rademacher_units_kernel(const ProbeUnit* __restrict__ units, int V, double* __restrict__ Z,
                            int64_t ld) {
    __shared__ uint64_t x[kN], nx[kN];
    const ProbeUnit u = units[blockIdx.x];
    const int t = threadIdx.x;
    if (t == 0) {
        x[0] = u.seed;
        for (int i = 1; i < kN; ++i)
            x[i] = 6364136223846793005ULL * (x[i - 1] ^ (x[i - 1] >> 62)) + (uint64_t)i;
    }
    __syncthreads();
    const int64_t total = (int64_t)u.L * V;
    for (int64_t p0 = 0; p0 < total; p0 += kN) {
        if (t < kM) nx[t] = twist_word(x[t], x[t + 1], x[t + kM]);
        __syncthreads();
        if (t >= kM && t < kN - 1) nx[t] = twist_word(x[t], x[t + 1], nx[t - kM]);
        __syncthreads();
        if (t == kN - 1) nx[t] = twist_word(x[t], nx[0], nx[t - kM]);
        __syncthreads();
        if (t < kN) {
            x[t] = nx[t];
            const int64_t p = p0 + t;
            if (p < total) {
                const int64_t c = p / u.L, r = p - c * u.L;
                Z[c * ld + u.row0 + r] = (temper(nx[t]) & 1ULL) ? 1.0 : -1.0;
            }
        }
        __syncthreads();
    }
}

}  // namespace

void launch_rademacher_units(const ProbeUnit* units, int64_t n_units, int V, double* Z, int64_t ld,
                             cudaStream_t st) {
    if (n_units <= 0 || V <= 0) return;
    rademacher_units_kernel<<<(unsigned)n_units, kGenThreads, 0, st>>>(units, V, Z, ld);
    count_launch();
}

}  // namespace lds
