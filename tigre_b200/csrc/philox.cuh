// Philox4x32-10 counter-based generator (Salmon, Moraes, Dror, Shaw, "Parallel random numbers:
// as easy as 1, 2, 3", SC 2011): multipliers 0xD2511F53 / 0xCD9E8D57, key increments
// 0x9E3779B9 / 0xBB67AE85, the published constants of the paper.  Shared by the noise
// generator and the stochastic rounding of 16-bit volume updates.
#pragma once

#include <cstdint>

namespace tigre {

struct U4 {
    uint32_t x, y, z, w;
};

__host__ __device__ __forceinline__ void mulhilo(uint32_t a, uint32_t b, uint32_t& hi, uint32_t& lo) {
    const uint64_t p = (uint64_t)a * (uint64_t)b;
    hi = (uint32_t)(p >> 32);
    lo = (uint32_t)p;
}

__host__ __device__ __forceinline__ U4 philox4x32_10(U4 c, uint32_t k0, uint32_t k1) {
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        if (r > 0) {
            k0 += 0x9E3779B9u;
            k1 += 0xBB67AE85u;
        }
        uint32_t hi0, lo0, hi1, lo1;
        mulhilo(0xD2511F53u, c.x, hi0, lo0);
        mulhilo(0xCD9E8D57u, c.z, hi1, lo1);
        c = U4{hi1 ^ c.y ^ k0, lo1, hi0 ^ c.w ^ k1, lo0};
    }
    return c;
}

}  // namespace tigre
