// Poisson and Gaussian noise for projections, sm_100a.
//
// Same operation as poisson_1d / poisson_gaussian_1d (Common/CUDA/RandomNumberGenerator.cu:
// GeneratePoisson, GeneratePoissonAddGaussian): out[i] = Poisson(in[i]) (+ N(mu, sigma)).
// The reference draws from curand XORWOW states seeded with 1234 per thread of a fixed
// 64-block grid, so its stream depends on the grid; here every element has its own
// counter-based stream, so results depend only on (seed, element index):
//
//   uniforms: Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as easy
//     as 1, 2, 3", SC 2011), key = seed, counter = {i_lo, i_hi, attempt, purpose};
//   Poisson, lambda < 10: inversion by sequential search of the CDF with one uniform;
//   Poisson, lambda >= 10: PTRS transformed rejection (W. Hormann, "The transformed
//     rejection method for generating Poisson random variables", Insurance: Mathematics and
//     Economics 12, 1993), evaluated in FP64 (its acceptance test is a difference of
//     terms of size lambda log lambda);
//   Gaussian: Box-Muller on two uniforms of the purpose-1 counter.
//
// One thread per element, grid-stride; HBM bound (8 bytes per element).

#include <cmath>
#include <cstdint>

#include "philox.cuh"
#include "tigre_internal.h"

namespace tigre {
namespace {

// uniform in (0, 1): 24 random bits at the centre of their cell (exact in FP32)
__device__ __forceinline__ float u01f(uint32_t x) { return ((float)(x >> 8) + 0.5f) * (1.0f / 16777216.0f); }
// uniform in (0, 1) with 53 bits from two words (FP64)
__device__ __forceinline__ double u01d(uint32_t a, uint32_t b) {
    const uint64_t v = ((uint64_t)a << 21) ^ (uint64_t)(b >> 11);   // 53 bits
    return ((double)(v & ((1ull << 53) - 1)) + 0.5) * (1.0 / 9007199254740992.0);
}

struct NoiseArgs {
    const float* in;
    float* out;
    long long n;
    uint32_t k0, k1;   // seed
    float mu, sigma;
    int gaussian;
};

constexpr int kPtrsMaxAttempts = 64;   // acceptance is > 0.9 per attempt

__device__ float poisson_sample(float lam_f, long long i, uint32_t k0, uint32_t k1) {
    if (!(lam_f > 0.f)) return lam_f == 0.f ? 0.f : (lam_f != lam_f ? lam_f : 0.f);   // NaN stays NaN
    const uint32_t ilo = (uint32_t)i, ihi = (uint32_t)((unsigned long long)i >> 32);
    if (lam_f < 10.f) {
        const U4 r = philox4x32_10(U4{ilo, ihi, 0u, 0u}, k0, k1);
        const double u = u01d(r.x, r.y);
        const double lam = (double)lam_f;
        double p = exp(-lam), s = p;
        int k = 0;
        while (u > s && k < 200) {
            ++k;
            p *= lam / (double)k;
            s += p;
        }
        return (float)k;
    }
    const double lam = (double)lam_f;
    const double slam = sqrt(lam), loglam = log(lam);
    const double b = 0.931 + 2.53 * slam;
    const double a = -0.059 + 0.02483 * b;
    const double invalpha = 1.1239 + 1.1328 / (b - 3.4);
    const double vr = 0.9277 - 3.6224 / (b - 2.0);
    for (uint32_t att = 0; att < (uint32_t)kPtrsMaxAttempts; ++att) {
        const U4 r = philox4x32_10(U4{ilo, ihi, att, 0u}, k0, k1);
        const double U = u01d(r.x, r.y) - 0.5;
        const double V = u01d(r.z, r.w);
        const double us = 0.5 - fabs(U);
        const double k = floor((2.0 * a / us + b) * U + lam + 0.43);
        if (us >= 0.07 && V <= vr) return (float)k;
        if (k < 0.0 || (us < 0.013 && V > us)) continue;
        if (log(V) + log(invalpha) - log(a / (us * us) + b) <= -lam + k * loglam - lgamma(k + 1.0)) return (float)k;
    }
    // not reached in practice (probability < 0.1^64): the normal approximation
    const U4 r = philox4x32_10(U4{ilo, ihi, (uint32_t)kPtrsMaxAttempts, 0u}, k0, k1);
    const double z = sqrt(-2.0 * log(u01d(r.x, r.y))) * cos(6.283185307179586 * u01d(r.z, r.w));
    return (float)fmax(0.0, floor(lam + slam * z + 0.5));
}

__global__ void __launch_bounds__(256) noise_kernel(NoiseArgs a) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < a.n;
         i += (long long)gridDim.x * blockDim.x) {
        float v = poisson_sample(__ldg(a.in + i), i, a.k0, a.k1);
        if (a.gaussian) {
            const U4 r = philox4x32_10(U4{(uint32_t)i, (uint32_t)((unsigned long long)i >> 32), 0u, 1u}, a.k0, a.k1);
            const float u1 = u01f(r.x), u2 = u01f(r.y);
            const float z = sqrtf(-2.f * logf(u1)) * cospif(2.f * u2);
            v += fmaf(z, a.sigma, a.mu);
        }
        a.out[i] = v;
    }
}

__global__ void __launch_bounds__(256) philox_kernel(uint32_t* __restrict__ out, long long nblocks, uint32_t c2,
                                                     uint32_t c3, uint32_t k0, uint32_t k1) {
    for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < nblocks;
         j += (long long)gridDim.x * blockDim.x) {
        const U4 r = philox4x32_10(U4{(uint32_t)j, (uint32_t)((unsigned long long)j >> 32), c2, c3}, k0, k1);
        reinterpret_cast<uint4*>(out)[j] = make_uint4(r.x, r.y, r.z, r.w);
    }
}

int grid_for_noise(long long n) { return (int)std::min<long long>((n + 255) / 256, 148LL * 16); }

}  // namespace
}  // namespace tigre

using namespace tigre;

extern "C" {

int tigre_add_noise(const float* d_in, float* d_out, long long n, int gaussian, float mu, float sigma,
                    unsigned long long seed, void* stream) {
    if (n < 0 || (n > 0 && (!d_in || !d_out))) return fail(TIGRE_ERR_BAD_ASSERT, "bad noise arguments");
    if (gaussian && !(sigma >= 0.f)) return fail(TIGRE_ERR_BAD_ASSERT, "noise: sigma must be >= 0");
    if (n == 0) return TIGRE_SUCCESS;
    NoiseArgs a{d_in, d_out, n, (uint32_t)seed, (uint32_t)(seed >> 32), mu, sigma, gaussian ? 1 : 0};
    noise_kernel<<<grid_for_noise(n), 256, 0, (cudaStream_t)stream>>>(a);
    TIGRE_LAUNCHED();
    return TIGRE_SUCCESS;
}

int tigre_philox4x32(unsigned int* d_out, long long nblocks, unsigned long long counter_hi, unsigned long long seed,
                     void* stream) {
    if (nblocks < 0 || (nblocks > 0 && !d_out)) return fail(TIGRE_ERR_BAD_ASSERT, "bad Philox arguments");
    if (((uintptr_t)d_out & 15u) != 0) return fail(TIGRE_ERR_BAD_ASSERT, "Philox output must be 16-byte aligned");
    if (nblocks == 0) return TIGRE_SUCCESS;
    philox_kernel<<<grid_for_noise(nblocks), 256, 0, (cudaStream_t)stream>>>(
        d_out, nblocks, (uint32_t)counter_hi, (uint32_t)(counter_hi >> 32), (uint32_t)seed, (uint32_t)(seed >> 32));
    TIGRE_LAUNCHED();
    return TIGRE_SUCCESS;
}

}  // extern "C"
