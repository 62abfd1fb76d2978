// SART-family volume update, sm_100a.
//
//   x[z, y, x] <- max(x[z, y, x] + (lambda / V[y, x]) * bp[z, y, x], 0)
//
// The update of IterativeReconAlg.update_image (Python/tigre/algorithms/iterative_recon_alg.py:
// 389-401: res += lmbda * 1.0 / V * Atb(W * (proj - Ax(res)))) with the nonnegativity clip of
// art_data_minimizing (:344-345), fused into one pass over the volume.  Operation order is the
// reference's numpy expression: t = lambda / V, then t * bp, then x + t * bp, each rounded to
// FP32 (no contraction into an FMA), and the clip keeps NaN as numpy's clip does.
//
// 16-bit storage rounds the FP32 result to nearest (ROUND_NEAREST) or stochastically
// (ROUND_STOCHASTIC), which keeps updates smaller than half a unit in the last place in
// expectation instead of dropping them:
//   BF16: add 16 random bits to the FP32 bit pattern and truncate to the upper half;
//   FP16: take the round-up neighbour hi over the round-down neighbour lo when a 16-bit
//         uniform u = (r + 1/2) / 2^16 is below (v - lo) / (hi - lo).
// Random bits come from Philox4x32-10 with key = seed and counter = {g, z, step_lo, step_hi},
// g the 8-voxel group index within the z plane (voxels 8g .. 8g+7 of the plane); voxel 8g + e
// takes the low (e even) or high (e odd) 16 bits of word e / 2.  They depend only on (seed, step,
// voxel), not on the launch shape.
//
// One thread per 8-voxel group of a z plane.  HBM bound: 2 e + 4 bytes per voxel (e = storage
// bytes: read and write x, read bp); the V plane is re-read from L2 by every z.

#include <cstdint>

#include "philox.cuh"
#include "tigre_internal.h"

namespace tigre {
namespace {

struct SartArgs {
    const float* bp;
    const float* v;
    long long nz, nyx, ngroups;
    float lambda;
    int noneg;
    uint32_t k0, k1, s0, s1;
};

__device__ __forceinline__ float sart_value(float x, float bp, float v, float lambda, int noneg) {
    const float t = __fmul_rn(__fdiv_rn(lambda, v), bp);
    const float r = __fadd_rn(x, t);
    return (noneg && r < 0.f) ? 0.f : r;
}

template <typename T, bool SR> struct Rounder;

template <bool SR> struct Rounder<float, SR> {
    static __device__ __forceinline__ float apply(float v, uint32_t) { return v; }
};

template <> struct Rounder<__nv_bfloat16, false> {
    static __device__ __forceinline__ __nv_bfloat16 apply(float v, uint32_t) { return __float2bfloat16_rn(v); }
};

template <> struct Rounder<__nv_bfloat16, true> {
    static __device__ __forceinline__ __nv_bfloat16 apply(float v, uint32_t r16) {
        const uint32_t b = __float_as_uint(v);
        if ((b & 0x7F800000u) == 0x7F800000u) return __float2bfloat16_rn(v);   // Inf, NaN
        const uint32_t r = (b + r16) >> 16;
        // a finite value rounded up past the largest finite BF16 stays at it (as the FP16 path)
        if ((r & 0x7F80u) == 0x7F80u) return __ushort_as_bfloat16((unsigned short)(((b >> 16) & 0x8000u) | 0x7F7Fu));
        return __ushort_as_bfloat16((unsigned short)r);
    }
};

template <> struct Rounder<__half, false> {
    static __device__ __forceinline__ __half apply(float v, uint32_t) { return __float2half_rn(v); }
};

template <> struct Rounder<__half, true> {
    static __device__ __forceinline__ __half apply(float v, uint32_t r16) {
        const __half lo = __float2half_rd(v), hi = __float2half_ru(v);
        const float lf = __half2float(lo), hf = __half2float(hi);
        if (!(hf > lf)) return lo;          // exact, or NaN
        if (isinf(lf)) return hi;           // below -65504: stay finite, as above +65504
        const float p = __fdiv_rn(__fsub_rn(v, lf), __fsub_rn(hf, lf));
        const float u = ((float)r16 + 0.5f) * (1.0f / 65536.0f);
        return u < p ? hi : lo;
    }
};

__device__ __forceinline__ void load8(const float* p, float (&o)[8]) {
    const float4 a = __ldg(reinterpret_cast<const float4*>(p));
    const float4 b = __ldg(reinterpret_cast<const float4*>(p) + 1);
    o[0] = a.x; o[1] = a.y; o[2] = a.z; o[3] = a.w;
    o[4] = b.x; o[5] = b.y; o[6] = b.z; o[7] = b.w;
}

template <typename T> __device__ __forceinline__ void load8x(const T* p, float (&o)[8]) {
    const uint4 u = *reinterpret_cast<const uint4*>(p);
    const T* h = reinterpret_cast<const T*>(&u);
#pragma unroll
    for (int e = 0; e < 8; ++e) o[e] = to_f32<T>(h[e]);
}

template <> __device__ __forceinline__ void load8x<float>(const float* p, float (&o)[8]) {
    const float4 a = reinterpret_cast<const float4*>(p)[0];
    const float4 b = reinterpret_cast<const float4*>(p)[1];
    o[0] = a.x; o[1] = a.y; o[2] = a.z; o[3] = a.w;
    o[4] = b.x; o[5] = b.y; o[6] = b.z; o[7] = b.w;
}

template <typename T> __device__ __forceinline__ void store8x(T* p, const T (&v)[8]) {
    uint4 u;
    T* h = reinterpret_cast<T*>(&u);
#pragma unroll
    for (int e = 0; e < 8; ++e) h[e] = v[e];
    *reinterpret_cast<uint4*>(p) = u;
}

template <> __device__ __forceinline__ void store8x<float>(float* p, const float (&v)[8]) {
    reinterpret_cast<float4*>(p)[0] = make_float4(v[0], v[1], v[2], v[3]);
    reinterpret_cast<float4*>(p)[1] = make_float4(v[4], v[5], v[6], v[7]);
}

// VEC: nyx % 8 == 0 and every pointer 16-byte aligned, so each group is two or three 16-byte
// loads and one or two 16-byte stores; otherwise element by element with the plane bound.
template <typename T, bool SR, bool VEC>
__global__ void __launch_bounds__(256) sart_update_kernel(T* __restrict__ x, const SartArgs a) {
    const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= a.ngroups) return;
    const long long j0 = g * 8;
    float vv[8], bb[8], xx[8];
    if (VEC) {
        load8(a.v + j0, vv);
    } else {
#pragma unroll
        for (int e = 0; e < 8; ++e) vv[e] = j0 + e < a.nyx ? __ldg(a.v + j0 + e) : 1.f;
    }
    for (long long z = blockIdx.y; z < a.nz; z += gridDim.y) {
        const long long base = z * a.nyx + j0;
        uint32_t rw[4] = {0u, 0u, 0u, 0u};
        if (SR) {
            const U4 r = philox4x32_10(U4{(uint32_t)g, (uint32_t)z, a.s0, a.s1}, a.k0, a.k1);
            rw[0] = r.x; rw[1] = r.y; rw[2] = r.z; rw[3] = r.w;
        }
        T out[8];
        if (VEC) {
            load8(a.bp + base, bb);
            load8x<T>(x + base, xx);
#pragma unroll
            for (int e = 0; e < 8; ++e) {
                const uint32_t r16 = (e & 1) ? (rw[e >> 1] >> 16) : (rw[e >> 1] & 0xFFFFu);
                out[e] = Rounder<T, SR>::apply(sart_value(xx[e], bb[e], vv[e], a.lambda, a.noneg), r16);
            }
            store8x<T>(x + base, out);
        } else {
#pragma unroll
            for (int e = 0; e < 8; ++e) {
                if (j0 + e >= a.nyx) break;
                const uint32_t r16 = (e & 1) ? (rw[e >> 1] >> 16) : (rw[e >> 1] & 0xFFFFu);
                const float xv = to_f32<T>(x[base + e]);
                x[base + e] = Rounder<T, SR>::apply(sart_value(xv, __ldg(a.bp + base + e), vv[e], a.lambda, a.noneg),
                                                    r16);
            }
        }
    }
}

template <typename T, bool SR>
void launch_sart(T* x, const SartArgs& a, bool vec, cudaStream_t st) {
    const long long gx = (a.ngroups + 255) / 256;
    const long long gy = a.nz < 65535 ? a.nz : 65535;
    const dim3 grid((unsigned)gx, (unsigned)gy);
    if (vec)
        sart_update_kernel<T, SR, true><<<grid, 256, 0, st>>>(x, a);
    else
        sart_update_kernel<T, SR, false><<<grid, 256, 0, st>>>(x, a);
}

}  // namespace
}  // namespace tigre

using namespace tigre;

extern "C" {

int tigre_sart_update(void* d_x, int dtype, const float* d_bp, const float* d_v, float lambda, int noneg,
                      long long nz, long long nyx, int rounding, unsigned long long seed, unsigned long long step,
                      void* stream) {
    TIGRE_NVTX("tigre_sart_update");
    if (!dtype_ok(dtype)) return fail(TIGRE_ERR_BAD_ASSERT, "sart_update: unknown storage dtype");
    if (nz < 0 || nyx < 0) return fail(TIGRE_ERR_BAD_ASSERT, "sart_update: negative size");
    if (rounding != TIGRE_ROUND_NEAREST && rounding != TIGRE_ROUND_STOCHASTIC)
        return fail(TIGRE_ERR_BAD_ASSERT, "sart_update: unknown rounding mode");
    if (nz == 0 || nyx == 0) return TIGRE_SUCCESS;
    if (!d_x || !d_bp || !d_v) return fail(TIGRE_ERR_BAD_ASSERT, "sart_update: null pointer");
    const long long ngroups = (nyx + 7) / 8;
    if (ngroups > 0xFFFFFFFFll || (ngroups + 255) / 256 > 0x7FFFFFFFll || nz > 0xFFFFFFFFll)
        return fail(TIGRE_ERR_BAD_ASSERT, "sart_update: volume too large");
    SartArgs a{d_bp, d_v, nz, nyx, ngroups, lambda, noneg ? 1 : 0, (uint32_t)seed, (uint32_t)(seed >> 32),
               (uint32_t)step, (uint32_t)(step >> 32)};
    const bool vec = (nyx % 8) == 0 && (((uintptr_t)d_x | (uintptr_t)d_bp | (uintptr_t)d_v) & 15u) == 0;
    const bool sr = rounding == TIGRE_ROUND_STOCHASTIC;
    cudaStream_t st = (cudaStream_t)stream;
    switch (dtype) {
        case TIGRE_F32: launch_sart<float, false>((float*)d_x, a, vec, st); break;
        case TIGRE_BF16:
            if (sr) launch_sart<__nv_bfloat16, true>((__nv_bfloat16*)d_x, a, vec, st);
            else launch_sart<__nv_bfloat16, false>((__nv_bfloat16*)d_x, a, vec, st);
            break;
        default:
            if (sr) launch_sart<__half, true>((__half*)d_x, a, vec, st);
            else launch_sart<__half, false>((__half*)d_x, a, vec, st);
            break;
    }
    TIGRE_LAUNCHED();
    return TIGRE_SUCCESS;
}

}  // extern "C"
