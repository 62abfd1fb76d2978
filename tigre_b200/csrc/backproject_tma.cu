// Voxel-driven backprojection with TMA-staged projection patches (sm_100a).
//
// Same arithmetic as backproject.cu (FDK weight of voxel_backprojection.cu:242-249,
// matched weight of voxel_backprojection2.cu:256-280, bilinear sampling with border 0),
// organised for the B200 memory system:
//
//  * a block owns 16 x 16 voxel columns x 64 slices (one thread per column,
//    64 accumulators in registers; a warp covers 8 x 4 columns) and loops over
//    every view of the call, so the volume is written once per call;
//  * for each view, the bilinear footprint of the block's voxels lies inside
//    the bounding box of its 8 projected corners; one elected lane issues a
//    cp.async.bulk.tensor load of that box of the projection into shared
//    memory (TMA zero-fills what lies outside the detector, which is exactly
//    the texture border rule), double-buffered on two mbarriers so the next
//    view's patch streams in while the current one is consumed;
//  * all per-view constants are precomputed on the host (FrameBPK), so a
//    (column, view) costs a few FP64 FMAs and one division, and a voxel
//    update a handful of packed FP32x2 instructions and four shared-memory
//    loads; the matched weight along a column is a cubic fitted at four
//    Chebyshev nodes per (column, view);
//  * every mbarrier wait is bounded, and a thread whose wait expired waits no
//    more; warp 0's lane 0 issues a copy into a buffer only while its own
//    waits have all succeeded (so only into a buffer whose previous copy has
//    landed); the warps of a thread that saw an expiry write nothing and set
//    TIGRE_STATUS_WAIT_EXPIRED in the plan's status word, and thread 0 waits,
//    bounded, for the copies it issued that may still be in flight -- the
//    block ends instead of hanging.  The steady state carries no extra block
//    barrier or shared flag for this (measured: either costs 2-3 %).
// A (block, view) whose footprint does not fit the box (possible for strongly
// magnified geometries) falls back to bounds-checked global loads.

#include <type_traits>
#include <cuda.h>
#include <cudaTypedefs.h>

#include <cmath>
#include <mutex>

#include "tigre_internal.h"

namespace tigre {
namespace {

constexpr int TXY = kBpTile;   // columns per block edge
constexpr int VZ = kBpSlices;  // slices per thread
constexpr unsigned kWaitLimit = 1u << 16;   // ~ a few ms with the back-off below

struct BPKArgs {
    const FrameBPK* frames;
    const void* proj;     // projection buffer the tensor map describes (fallback reads)
    void* vol;
    int* status;
    int a0, na;
    int nX, nY, nZ, nU, nV;
    int pitch;            // row pitch of proj in elements
    int BU, BV;           // patch box
    float dVZ;
    float scale;
    int accumulate;       // add into the existing volume instead of overwriting it
    int skip_view;        // failure-detection test: no copy is issued for this local view (-1: none)
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t phase) {
    for (unsigned i = 0; i < kWaitLimit; ++i) {
        uint32_t ok;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(ok)
            : "r"(bar), "r"(phase)
            : "memory");
        if (ok) return true;
        __nanosleep(32);
    }
    return false;
}

template <typename TP> __device__ __forceinline__ float lds(uint32_t a);
template <> __device__ __forceinline__ float lds<float>(uint32_t a) {
    float v;
    asm("ld.shared.f32 %0, [%1];" : "=f"(v) : "r"(a));
    return v;
}
template <> __device__ __forceinline__ float lds<__nv_bfloat16>(uint32_t a) {
    unsigned short v;
    asm("ld.shared.u16 %0, [%1];" : "=h"(v) : "r"(a));
    return __uint_as_float(((unsigned)v) << 16);
}

__device__ __forceinline__ float2 f2(float a, float b) { return make_float2(a, b); }
__device__ __forceinline__ float2 f2(float a) { return make_float2(a, a); }
__device__ __forceinline__ float2 neg2(float2 a) { return make_float2(-a.x, -a.y); }
// a + t (b - a), two lanes at once
__device__ __forceinline__ float2 lerp2(float2 a, float2 b, float2 t) {
    return __ffma2_rn(t, __ffma2_rn(a, f2(-1.f), b), a);
}

// texel-space (u - 0.5, v - 0.5) projection of voxel (x, y, z) for view frame F
__device__ __forceinline__ void project_texel(const FrameBPK& F, float x, float y, float z, float& ub, float& vb) {
    const double vx = fma((double)z, F.dz[0], fma((double)y, F.dy[0], fma((double)x, F.dx[0], F.b[0])));
    const double vy = fma((double)z, F.dz[1], fma((double)y, F.dy[1], fma((double)x, F.dx[1], F.b[1])));
    const double vz = fma((double)z, F.dz[2], fma((double)y, F.dy[2], fma((double)x, F.dx[2], F.b[2])));
    const float t = F.tnum / (float)vx;
    ub = fmaf((float)vy, t, F.cu) - 0.5f;
    vb = fmaf((float)vz, t, F.cv) - 0.5f;
}

// Warp 0: bounding box of the block's 8 corner voxels for local view la; lane 0 writes
// info[] and issues the TMA load (or a plain arrive when the box does not fit), unless
// `stopped` (lane 0's own wait for an earlier view expired: the buffer may still be awaiting
// that copy, so its barrier must not be re-armed).
template <typename TP>
__device__ __forceinline__ void plan_patch(const BPKArgs& p, const CUtensorMap* tmap, int la, int x0, int y0, int z0,
                                           TP* dst, uint32_t bar, int* info, bool stopped) {
    const int lane = threadIdx.x & 31;
    const FrameBPK& F = p.frames[p.a0 + la];
    float ub = 0.f, vb = 0.f;
    if (lane < 8) {
        const int x = min(x0 + ((lane & 1) ? TXY - 1 : 0), p.nX - 1);
        const int y = min(y0 + ((lane & 2) ? TXY - 1 : 0), p.nY - 1);
        const int z = min(z0 + ((lane & 4) ? VZ - 1 : 0), p.nZ - 1);
        project_texel(F, (float)x, (float)y, (float)z, ub, vb);
    }
    float umin = lane < 8 ? ub : 3e38f, umax = lane < 8 ? ub : -3e38f;
    float vmin = lane < 8 ? vb : 3e38f, vmax = lane < 8 ? vb : -3e38f;
#pragma unroll
    for (int o = 4; o > 0; o >>= 1) {
        umin = fminf(umin, __shfl_xor_sync(0xffffffffu, umin, o));
        umax = fmaxf(umax, __shfl_xor_sync(0xffffffffu, umax, o));
        vmin = fminf(vmin, __shfl_xor_sync(0xffffffffu, vmin, o));
        vmax = fmaxf(vmax, __shfl_xor_sync(0xffffffffu, vmax, o));
    }
    if (lane == 0) {
        if (stopped) return;
        constexpr int ALIGN = 16 / (int)sizeof(TP);   // TMA: x * sizeof(T) multiple of 16 bytes
        bool fits = isfinite(umin) && isfinite(umax) && isfinite(vmin) && isfinite(vmax) &&
                    fabsf(umin) < 1e7f && fabsf(vmin) < 1e7f;
        int u0 = 0, v0 = 0;
        if (fits) {
            u0 = (int)floorf(umin) - 1;
            u0 = (u0 >= 0) ? (u0 / ALIGN) * ALIGN : -(((-u0) + ALIGN - 1) / ALIGN) * ALIGN;
            v0 = (int)floorf(vmin) - 1;
            fits = ((int)ceilf(umax) + 2 - u0 <= p.BU - 1) && ((int)ceilf(vmax) + 2 - v0 <= p.BV - 1);
        }
        info[0] = u0;
        info[1] = v0;
        info[2] = fits ? 1 : 0;
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        if (la == p.skip_view) {
            // failure-detection test: neither a copy nor an arrival, so the wait for this view
            // runs out with nothing in flight
        } else if (fits) {
            const uint32_t bytes = (uint32_t)(p.BU * p.BV * sizeof(TP));
            asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
            asm volatile(
                "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
                "[%5];" ::"r"(smem_u32(dst)),
                "l"((unsigned long long)tmap), "r"(u0), "r"(v0), "r"(la), "r"(bar)
                : "memory");
        } else {
            asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
        }
    }
}

template <typename TP>
__device__ __forceinline__ float patch_sample(const TP* patch, int BU, int iu, float fu, float pv, float pvmax) {
    pv = fminf(fmaxf(pv, 0.f), pvmax);
    const int iv = (int)pv;
    const float fv = pv - (float)iv;
    const TP* r0 = patch + iv * BU + iu;
    const float p00 = to_f32<TP>(r0[0]), p01 = to_f32<TP>(r0[1]);
    const float p10 = to_f32<TP>(r0[BU]), p11 = to_f32<TP>(r0[BU + 1]);
    const float a0 = fmaf(fu, p01 - p00, p00), a1 = fmaf(fu, p11 - p10, p10);
    return fmaf(fv, a1 - a0, a0);
}

template <typename TP>
__device__ __forceinline__ float global_sample(const BPKArgs& p, const TP* P, float ub, float vb) {
    const float fx = floorf(ub), fy = floorf(vb);
    const float au = ub - fx, av = vb - fy;
    const int iu = (int)fmaxf(fminf(fx, 1e8f), -1e8f), iv = (int)fmaxf(fminf(fy, 1e8f), -1e8f);
    auto at = [&](int u, int v) -> float {
        return (u >= 0 && u < p.nU && v >= 0 && v < p.nV) ? to_f32<TP>(P[(long)v * p.pitch + u]) : 0.f;
    };
    const float a0 = fmaf(au, at(iu + 1, iv) - at(iu, iv), at(iu, iv));
    const float a1 = fmaf(au, at(iu + 1, iv + 1) - at(iu, iv + 1), at(iu, iv + 1));
    return fmaf(av, a1 - a0, a0);
}

template <typename TP, typename TV, bool MATCHED, bool AXIAL>
__global__ void __launch_bounds__(TXY* TXY, 2) bp_tma_kernel(const __grid_constant__ CUtensorMap tmap, BPKArgs p) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    __shared__ __align__(8) unsigned long long bars[2];
    __shared__ int info[2][4];
    // TMA destinations: 128-byte aligned, each buffer rounded up to 128 bytes
    const uint32_t base_off = (128u - (smem_u32(smem_raw) & 127u)) & 127u;
    const size_t buf_bytes = ((size_t)p.BU * p.BV * sizeof(TP) + 127) / 128 * 128;
    TP* buf0 = reinterpret_cast<TP*>(smem_raw + base_off);
    TP* buf1 = reinterpret_cast<TP*>(smem_raw + base_off + buf_bytes);
    const uint32_t buf0_u32 = smem_u32(buf0), buf1_u32 = smem_u32(buf1);
    const uint32_t rowb = (uint32_t)(p.BU * sizeof(TP));
    const int tid = threadIdx.x;
    // each warp covers an 8 x 4 patch of columns: at every view angle its 32 samples of one
    // slice fall on a compact set of detector texels (few shared-memory wavefronts)
    const int wid = tid >> 5, ln = tid & 31;
    const int tx = (wid & 1) * 8 + (ln & 7), ty = (wid >> 1) * 4 + (ln >> 3);
    const int x0 = blockIdx.x * TXY, y0 = blockIdx.y * TXY, z0 = blockIdx.z * VZ;
    const int x = x0 + tx, y = y0 + ty;
    const bool active = x < p.nX && y < p.nY;
    const uint32_t bar0 = smem_u32(&bars[0]), bar1 = smem_u32(&bars[1]);
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar0) : "memory");
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar1) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    if (tid < 32) {
        plan_patch<TP>(p, &tmap, 0, x0, y0, z0, buf0, bar0, info[0], false);
        if (p.na > 1) plan_patch<TP>(p, &tmap, 1, x0, y0, z0, buf1, bar1, info[1], false);
    }
    float acc[VZ];
#pragma unroll
    for (int k = 0; k < VZ; ++k) acc[k] = 0.f;
    const TP* Pg = (const TP*)p.proj;
    const float pumax = (float)(p.BU - 2), pvmax = (float)(p.BV - 2);
    int failed_at = -1;   // first view whose wait expired in this thread
    for (int la = 0; la < p.na; ++la) {
        const int s = la & 1;
        const uint32_t bar = s ? bar1 : bar0;
        // after one expired wait this thread waits no more (its sums are not written)
        if (failed_at < 0 && !mbar_wait(bar, (uint32_t)((la >> 1) & 1))) failed_at = la;
        const TP* patch = s ? buf1 : buf0;
        const uint32_t patch_u32 = s ? buf1_u32 : buf0_u32;
        const int u0 = info[s][0], v0 = info[s][1], fits = info[s][2];
        if (active) {
            const FrameBPK& F = p.frames[p.a0 + la];
            const double bxd = fma((double)z0, F.dz[0], fma((double)y, F.dy[0], fma((double)x, F.dx[0], F.b[0])));
            const double byd = fma((double)z0, F.dz[1], fma((double)y, F.dy[1], fma((double)x, F.dx[1], F.b[1])));
            const double bzd = fma((double)z0, F.dz[2], fma((double)y, F.dy[2], fma((double)x, F.dx[2], F.b[2])));
            const float vx = (float)bxd, vy = (float)byd, vz = (float)bzd;
            float wcol = 1.f, cu2 = 0.f, cxy = 0.f;
            if (!MATCHED) {
                const float den = fmaf((float)y, F.wy, fmaf((float)x, F.wx, F.w0));
                const float r = __fdividef(F.dso, den);
                wcol = r * r;
            } else {
                const float rvx = fmaf((float)x, F.dvx, F.rv0x), rvy = fmaf((float)y, F.dvy, F.rv0y);
                cxy = (F.rsx - rvx) * (F.rsx - rvx) + (F.rsy - rvy) * (F.rsy - rvy);
            }
            if (AXIAL) {
                const float t = F.tnum / vx;
                const float u = fmaf(vy, t, F.cu);            // texture coordinate
                const float vt0 = fmaf(vz, t, F.cv);
                const float vstep = (float)F.dz[2] * t;
                if (MATCHED) {
                    const float day = fmaf(u, F.ddu, F.du0);
                    const float dx = fmaf(day, F.sina, F.daxc), dy = fmaf(day, F.cosa, -F.daxs);
                    cu2 = (F.rsx - dx) * (F.rsx - dx) + (F.rsy - dy) * (F.rsy - dy);
                }
                if (fits) {
                    const float pu = fminf(fmaxf(u - 0.5f - (float)u0, 0.f), pumax);
                    const int iu = (int)pu;
                    const float2 fu2 = f2(pu - (float)iu);
                    const float pv0 = vt0 - 0.5f - (float)v0;
                    constexpr uint32_t ES = (uint32_t)sizeof(TP);
                    const uint32_t colb = patch_u32 + (uint32_t)iu * ES;
                    const float2 vstep2 = f2(vstep);
                    const float2 pv02 = f2(pv0);
                    const float2 w2 = f2(wcol);
                    // rows stay inside the patch for the whole column -> no per-voxel clamps
                    const float pvlast = fmaf((float)(VZ - 1), vstep, pv0);
                    const bool inside = fminf(pv0, pvlast) >= 0.f && fmaxf(pv0, pvlast) <= pvmax;
                    // Matched weight w(k) = L^3 / (DSD lsq) along the column: L^2 and lsq are
                    // quadratics in the slice index k with complex roots hundreds of slices away,
                    // so w is interpolated by the cubic through its exact values at the four
                    // Chebyshev nodes of [0, VZ-1] (relative error ~1e-7 at a 6:10 source/detector
                    // distance ratio, far below that at the usual ones).  In s = k - (VZ-1)/2,
                    // with nodes +-na, +-nb, the cubic is e0 + o1 s + e2 s^2 + o3 s^3.  The node
                    // values use the hardware reciprocal square root and the approximate
                    // division (each within 2 ulp), since they run once per column and view.
                    float2 c0 = f2(0.f), c1 = f2(0.f), c2 = f2(0.f), c3 = f2(0.f);
                    if (MATCHED) {
                        constexpr float hw = 0.5f * (float)(VZ - 1);
                        constexpr float na = hw * 0.92387953251f;   // cos(pi/8) = sqrt(2 + sqrt 2) / 2
                        constexpr float nb = hw * 0.38268343236f;   // cos(3pi/8) = sqrt(2 - sqrt 2) / 2
                        constexpr float inv = 1.f / (na * na - nb * nb);
                        const float rz0 = fmaf((float)z0, p.dVZ, F.rv0z);
                        auto wexact = [&](float kf) {
                            const float vt = fmaf(kf, vstep, vt0), dz = fmaf(vt, F.ddv, F.dzc), L2 = fmaf(dz, dz, cu2);
                            const float rvz = fmaf(kf, p.dVZ, rz0), lsq = fmaf(rvz, rvz, cxy);
                            return __fdividef(L2 * L2 * rsqrtf(L2), F.dsd * lsq);
                        };
                        const float wpa = wexact(hw + na), wma = wexact(hw - na);
                        const float wpb = wexact(hw + nb), wmb = wexact(hw - nb);
                        const float Ea = 0.5f * (wpa + wma), Eb = 0.5f * (wpb + wmb);
                        const float Oa = (wpa - wma) * (0.5f / na), Ob = (wpb - wmb) * (0.5f / nb);
                        const float e2 = (Ea - Eb) * inv, o3 = (Oa - Ob) * inv;
                        c0 = f2(fmaf(-e2, na * na, Ea));
                        c1 = f2(fmaf(-o3, na * na, Oa));
                        c2 = f2(e2);
                        c3 = f2(o3);
                    }
                    // the float bits of the floor below index the patch directly:
                    // row address = bits * rowb + colb - 0x4B400000 * rowb (32-bit wrap)
                    const uint32_t colb_m = colb - 0x4B400000u * rowb;
                    auto pairs = [&](auto clamp_tag) {
                        constexpr bool CLAMP = decltype(clamp_tag)::value;
#pragma unroll
                        for (int k = 0; k < VZ; k += 2) {
                            const float2 kk = f2((float)k, (float)(k + 1));
                            float2 pv = __ffma2_rn(kk, vstep2, pv02);
                            if (CLAMP) {
                                pv.x = fminf(fmaxf(pv.x, 0.f), pvmax);
                                pv.y = fminf(fmaxf(pv.y, 0.f), pvmax);
                            }
                            // floor / fraction with packed arithmetic: pv >= 0 here, and at 1.5*2^23
                            // the float spacing is 1, so a round-toward-zero add of 1.5*2^23 leaves
                            // floor(pv) in the low mantissa bits; subtracting it back is exact
                            const float2 t = __fadd2_rz(pv, f2(12582912.0f));
                            const float2 fv = __ffma2_rn(__fadd2_rn(t, f2(-12582912.0f)), f2(-1.f), pv);
                            const uint32_t aa = (uint32_t)__float_as_int(t.x) * rowb + colb_m;
                            const uint32_t ab = (uint32_t)__float_as_int(t.y) * rowb + colb_m;
                            const float2 r0 = f2(lds<TP>(aa), lds<TP>(ab)), r0r = f2(lds<TP>(aa + ES), lds<TP>(ab + ES));
                            const float2 r1 = f2(lds<TP>(aa + rowb), lds<TP>(ab + rowb));
                            const float2 r1r = f2(lds<TP>(aa + rowb + ES), lds<TP>(ab + rowb + ES));
                            const float2 smp = lerp2(lerp2(r0, r0r, fu2), lerp2(r1, r1r, fu2), fv);
                            float2 w = w2;
                            if (MATCHED) {
                                const float2 s2 = f2((float)k - 0.5f * (float)(VZ - 1), (float)(k + 1) - 0.5f * (float)(VZ - 1));
                                w = __ffma2_rn(__ffma2_rn(__ffma2_rn(c3, s2, c2), s2, c1), s2, c0);
                            }
                            const float2 acc2 = __ffma2_rn(smp, w, f2(acc[k], acc[k + 1]));
                            acc[k] = acc2.x;
                            acc[k + 1] = acc2.y;
                        }
                    };
                    if (inside) pairs(std::false_type{});
                    else pairs(std::true_type{});
                } else {
                    // unrolled: a runtime index into acc[] would move it to local memory
#pragma unroll
                    for (int k = 0; k < VZ; ++k) {
                        const float vtex = fmaf((float)k, vstep, vt0);
                        const float smp = global_sample<TP>(p, Pg + (long)la * p.pitch * p.nV, u - 0.5f, vtex - 0.5f);
                        float w = wcol;
                        if (MATCHED) {
                            const float dz = fmaf(vtex, F.ddv, F.dzc);
                            const float L2 = fmaf(dz, dz, cu2);
                            const float rvz = fmaf((float)(z0 + k), p.dVZ, F.rv0z);
                            const float lsq = fmaf(rvz, rvz, cxy);
                            w = L2 * (L2 * rsqrtf(L2)) * __frcp_rn(F.dsd * lsq);
                        }
                        acc[k] = fmaf(smp, w, acc[k]);
                    }
                }
            } else {
                const float dzx = (float)F.dz[0], dzy = (float)F.dz[1], dzz = (float)F.dz[2];
#pragma unroll
                for (int k = 0; k < VZ; ++k) {
                    const float kf = (float)k;
                    const float ex = fmaf(kf, dzx, vx), ey = fmaf(kf, dzy, vy), ez = fmaf(kf, dzz, vz);
                    const float t = F.tnum / ex;
                    const float u = fmaf(ey, t, F.cu), vtex = fmaf(ez, t, F.cv);
                    float smp;
                    if (fits) {
                        const float pu = fminf(fmaxf(u - 0.5f - (float)u0, 0.f), pumax);
                        const int iu = (int)pu;
                        smp = patch_sample<TP>(patch, p.BU, iu, pu - (float)iu, vtex - 0.5f - (float)v0, pvmax);
                    } else {
                        smp = global_sample<TP>(p, Pg + (long)la * p.pitch * p.nV, u - 0.5f, vtex - 0.5f);
                    }
                    float w = wcol;
                    if (MATCHED) {
                        const float day = fmaf(u, F.ddu, F.du0);
                        const float dx = fmaf(day, F.sina, F.daxc), dy = fmaf(day, F.cosa, -F.daxs);
                        const float dz = fmaf(vtex, F.ddv, F.dzc);
                        const float L2 = (F.rsx - dx) * (F.rsx - dx) + (F.rsy - dy) * (F.rsy - dy) + dz * dz;
                        const float rvz = fmaf((float)(z0 + k), p.dVZ, F.rv0z);
                        const float lsq = fmaf(rvz, rvz, cxy);
                        w = L2 * (L2 * rsqrtf(L2)) * __frcp_rn(F.dsd * lsq);
                    }
                    acc[k] = fmaf(smp, w, acc[k]);
                }
            }
        }
        __syncthreads();   // everyone is done with buffer s
        if (tid < 32 && la + 2 < p.na) plan_patch<TP>(p, &tmap, la + 2, x0, y0, z0, s ? buf1 : buf0, bar, info[s], failed_at >= 0);
    }
    if (tid == 0 && failed_at >= 0) {
        // thread 0 issued nothing after its failed view: the copies of that view and the next
        // may still be in flight, so wait for them (bounded) before the block's shared memory
        // is released
        for (int v = failed_at; v < min(failed_at + 2, p.na); ++v)
            if (v != p.skip_view) mbar_wait((v & 1) ? bar1 : bar0, (uint32_t)((v >> 1) & 1));
    }
    if (__any_sync(0xffffffffu, failed_at >= 0)) {
        if ((tid & 31) == 0 && p.status) atomicOr(p.status, TIGRE_STATUS_WAIT_EXPIRED);
        return;
    }
    if (!active) return;
    TV* V = (TV*)p.vol;
#pragma unroll
    for (int k = 0; k < VZ; ++k) {
        const int z = z0 + k;
        if (z < p.nZ) {
            const size_t i = ((size_t)z * p.nY + y) * p.nX + x;
            const float o = p.accumulate ? to_f32<TV>(V[i]) : 0.f;
            V[i] = from_f32<TV>(fmaf(acc[k], p.scale, o));
        }
    }
}

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(f);
    });
    return fn;
}

template <typename TP, typename TV>
int launch_typed(const CUtensorMap& tm, const BPKArgs& a, bool matched, bool axial, cudaStream_t st) {
    dim3 grid((a.nX + TXY - 1) / TXY, (a.nY + TXY - 1) / TXY, (a.nZ + VZ - 1) / VZ);
    const size_t smem = 2 * (((size_t)a.BU * a.BV * sizeof(TP) + 127) / 128 * 128) + 128;
    auto go = [&](auto kern) -> int {
        TIGRE_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        kern<<<grid, TXY * TXY, smem, st>>>(tm, a);
        TIGRE_LAUNCHED();
        return TIGRE_SUCCESS;
    };
    if (matched) return axial ? go(bp_tma_kernel<TP, TV, true, true>) : go(bp_tma_kernel<TP, TV, true, false>);
    return axial ? go(bp_tma_kernel<TP, TV, false, true>) : go(bp_tma_kernel<TP, TV, false, false>);
}

}  // namespace

bool bp_tma_supported(const TigrePlan* P, int pdt) {
    if (pdt == TIGRE_F16) return false;
    return P->bp_box_u > 0 && encode_fn() != nullptr;
}

int launch_backproject_tma(TigrePlan* P, const void* proj, int pitch, int pdt, void* vol, int vdt, int matched,
                           int a0, int a1, int accumulate, cudaStream_t st) {
    auto enc = encode_fn();
    if (!enc) return fail(TIGRE_ERR_CUDA, "cuTensorMapEncodeTiled unavailable");
    const int na = a1 - a0;
    const size_t es = dtype_size(pdt);
    CUtensorMap tm;
    cuuint64_t dims[3] = {(cuuint64_t)pitch, (cuuint64_t)P->d.nV, (cuuint64_t)na};
    cuuint64_t strides[2] = {(cuuint64_t)pitch * es, (cuuint64_t)pitch * P->d.nV * es};
    const int BU = pdt == TIGRE_F32 ? P->bp_box_u : P->bp_box_u16;
    cuuint32_t box[3] = {(cuuint32_t)BU, (cuuint32_t)P->bp_box_v, 1};
    cuuint32_t estr[3] = {1, 1, 1};
    CUresult r = enc(&tm, pdt == TIGRE_F32 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 3,
                     const_cast<void*>(proj), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                     CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return fail(TIGRE_ERR_CUDA, "cuTensorMapEncodeTiled failed");
    BPKArgs a{};
    a.frames = P->d_bpk;
    a.proj = proj;
    a.vol = vol;
    a.status = P->d_status;
    a.a0 = a0;
    a.na = na;
    a.nX = P->d.nX; a.nY = P->d.nY; a.nZ = P->d.nZ; a.nU = P->d.nU; a.nV = P->d.nV;
    a.pitch = pitch;
    a.BU = BU;
    a.BV = P->bp_box_v;
    a.dVZ = (float)P->d.dVZ;
    a.scale = matched ? (float)(P->d.dVX * P->d.dVY * P->d.dVZ / (P->d.dDU * P->d.dDV)) : 1.f;
    a.accumulate = accumulate;
    const long long skip = option(TIGRE_OPT_BP_SKIP_COPY);
    a.skip_view = (skip >= 0 && skip < na) ? (int)skip : -1;
    const bool ax = P->axial;
    if (pdt == TIGRE_F32 && vdt == TIGRE_F32) return launch_typed<float, float>(tm, a, matched, ax, st);
    if (pdt == TIGRE_BF16 && vdt == TIGRE_BF16) return launch_typed<__nv_bfloat16, __nv_bfloat16>(tm, a, matched, ax, st);
    if (pdt == TIGRE_BF16 && vdt == TIGRE_F32) return launch_typed<__nv_bfloat16, float>(tm, a, matched, ax, st);
    if (pdt == TIGRE_F32 && vdt == TIGRE_BF16) return launch_typed<float, __nv_bfloat16>(tm, a, matched, ax, st);
    return fail(TIGRE_ERR_BAD_ASSERT, "unsupported dtype pair for the staged backprojector");
}

}  // namespace tigre
