// Voxel-driven cone-beam backprojection (FDK-weighted and matched), sm_100a.
//
// For every voxel and view: project the voxel centre on the detector,
// bilinearly sample the projection (border 0, texel centres at +0.5), weight,
// accumulate.  Formulas of Common/CUDA/voxel_backprojection.cu:196-258 (FDK
// weight ((DSO + y sin a - x cos a)/DSO)^-2) and
// Common/CUDA/voxel_backprojection2.cu:186-281 (matched weight
// L^3/(DSD |S-x|^2), final scale dVx dVy dVz / (dU dV), :585), with the
// reference's view angles negated in the frames (voxel_backprojection.cu:510-515).
//
// Design (B200):
//  * one thread per (x, y) column of VZ voxels in z; a block is 32 x 8 columns,
//    a warp is 32 neighbouring x, whose projections land on neighbouring
//    detector columns of the same rows (coalesced gathers);
//  * ALL views of the call are accumulated in registers inside one launch, so
//    the volume is written exactly once (the reference writes it back after
//    every 32 views); view frames are staged in shared memory 32 at a time;
//  * the column's projected position is evaluated in FP64 once per
//    (column, view), the per-voxel steps in FP32;
//  * AXIAL specialisation: when no frame tilts the z axis (no theta/psi/detector
//    roll), u and the FDK weight are constant along a column and v steps
//    linearly, so a voxel costs one bilinear gather and a few FMAs;
//  * the projections are read from a zero-bordered copy (1 pixel before, 2 after)
//    so the 4-tap gather needs no bounds tests; interpolation weights are exact
//    FP32 (the reference's texture unit quantises them to 8 fractional bits).

#include <cmath>

#include "tigre_internal.h"

namespace tigre {
namespace {

struct BPArgs {
    const void* proj;   // padded (na, nV+3, nU+3)
    void* vol;          // (nZ, nY, nX)
    const FrameBP* frames;
    int a0, na;
    int nX, nY, nZ, nU, nV;
    float sVX, sVY, sVZ, dVX, dVY, dVZ;
    float sDU, sDV, dDU, dDV;
    float scale;
    int accumulate;       // add into the existing volume instead of overwriting it
};

constexpr int BX = 32, BY = 8, CHUNK = 32;

template <typename TP>
__device__ __forceinline__ float bilinear(const TP* __restrict__ P, long pitch, float u, float v, float umax,
                                          float vmax) {
    // texture coordinate u -> padded texel base u - 0.5 + 1
    const float xb = fminf(fmaxf(u + 0.5f, 0.f), umax);
    const float yb = fminf(fmaxf(v + 0.5f, 0.f), vmax);
    const int iu = (int)xb, iv = (int)yb;
    const float fu = xb - (float)iu, fv = yb - (float)iv;
    const TP* b = P + (long)iv * pitch + iu;
    const float p00 = ldg_f<TP>(b), p01 = ldg_f<TP>(b + 1);
    const float p10 = ldg_f<TP>(b + pitch), p11 = ldg_f<TP>(b + pitch + 1);
    const float r0 = fmaf(fu, p01 - p00, p00), r1 = fmaf(fu, p11 - p10, p10);
    return fmaf(fv, r1 - r0, r0);
}

template <typename TP, typename TV, bool MATCHED, bool AXIAL, int VZ>
__global__ void __launch_bounds__(BX* BY) bp_kernel(BPArgs p) {
    __shared__ FrameBP sf[CHUNK];
    const int tid = threadIdx.y * BX + threadIdx.x;
    const int x = blockIdx.x * BX + threadIdx.x;
    const int y = blockIdx.y * BY + threadIdx.y;
    const int z0 = blockIdx.z * VZ;
    const bool active = x < p.nX && y < p.nY;
    float acc[VZ];
#pragma unroll
    for (int j = 0; j < VZ; ++j) acc[j] = 0.f;
    const long pitch = bp_pitch(p.nU), plane = pitch * bp_rows(p.nV);
    const float umax = (float)(p.nU + 1), vmax = (float)(p.nV + 1);
    const TP* P = (const TP*)p.proj;
    const float hu = 0.5f * (float)p.nU, hv = 0.5f * (float)p.nV;
    // voxel centre in mm, without the per-view offsets
    const float rx0 = -(p.sVX - p.dVX) * 0.5f + (float)x * p.dVX;
    const float ry0 = -(p.sVY - p.dVY) * 0.5f + (float)y * p.dVY;
    const float rz0 = -(p.sVZ - p.dVZ) * 0.5f + (float)z0 * p.dVZ;

    for (int c0 = 0; c0 < p.na; c0 += CHUNK) {
        const int cn = min(CHUNK, p.na - c0);
        __syncthreads();
        {
            const int words = cn * (int)(sizeof(FrameBP) / 4);
            const int* src = (const int*)(p.frames + p.a0 + c0);
            int* dst = (int*)sf;
            for (int i = tid; i < words; i += BX * BY) dst[i] = src[i];
        }
        __syncthreads();
        if (!active) continue;
        for (int j = 0; j < cn; ++j) {
            const FrameBP& F = sf[j];
            const TP* Pa = P + (long)(c0 + j) * plane;
            const double bx = fma((double)z0, F.dz[0], fma((double)y, F.dy[0], fma((double)x, F.dx[0], F.o[0])));
            const double by = fma((double)z0, F.dz[1], fma((double)y, F.dy[1], fma((double)x, F.dx[1], F.o[1]))) -
                              (double)F.cor / (double)p.dDU;
            const double bz = fma((double)z0, F.dz[2], fma((double)y, F.dy[2], fma((double)x, F.dx[2], F.o[2])));
            const float vx = (float)(bx - F.s[0]), vy = (float)(by - F.s[1]), vz = (float)(bz - F.s[2]);
            const float tnum = (float)((double)F.dso - (double)F.dsd - F.s[0]);
            const float cu = (float)(F.s[1] + (double)hu), cv = (float)(F.s[2] + (double)hv);
            const float dzx = (float)F.dz[0], dzy = (float)F.dz[1], dzz = (float)F.dz[2];
            float wcol = 1.f;
            float rsx = 0.f, rsy = 0.f, rvx = 0.f, rvy = 0.f, dax = 0.f, dzc = 0.f, cxy = 0.f;
            if (!MATCHED) {
                const float realx = rx0 + F.offx, realy = ry0 + F.offy + F.cor;
                const float ww = (F.dso + realy * F.sina - realx * F.cosa) / F.dso;
                wcol = 1.f / (ww * ww);
            } else {
                rsx = F.dso * F.cosa;
                rsy = -F.dso * F.sina;
                rvx = rx0 + F.offx;
                rvy = ry0 + F.offy;
                dax = -(F.dsd - F.dso);
                dzc = (-p.sDV + p.dDV) * 0.5f + F.offv;
                cxy = (rsx - rvx) * (rsx - rvx) + (rsy - rvy) * (rsy - rvy);
            }
            if (AXIAL) {
                const float t = tnum / vx;
                const float u = fmaf(vy, t, cu);
                const float v0 = fmaf(vz, t, cv);
                const float vstep = dzz * t;
                float cu2 = 0.f;
                if (MATCHED) {
                    const float day = (-p.sDU + p.dDU) * 0.5f + u * p.dDU + F.offu;
                    const float dx = dax * F.cosa + day * F.sina;
                    const float dy = -dax * F.sina + day * F.cosa;
                    cu2 = (rsx - dx) * (rsx - dx) + (rsy - dy) * (rsy - dy);
                }
#pragma unroll
                for (int k = 0; k < VZ; ++k) {
                    const float v = fmaf((float)k, vstep, v0);
                    const float smp = bilinear<TP>(Pa, pitch, u, v, umax, vmax);
                    if (!MATCHED) {
                        acc[k] = fmaf(smp, wcol, acc[k]);
                    } else {
                        const float dz = fmaf(v, p.dDV, dzc);
                        const float L2 = fmaf(dz, dz, cu2);
                        const float rvz = rz0 + (float)k * p.dVZ + F.offz;
                        const float lsq = fmaf(rvz, rvz, cxy);
                        const float w = L2 * sqrtf(L2) / (F.dsd * lsq);
                        acc[k] = fmaf(smp, w, acc[k]);
                    }
                }
            } else {
#pragma unroll
                for (int k = 0; k < VZ; ++k) {
                    const float kf = (float)k;
                    const float ex = fmaf(kf, dzx, vx), ey = fmaf(kf, dzy, vy), ez = fmaf(kf, dzz, vz);
                    const float t = tnum / ex;
                    const float u = fmaf(ey, t, cu), v = fmaf(ez, t, cv);
                    const float smp = bilinear<TP>(Pa, pitch, u, v, umax, vmax);
                    if (!MATCHED) {
                        acc[k] = fmaf(smp, wcol, acc[k]);
                    } else {
                        const float day = (-p.sDU + p.dDU) * 0.5f + u * p.dDU + F.offu;
                        const float dx = dax * F.cosa + day * F.sina;
                        const float dy = -dax * F.sina + day * F.cosa;
                        const float dz = fmaf(v, p.dDV, dzc);
                        const float L2 = (rsx - dx) * (rsx - dx) + (rsy - dy) * (rsy - dy) + dz * dz;
                        const float rvz = rz0 + kf * p.dVZ + F.offz;
                        const float lsq = fmaf(rvz, rvz, cxy);
                        const float w = L2 * sqrtf(L2) / (F.dsd * lsq);
                        acc[k] = fmaf(smp, w, acc[k]);
                    }
                }
            }
        }
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

constexpr int kVZ = 8;

template <typename TP, typename TV>
void launch_typed(const BPArgs& a, bool matched, bool axial, cudaStream_t st) {
    dim3 block(BX, BY);
    dim3 grid((a.nX + BX - 1) / BX, (a.nY + BY - 1) / BY, (a.nZ + kVZ - 1) / kVZ);
    if (matched) {
        if (axial) bp_kernel<TP, TV, true, true, kVZ><<<grid, block, 0, st>>>(a);
        else bp_kernel<TP, TV, true, false, kVZ><<<grid, block, 0, st>>>(a);
    } else {
        if (axial) bp_kernel<TP, TV, false, true, kVZ><<<grid, block, 0, st>>>(a);
        else bp_kernel<TP, TV, false, false, kVZ><<<grid, block, 0, st>>>(a);
    }
}

}  // namespace

int launch_backproject(TigrePlan* P, const void* proj_pad, int pdt, void* vol, int vdt, int matched, int a0, int a1,
                       int accumulate, cudaStream_t st) {
    static_assert(sizeof(FrameBP) % 4 == 0, "frame must be word-sized");
    BPArgs a{};
    a.proj = proj_pad; a.vol = vol; a.frames = P->d_bp; a.a0 = a0; a.na = a1 - a0;
    a.nX = P->d.nX; a.nY = P->d.nY; a.nZ = P->d.nZ; a.nU = P->d.nU; a.nV = P->d.nV;
    a.sVX = (float)P->d.sVX; a.sVY = (float)P->d.sVY; a.sVZ = (float)P->d.sVZ;
    a.dVX = (float)P->d.dVX; a.dVY = (float)P->d.dVY; a.dVZ = (float)P->d.dVZ;
    a.sDU = (float)P->d.sDU; a.sDV = (float)P->d.sDV; a.dDU = (float)P->d.dDU; a.dDV = (float)P->d.dDV;
    a.scale = matched ? (float)(P->d.dVX * P->d.dVY * P->d.dVZ / (P->d.dDU * P->d.dDV)) : 1.f;
    a.accumulate = accumulate;
    const bool ax = P->axial;
    if (pdt == TIGRE_F32 && vdt == TIGRE_F32) launch_typed<float, float>(a, matched, ax, st);
    else if (pdt == TIGRE_BF16 && vdt == TIGRE_BF16) launch_typed<__nv_bfloat16, __nv_bfloat16>(a, matched, ax, st);
    else if (pdt == TIGRE_F16 && vdt == TIGRE_F16) launch_typed<__half, __half>(a, matched, ax, st);
    else if (pdt == TIGRE_BF16 && vdt == TIGRE_F32) launch_typed<__nv_bfloat16, float>(a, matched, ax, st);
    else if (pdt == TIGRE_F16 && vdt == TIGRE_F32) launch_typed<__half, float>(a, matched, ax, st);
    else return fail(TIGRE_ERR_BAD_ASSERT, "unsupported dtype pair for backprojection");
    TIGRE_LAUNCHED();
    return TIGRE_SUCCESS;
}

}  // namespace tigre
