// Interpolated (fixed-step trilinear) cone-beam forward projection, sm_100a.
//
// Per detector pixel: n = ceil(|P-S| / accuracy) steps, step vector
// (P-S)/n, samples at S + i*step for i from floor(cropdist/accuracy) to n
// (n optionally capped), trilinear value at each sample with border 0, sum
// times the step length in mm -- kernelPixelDetector<sphericalrotation> of
// Common/CUDA/ray_interpolated_projection.cu:117-206.  With accuracy > 1 the
// reference switches its texture to point filtering (:589-592); so does this
// kernel (NEAREST).
//
// Differences in how, not what:
//  * interpolation weights are exact FP32 (the reference's texture unit uses
//    9-bit weights); sample positions come from an FP64 ray setup;
//  * samples whose trilinear footprint lies outside the volume contribute
//    exactly 0 in the reference; the sample range is clipped to the open box
//    (-1, n) per axis first, so only samples that can be nonzero are taken;
//  * the volume is read from a zero-padded working copy (1 voxel before, 2
//    after, per axis), x- or y-fastest per view like the Siddon kernel, so the
//    8-corner gather needs no bounds tests.

#include <cmath>

#include "tigre_internal.h"

namespace tigre {
namespace {

struct InterpArgs {
    const void* vol_x;   // padded, (nZ+3, nY+3, nX+3)
    const void* vol_y;   // padded, (nZ+3, nX+3, nY+3)
    void* proj;
    const FrameInterp* frames;
    int a0;
    int nX, nY, nZ, nU, nV;
    double dVX, dVY, dVZ, acc;
};

template <typename TV, typename TP, bool NEAREST>
__global__ void __launch_bounds__(256) interp_kernel(InterpArgs p) {
    const int u = blockIdx.x * 32 + threadIdx.x;
    const int v = blockIdx.y * blockDim.y + threadIdx.y;
    const int la = blockIdx.z;
    if (u >= p.nU || v >= p.nV) return;
    const FrameInterp& F = p.frames[p.a0 + la];
    const double pv = (double)(p.nV - 1 - v);
    double d[3], s[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        s[k] = F.s[k];
        d[k] = fma(pv, F.dv[k], fma((double)u, F.du[k], F.o[k])) - s[k];
    }
    const double len = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
    double length = ceil(len / p.acc);
    double vec[3] = {d[0] / length, d[1] / length, d[2] / length};
    if (F.cap < length) length = ceil(F.cap);
    double lo = F.first_sample, hi = length;
    const int n[3] = {p.nX, p.nY, p.nZ};
    bool empty = false;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        if (vec[k] != 0.0) {
            const double ta = (-1.0 - s[k]) / vec[k], tb = ((double)n[k] - s[k]) / vec[k];
            lo = fmax(lo, floor(fmin(ta, tb)));
            hi = fmin(hi, ceil(fmax(ta, tb)));
        } else if (s[k] <= -1.0 || s[k] >= (double)n[k]) {
            empty = true;
        }
    }
    const size_t oidx = ((size_t)la * p.nV + v) * (size_t)p.nU + u;
    if (empty || lo > hi) {
        ((TP*)p.proj)[oidx] = from_f32<TP>(0.f);
        return;
    }
    const int nsamp = (int)(hi - lo) + 1;
    // padded coordinates (+1) of the first sample
    const float q0x = (float)(fma(vec[0], lo, s[0]) + 1.0);
    const float q0y = (float)(fma(vec[1], lo, s[1]) + 1.0);
    const float q0z = (float)(fma(vec[2], lo, s[2]) + 1.0);
    const float vx = (float)vec[0], vy = (float)vec[1], vz = (float)vec[2];
    const float mx = (float)(p.nX + 1), my = (float)(p.nY + 1), mz = (float)(p.nZ + 1);
    const int XP = p.nX + 3, YP = p.nY + 3;
    const int layout = F.layout;
    const TV* vol = (const TV*)(layout ? p.vol_y : p.vol_x);
    const int sx = layout ? YP : 1;
    const int sy = layout ? 1 : XP;
    const int sz = XP * YP;
    float sum = 0.f;
#pragma unroll 2
    for (int k = 0; k < nsamp; ++k) {
        const float kf = (float)k;
        const float qx = fminf(fmaxf(fmaf(kf, vx, q0x), 0.f), mx);
        const float qy = fminf(fmaxf(fmaf(kf, vy, q0y), 0.f), my);
        const float qz = fminf(fmaxf(fmaf(kf, vz, q0z), 0.f), mz);
        if (NEAREST) {
            const int ix = (int)(qx + 0.5f), iy = (int)(qy + 0.5f), iz = (int)(qz + 0.5f);
            sum += ldg_f<TV>(vol + ix * sx + iy * sy + iz * sz);
        } else {
            const int ix = (int)qx, iy = (int)qy, iz = (int)qz;
            const float fx = qx - (float)ix, fy = qy - (float)iy, fz = qz - (float)iz;
            const TV* b = vol + ix * sx + iy * sy + iz * sz;
            const float c000 = ldg_f<TV>(b), c100 = ldg_f<TV>(b + sx);
            const float c010 = ldg_f<TV>(b + sy), c110 = ldg_f<TV>(b + sx + sy);
            const float c001 = ldg_f<TV>(b + sz), c101 = ldg_f<TV>(b + sx + sz);
            const float c011 = ldg_f<TV>(b + sy + sz), c111 = ldg_f<TV>(b + sx + sy + sz);
            const float c00 = fmaf(fx, c100 - c000, c000), c10 = fmaf(fx, c110 - c010, c010);
            const float c01 = fmaf(fx, c101 - c001, c001), c11 = fmaf(fx, c111 - c011, c011);
            const float c0 = fmaf(fy, c10 - c00, c00), c1 = fmaf(fy, c11 - c01, c01);
            sum += fmaf(fz, c1 - c0, c0);
        }
    }
    const double dl = sqrt(vec[0] * p.dVX * vec[0] * p.dVX + vec[1] * p.dVY * vec[1] * p.dVY +
                           vec[2] * p.dVZ * vec[2] * p.dVZ);
    ((TP*)p.proj)[oidx] = from_f32<TP>(sum * (float)dl);
}

template <typename TV, typename TP>
void launch_typed(const InterpArgs& a, bool nearest, dim3 grid, dim3 block, cudaStream_t st) {
    if (nearest) interp_kernel<TV, TP, true><<<grid, block, 0, st>>>(a);
    else interp_kernel<TV, TP, false><<<grid, block, 0, st>>>(a);
}

}  // namespace

int launch_interp(TigrePlan* P, const void* vol_x, const void* vol_y, int vdt, void* proj, int pdt, int a0, int a1,
                  cudaStream_t st) {
    InterpArgs a{};
    a.vol_x = vol_x; a.vol_y = vol_y; a.frames = P->d_interp;
    a.nX = P->d.nX; a.nY = P->d.nY; a.nZ = P->d.nZ; a.nU = P->d.nU; a.nV = P->d.nV;
    a.dVX = P->d.dVX; a.dVY = P->d.dVY; a.dVZ = P->d.dVZ; a.acc = P->d.accuracy;
    const bool nearest = P->d.accuracy > 1.0;
    const int rows = 8;
    dim3 block(32, rows);
    dim3 grid((P->d.nU + 31) / 32, (P->d.nV + rows - 1) / rows, 1);
    const int na = a1 - a0;
    for (int c = 0; c < na; c += 65535) {
        InterpArgs ac = a;
        ac.a0 = a0 + c;
        ac.proj = (char*)proj + (size_t)c * P->d.nU * P->d.nV * dtype_size(pdt);
        grid.z = std::min(65535, na - c);
        if (vdt == TIGRE_F32 && pdt == TIGRE_F32) launch_typed<float, float>(ac, nearest, grid, block, st);
        else if (vdt == TIGRE_BF16 && pdt == TIGRE_BF16)
            launch_typed<__nv_bfloat16, __nv_bfloat16>(ac, nearest, grid, block, st);
        else if (vdt == TIGRE_F16 && pdt == TIGRE_F16) launch_typed<__half, __half>(ac, nearest, grid, block, st);
        else if (vdt == TIGRE_BF16 && pdt == TIGRE_F32) launch_typed<__nv_bfloat16, float>(ac, nearest, grid, block, st);
        else if (vdt == TIGRE_F16 && pdt == TIGRE_F32) launch_typed<__half, float>(ac, nearest, grid, block, st);
        else return fail(TIGRE_ERR_BAD_ASSERT, "unsupported dtype pair for interpolated projection");
        TIGRE_LAUNCHED();
    }
    return TIGRE_SUCCESS;
}

}  // namespace tigre
