// Siddon (Jacobs) ray-driven cone-beam forward projection for sm_100a.
//
// Computes, per detector pixel, the line integral of the voxel volume along
// the source->pixel ray: sum over voxel segments of (segment length) x value,
// as kernelPixelDetector does (Common/CUDA/Siddon_projection.cu:110-268),
// including its conventions: detector rows flipped (pixelV = nV-1-v, :141),
// ray components below 1e-3 voxel treated as parallel (:156-159), no clipping
// of the ray parameter to [source, detector] (:168-176), result scaled by the
// ray length in mm (:241,267).
//
// Design (B200):
//  * one thread per ray; a warp covers 32 neighbouring detector columns of one
//    row; a block covers 32 x 8 pixels of one view;
//  * the volume is read from the working layout in which those 32 rays sit on
//    consecutive addresses (x-fastest caller copy, or the y-fastest transposed
//    copy, chosen per view), so each warp gather touches 1-2 cache lines;
//  * ray entry/exit, first crossings and per-axis crossing increments are
//    computed in FP64 once per ray; the traversal runs in FP32 in "alpha from
//    entry" units, each crossing evaluated directly as t0 + k*dt (no running
//    sum, so no drift along the ray);
//  * per-axis remaining-crossing counters stop each axis at its last voxel, so
//    every gather is in bounds without a per-step bounds test.

#include <cmath>

#include "tigre_internal.h"

namespace tigre {
namespace {

struct SiddonArgs {
    const void* vol_x;
    const void* vol_y;
    void* proj;
    const FrameSiddon* frames;
    int a0;
    int nX, nY, nZ, nU, nV;
    double dVX, dVY, dVZ;
    unsigned long long* count;   // segment-count mode
};

constexpr float kInf = __builtin_huge_valf();

struct AxisSetup {
    int i;          // first voxel index along the axis
    int rem;        // crossings available before leaving the box
    int step;       // +1 / -1 / 0
    float t0, dt;   // first crossing (alpha from entry) and increment
    long long ncross;  // crossings strictly inside the segment [0, T) (count mode)
};

__device__ __forceinline__ AxisSetup axis_setup(double s, double r, double am, double aM, int n) {
    AxisSetup a;
    double e = fma(am, r, s);
    e = fmin(fmax(e, 0.0), (double)n);
    if (r > 0.0) {
        const double k = floor(e) + 1.0;
        a.i = min((int)k - 1, n - 1);
        a.rem = n - 1 - a.i;
        a.step = 1;
        a.t0 = (float)((k - e) / r);
        a.dt = (float)(1.0 / r);
        const double x = fma(aM, r, s);
        a.ncross = max(0LL, min((long long)a.rem, (long long)ceil(x) - 1 - (long long)k + 1));
    } else if (r < 0.0) {
        const double k = ceil(e) - 1.0;
        a.i = max((int)k, 0);
        a.rem = a.i;
        a.step = -1;
        a.t0 = (float)((k - e) / r);
        a.dt = (float)(-1.0 / r);
        const double x = fma(aM, r, s);
        a.ncross = max(0LL, min((long long)a.rem, (long long)k - (long long)floor(x) - 1 + 1));
    } else {
        a.i = min(max((int)floor(e), 0), n - 1);
        a.rem = 0;
        a.step = 0;
        a.t0 = kInf;
        a.dt = 0.f;
        a.ncross = 0;
    }
    if (a.rem <= 0) a.t0 = kInf;
    return a;
}

struct RaySetup {
    bool hit;
    double r[3];
    double am, aM;
};

__device__ __forceinline__ RaySetup ray_setup(const SiddonArgs& p, const FrameSiddon& F, int u, int v) {
    RaySetup R;
    const double pv = (double)(p.nV - 1 - v);   // detector v flip, Siddon_projection.cu:141
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        R.r[k] = fma(pv, F.dv[k], fma((double)u, F.du[k], F.o[k])) - F.s[k];
        if (fabs(R.r[k]) < 0.001) R.r[k] = 0.0;   // Siddon_projection.cu:156-159
    }
    const int n[3] = {p.nX, p.nY, p.nZ};
    double am = -1e300, aM = 1e300;
    bool miss = false;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        if (R.r[k] != 0.0) {
            const double inv = 1.0 / R.r[k];
            const double a0 = -F.s[k] * inv, a1 = ((double)n[k] - F.s[k]) * inv;
            am = fmax(am, fmin(a0, a1));
            aM = fmin(aM, fmax(a0, a1));
        } else if (F.s[k] < 0.0 || F.s[k] > (double)n[k]) {
            miss = true;
        }
    }
    R.am = am;
    R.aM = aM;
    R.hit = !miss && am < aM;
    return R;
}

template <typename TV, typename TP>
__global__ void __launch_bounds__(256) siddon_kernel(SiddonArgs p) {
    const int u = blockIdx.x * 32 + threadIdx.x;
    const int v = blockIdx.y * blockDim.y + threadIdx.y;
    const int la = blockIdx.z;
    if (u >= p.nU || v >= p.nV) return;
    const FrameSiddon& F = p.frames[p.a0 + la];
    const RaySetup R = ray_setup(p, F, u, v);
    const size_t oidx = ((size_t)la * p.nV + v) * (size_t)p.nU + u;
    if (!R.hit) {
        ((TP*)p.proj)[oidx] = from_f32<TP>(0.f);
        return;
    }
    const AxisSetup ax = axis_setup(F.s[0], R.r[0], R.am, R.aM, p.nX);
    const AxisSetup ay = axis_setup(F.s[1], R.r[1], R.am, R.aM, p.nY);
    const AxisSetup az = axis_setup(F.s[2], R.r[2], R.am, R.aM, p.nZ);
    // strides of the working layout chosen for this view
    const int layout = F.layout;
    const TV* vol = (const TV*)(layout ? p.vol_y : p.vol_x);
    const int stx = layout ? p.nY : 1;
    const int sty = layout ? 1 : p.nX;
    const int stz = p.nX * p.nY;
    int idx = ax.i * stx + ay.i * sty + az.i * stz;
    const int dix = ax.step * stx, diy = ay.step * sty, diz = az.step * stz;
    int remx = ax.rem, remy = ay.rem, remz = az.rem;
    float tx = ax.t0, ty = ay.t0, tz = az.t0;
    float kx = 0.f, ky = 0.f, kz = 0.f;
    const float T = (float)(R.aM - R.am);
    float tc = 0.f, sum = 0.f;
#pragma unroll 1
    for (;;) {
        const float tn = fminf(fminf(tx, ty), tz);
        const float val = ldg_f<TV>(vol + idx);
        if (tn >= T) {
            sum = fmaf(T - tc, val, sum);
            break;
        }
        sum = fmaf(tn - tc, val, sum);
        tc = tn;
        if (tx == tn) {
            idx += dix;
            kx += 1.f;
            tx = (--remx > 0) ? fmaf(kx, ax.dt, ax.t0) : kInf;
        } else if (ty == tn) {
            idx += diy;
            ky += 1.f;
            ty = (--remy > 0) ? fmaf(ky, ay.dt, ay.t0) : kInf;
        } else {
            idx += diz;
            kz += 1.f;
            tz = (--remz > 0) ? fmaf(kz, az.dt, az.t0) : kInf;
        }
    }
    const double* r = R.r;
    const double len = sqrt(r[0] * r[0] * p.dVX * p.dVX + r[1] * r[1] * p.dVY * p.dVY + r[2] * r[2] * p.dVZ * p.dVZ);
    ((TP*)p.proj)[oidx] = from_f32<TP>(sum * (float)len);
}

// Number of voxel segments per ray (crossings inside the box + 1), summed with
// one atomic per warp; no traversal.
__global__ void __launch_bounds__(256) siddon_count_kernel(SiddonArgs p) {
    const int u = blockIdx.x * 32 + threadIdx.x;
    const int v = blockIdx.y * blockDim.y + threadIdx.y;
    unsigned long long c = 0;
    if (u < p.nU && v < p.nV) {
        const FrameSiddon& F = p.frames[p.a0 + blockIdx.z];
        const RaySetup R = ray_setup(p, F, u, v);
        if (R.hit) {
            const AxisSetup ax = axis_setup(F.s[0], R.r[0], R.am, R.aM, p.nX);
            const AxisSetup ay = axis_setup(F.s[1], R.r[1], R.am, R.aM, p.nY);
            const AxisSetup az = axis_setup(F.s[2], R.r[2], R.am, R.aM, p.nZ);
            c = 1 + ax.ncross + ay.ncross + az.ncross;
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) c += __shfl_down_sync(0xffffffffu, c, o);
    if ((threadIdx.x & 31) == 0 && c) atomicAdd(p.count, c);
}

SiddonArgs make_args(TigrePlan* P, int a0) {
    SiddonArgs a{};
    a.frames = P->d_siddon;
    a.a0 = a0;
    a.nX = P->d.nX; a.nY = P->d.nY; a.nZ = P->d.nZ; a.nU = P->d.nU; a.nV = P->d.nV;
    a.dVX = P->d.dVX; a.dVY = P->d.dVY; a.dVZ = P->d.dVZ;
    return a;
}

constexpr int kRowsPerBlock = 8;

}  // namespace

int launch_siddon(TigrePlan* P, const void* vol_x, const void* vol_y, int vdt, void* proj, int pdt, int a0, int a1,
                  cudaStream_t st) {
    SiddonArgs a = make_args(P, a0);
    a.vol_x = vol_x; a.vol_y = vol_y; a.proj = proj;
    const int na = a1 - a0;
    dim3 block(32, kRowsPerBlock);
    dim3 grid((P->d.nU + 31) / 32, (P->d.nV + kRowsPerBlock - 1) / kRowsPerBlock, 1);
    // grid.z is limited to 65535 views per launch
    for (int c = 0; c < na; c += 65535) {
        const int cnt = std::min(65535, na - c);
        SiddonArgs ac = a;
        ac.a0 = a0 + c;
        ac.proj = (char*)proj + (size_t)c * P->d.nU * P->d.nV * dtype_size(pdt);
        grid.z = cnt;
        if (vdt == TIGRE_F32 && pdt == TIGRE_F32) siddon_kernel<float, float><<<grid, block, 0, st>>>(ac);
        else if (vdt == TIGRE_BF16 && pdt == TIGRE_BF16)
            siddon_kernel<__nv_bfloat16, __nv_bfloat16><<<grid, block, 0, st>>>(ac);
        else if (vdt == TIGRE_F16 && pdt == TIGRE_F16) siddon_kernel<__half, __half><<<grid, block, 0, st>>>(ac);
        else if (vdt == TIGRE_BF16 && pdt == TIGRE_F32)
            siddon_kernel<__nv_bfloat16, float><<<grid, block, 0, st>>>(ac);
        else if (vdt == TIGRE_F16 && pdt == TIGRE_F32) siddon_kernel<__half, float><<<grid, block, 0, st>>>(ac);
        else if (vdt == TIGRE_F32 && pdt == TIGRE_BF16)
            siddon_kernel<float, __nv_bfloat16><<<grid, block, 0, st>>>(ac);
        else if (vdt == TIGRE_F32 && pdt == TIGRE_F16) siddon_kernel<float, __half><<<grid, block, 0, st>>>(ac);
        else return fail(TIGRE_ERR_BAD_ASSERT, "unsupported dtype pair for Siddon");
        TIGRE_CUDA(cudaGetLastError());
    }
    return TIGRE_SUCCESS;
}

int launch_siddon_count(TigrePlan* P, int a0, int a1, unsigned long long* d_total, cudaStream_t st) {
    SiddonArgs a = make_args(P, a0);
    a.count = d_total;
    const int na = a1 - a0;
    dim3 block(32, kRowsPerBlock);
    dim3 grid((P->d.nU + 31) / 32, (P->d.nV + kRowsPerBlock - 1) / kRowsPerBlock, 1);
    for (int c = 0; c < na; c += 65535) {
        SiddonArgs ac = a;
        ac.a0 = a0 + c;
        grid.z = std::min(65535, na - c);
        siddon_count_kernel<<<grid, block, 0, st>>>(ac);
        TIGRE_CUDA(cudaGetLastError());
    }
    return TIGRE_SUCCESS;
}

}  // namespace tigre
