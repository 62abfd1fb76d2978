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

#include <cstdlib>

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
    int zpad;                    // zero slices before and after each z-run of the z-fast copy
    int parallel;                // parallel beam: each pixel's source is s + u du + v dv
    int* status;                 // plan status word (bit 1: a ray outside the host's z bound)
    int grid_nug, grid_nviews, grid_vtile;   // cell kernel: 1-D grid of u groups x views x row bands
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
    double s[3];   // source of this ray (the view's source, or the pixel's in parallel beam)
    double am, aM;
};

__device__ __forceinline__ RaySetup ray_setup(const SiddonArgs& p, const FrameSiddon& F, int u, int v) {
    RaySetup R;
    const double pv = (double)(p.nV - 1 - v);   // detector v flip, Siddon_projection.cu:141
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        R.s[k] = p.parallel ? fma(pv, F.dv[k], fma((double)u, F.du[k], F.s[k])) : F.s[k];
        R.r[k] = fma(pv, F.dv[k], fma((double)u, F.du[k], F.o[k])) - R.s[k];
        if (fabs(R.r[k]) < 0.001) R.r[k] = 0.0;   // Siddon_projection.cu:156-159
    }
    const int n[3] = {p.nX, p.nY, p.nZ};
    double am = -1e300, aM = 1e300;
    bool miss = false;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        if (R.r[k] != 0.0) {
            const double inv = 1.0 / R.r[k];
            const double a0 = -R.s[k] * inv, a1 = ((double)n[k] - R.s[k]) * inv;
            am = fmax(am, fmin(a0, a1));
            aM = fmin(aM, fmax(a0, a1));
        } else if (R.s[k] < 0.0 || R.s[k] > (double)n[k]) {
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
    const AxisSetup ax = axis_setup(R.s[0], R.r[0], R.am, R.aM, p.nX);
    const AxisSetup ay = axis_setup(R.s[1], R.r[1], R.am, R.aM, p.nY);
    const AxisSetup az = axis_setup(R.s[2], R.r[2], R.am, R.aM, p.nZ);
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
            const AxisSetup ax = axis_setup(R.s[0], R.r[0], R.am, R.aM, p.nX);
            const AxisSetup ay = axis_setup(R.s[1], R.r[1], R.am, R.aM, p.nY);
            const AxisSetup az = axis_setup(R.s[2], R.r[2], R.am, R.aM, p.nZ);
            c = 1 + ax.ncross + ay.ncross + az.ncross;
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) c += __shfl_down_sync(0xffffffffu, c, o);
    if ((threadIdx.x & 31) == 0 && c) atomicAdd(p.count, c);
}

// ---------------------------------------------------------------------------
// Column-coherent Siddon.  When the detector's v axis is parallel to the
// volume's z axis (no tilt: theta = psi = 0 and no detector roll/pitch/yaw),
// every ray of one detector column lies in the same vertical plane through the
// source: all of them share x- and y-components of direction and therefore
// the same sequence of x/y plane crossings.  One warp takes one column and
// 32*R of its rows (row = lane + 32 r): the xy traversal is warp-uniform (no
// divergence), and each row only adds its own z crossings, which are rare at
// cone-beam angles.  The volume is read from a z-fastest copy (x, y, z) with
// one zero voxel before and after each z-run, so the 32 lanes of a warp load
// ~17 consecutive floats of the same (x, y) column per step, and a ray that
// leaves the volume through its top or bottom reads zeros.  Grid order
// (column groups fastest, then views, then row tiles) keeps the z-slab of the
// current row tile L2-resident while every view is processed.
template <typename TV, typename TP, int R, bool SINGLE>
__global__ void __launch_bounds__(128, 6) siddon_columns_kernel(SiddonArgs p) {
    const int lane = threadIdx.x & 31;
    const int u = blockIdx.x * 4 + (threadIdx.x >> 5);
    const int la = blockIdx.y;
    if (u >= p.nU) return;
    const FrameSiddon& F = p.frames[p.a0 + la];
    const int vbase = blockIdx.z * (32 * R) + lane;
    TP* out = (TP*)p.proj + (size_t)la * p.nV * p.nU + u;
    // ---- shared xy ray (identical in every lane of the warp); in parallel beam the column's
    // source is s + u du (dv has no xy part on this path) ----
    const double sx = p.parallel ? fma((double)u, F.du[0], F.s[0]) : F.s[0];
    const double sy = p.parallel ? fma((double)u, F.du[1], F.s[1]) : F.s[1];
    double rx = fma((double)u, F.du[0], F.o[0]) - sx;
    double ry = fma((double)u, F.du[1], F.o[1]) - sy;
    if (fabs(rx) < 0.001) rx = 0.0;   // Siddon_projection.cu:156-159
    if (fabs(ry) < 0.001) ry = 0.0;
    double am = -1e300, aM = 1e300;
    bool miss = false;
    if (rx != 0.0) {
        const double i = 1.0 / rx, a0 = -sx * i, a1 = ((double)p.nX - sx) * i;
        am = fmax(am, fmin(a0, a1)); aM = fmin(aM, fmax(a0, a1));
    } else if (sx < 0.0 || sx > (double)p.nX) miss = true;
    if (ry != 0.0) {
        const double i = 1.0 / ry, a0 = -sy * i, a1 = ((double)p.nY - sy) * i;
        am = fmax(am, fmin(a0, a1)); aM = fmin(aM, fmax(a0, a1));
    } else if (sy < 0.0 || sy > (double)p.nY) miss = true;
    if (miss || !(am < aM)) {
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const int v = vbase + 32 * r;
            if (v < p.nV) out[(size_t)v * p.nU] = from_f32<TP>(0.f);
        }
        return;
    }
    const AxisSetup ax = axis_setup(sx, rx, am, aM, p.nX);
    const AxisSetup ay = axis_setup(sy, ry, am, aM, p.nY);
    const int ncells = 1 + (int)ax.ncross + (int)ay.ncross;
    const float T = (float)(aM - am);
    // ---- per-row z state ----
    int iz[R], sz[R];
    float tz[R], tz0[R], dtz[R], kz[R], sum[R], len[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const int v = min(vbase + 32 * r, p.nV - 1);
        const double pv = (double)(p.nV - 1 - v);
        const double srcz = p.parallel ? fma(pv, F.dv[2], fma((double)u, F.du[2], F.s[2])) : F.s[2];
        double rz = fma(pv, F.dv[2], fma((double)u, F.du[2], F.o[2])) - srcz;
        if (fabs(rz) < 0.001) rz = 0.0;
        const double ze = fma(am, rz, srcz);
        int z = (int)fmin(fmax(floor(ze), -1.0), (double)p.nZ);
        iz[r] = z;
        sum[r] = 0.f;
        kz[r] = 0.f;
        len[r] = (float)sqrt(rx * rx * p.dVX * p.dVX + ry * ry * p.dVY * p.dVY + rz * rz * p.dVZ * p.dVZ);
        if (rz > 0.0 && z < p.nZ) {
            sz[r] = 1;
            tz0[r] = (float)(((double)(z + 1) - srcz) / rz - am);
            dtz[r] = (float)(1.0 / rz);
        } else if (rz < 0.0 && z >= 0) {
            sz[r] = -1;
            tz0[r] = (float)(((double)z - srcz) / rz - am);
            dtz[r] = (float)(-1.0 / rz);
        } else {
            sz[r] = 0;
            tz0[r] = kInf;
            dtz[r] = 0.f;
        }
        tz[r] = tz0[r];
    }
    const TV* __restrict__ vol = (const TV*)p.vol_x;
    const int ZP = p.nZ + 2 * p.zpad;
    int cidx = ax.i * p.nY + ay.i;
    const int dcx = ax.step * p.nY, dcy = ay.step;
    int remx = ax.rem, remy = ay.rem;
    float tx = ax.t0, ty = ay.t0, kx = 0.f, ky = 0.f;
    float a = 0.f;
    // value of each row's current voxel in the current cell, loaded one cell ahead
    float vcur[R];
    {
        const TV* col = vol + cidx * ZP + 1;
#pragma unroll
        for (int r = 0; r < R; ++r) vcur[r] = ldg_f<TV>(col + iz[r]);
    }
#pragma unroll 1
    for (int c = 0; c < ncells; ++c) {
        const float tn = fminf(tx, ty);
        const float b = fminf(tn, T);
        const float seg = b - a;
        const TV* col = vol + cidx * ZP + 1;
        bool again = false;
#pragma unroll
        for (int r = 0; r < R; ++r) {
            // no-crossing contribution; a z crossing at tz inside the cell adds
            // (b - tz) * (v_after - v_before).  The first crossing is handled by a short
            // predicated body; z indices are clamped to the zero pads [-1, nZ], so a ray
            // that has left the volume keeps crossing planes at no cost and reads 0.
            sum[r] = fmaf(seg, vcur[r], sum[r]);
            if (tz[r] < b) {
                const int izn = min(max(iz[r] + sz[r], -1), p.nZ);
                const float vn = ldg_f<TV>(col + izn);
                sum[r] = fmaf(b - tz[r], vn - vcur[r], sum[r]);
                vcur[r] = vn;
                iz[r] = izn;
                kz[r] += 1.f;
                tz[r] = fmaf(kz[r], dtz[r], tz0[r]);
                if (!SINGLE) again |= tz[r] < b;
            }
        }
        if (!SINGLE && __any_sync(0xffffffffu, again)) {
            // steep rays: further crossings inside the same cell (warp-uniform, rare)
#pragma unroll
            for (int r = 0; r < R; ++r) {
                while (tz[r] < b) {
                    const int izn = min(max(iz[r] + sz[r], -1), p.nZ);
                    const float vn = ldg_f<TV>(col + izn);
                    sum[r] = fmaf(b - tz[r], vn - vcur[r], sum[r]);
                    vcur[r] = vn;
                    iz[r] = izn;
                    kz[r] += 1.f;
                    tz[r] = fmaf(kz[r], dtz[r], tz0[r]);
                }
            }
        }
        a = b;
        const bool stepx = tx <= ty;
        cidx += stepx ? dcx : dcy;
        if (stepx) {
            kx += 1.f;
            tx = (--remx > 0) ? fmaf(kx, ax.dt, ax.t0) : kInf;
        } else {
            ky += 1.f;
            ty = (--remy > 0) ? fmaf(ky, ay.dt, ay.t0) : kInf;
        }
        if (c + 1 < ncells) {
            const TV* nc = vol + cidx * ZP + 1;
#pragma unroll
            for (int r = 0; r < R; ++r) vcur[r] = ldg_f<TV>(nc + iz[r]);
        }
    }
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const int v = vbase + 32 * r;
        if (v < p.nV) out[(size_t)v * p.nU] = from_f32<TP>(sum[r] * len[r]);
    }
}

// Cell-interval Siddon, for plans whose rays change z by less than one slice per xy
// cell (the host checks this exactly for every ray).  Same warp organisation as
// siddon_columns_kernel, but the z state is not stepped: with z(alpha) = zA + alpha*rz
// the slice at the end b of each xy cell is floor(z(b)), and since at most one z plane
// lies inside the cell, its contribution is
//     seg * v(z_start) + (b - alpha_k) * (v(z_end) - v(z_start)),
// where alpha_k is the crossing, taken in alpha space from the crossing count
// (alpha_k = tz0 + (z_end - q) / rz, exact small integers in the difference).  Without a
// crossing v(z_end) = v(z_start) and the second term is zero, so every cell of every row
// runs the same branch-free code on the FMA pipe, two rows at a time in packed FP32x2.
// The floor is a round-toward-zero add of 1.5*2^23 (z is kept positive by the pads), and
// its float bits index the column directly.  The pads (at least the largest z extent of
// any ray inside the xy box, from the host) make every index valid without clamping:
// a ray whose z range misses the volume reads one zero slice.
constexpr int kCellWarps = 4;                  // warps (neighbouring detector columns) per block
constexpr float kMagic = 12582912.0f;          // 1.5 * 2^23
constexpr unsigned kMagicBits = 0x4B400000u;   // its bit pattern

__device__ __forceinline__ float2 pk(float a, float b) { return make_float2(a, b); }
__device__ __forceinline__ float2 pk(float a) { return make_float2(a, a); }

template <typename TV>
__device__ __forceinline__ float ldz(uintptr_t cb, float t) {
    return ldg_f<TV>(reinterpret_cast<const TV*>(cb + (uintptr_t)__float_as_uint(t) * sizeof(TV)));
}

template <typename TV, typename TP, int R>
__global__ void __launch_bounds__(32 * kCellWarps, (R >= 8 ? 16 : 24) / kCellWarps) siddon_cells_kernel(SiddonArgs p) {
    static_assert(R % 2 == 0, "rows are processed in pairs");
    constexpr int H = R / 2;
    const int lane = threadIdx.x & 31;
    // Block order: row band slowest, then tiles of grid_vtile views; inside a tile the views
    // vary fastest, so the blocks resident at one time are a few u groups of many
    // neighbouring views, whose rays cross nearly the same voxel columns (L2 reuse).
    const long per_band = (long)p.grid_nug * p.grid_nviews;
    const int band = (int)(blockIdx.x / per_band);
    const long rr = blockIdx.x - (long)band * per_band;
    const long tile_blocks = (long)p.grid_nug * p.grid_vtile;
    const int vt = (int)(rr / tile_blocks);
    const int r2 = (int)(rr - (long)vt * tile_blocks);
    const int tsize = min(p.grid_vtile, p.grid_nviews - vt * p.grid_vtile);
    const int ug = r2 / tsize;
    const int la = vt * p.grid_vtile + (r2 - ug * tsize);
    const int u = ug * kCellWarps + (threadIdx.x >> 5);
    if (u >= p.nU) return;
    const FrameSiddon& F = p.frames[p.a0 + la];
    const int vbase = band * (32 * R) + lane;
    TP* out = (TP*)p.proj + (size_t)la * p.nV * p.nU + u;
    // ---- shared xy ray ----
    const double sx = p.parallel ? fma((double)u, F.du[0], F.s[0]) : F.s[0];
    const double sy = p.parallel ? fma((double)u, F.du[1], F.s[1]) : F.s[1];
    double rx = fma((double)u, F.du[0], F.o[0]) - sx;
    double ry = fma((double)u, F.du[1], F.o[1]) - sy;
    if (fabs(rx) < 0.001) rx = 0.0;   // Siddon_projection.cu:156-159
    if (fabs(ry) < 0.001) ry = 0.0;
    double am = -1e300, aM = 1e300;
    bool miss = false;
    if (rx != 0.0) {
        const double i = 1.0 / rx, a0 = -sx * i, a1 = ((double)p.nX - sx) * i;
        am = fmax(am, fmin(a0, a1)); aM = fmin(aM, fmax(a0, a1));
    } else if (sx < 0.0 || sx > (double)p.nX) miss = true;
    if (ry != 0.0) {
        const double i = 1.0 / ry, a0 = -sy * i, a1 = ((double)p.nY - sy) * i;
        am = fmax(am, fmin(a0, a1)); aM = fmin(aM, fmax(a0, a1));
    } else if (sy < 0.0 || sy > (double)p.nY) miss = true;
    if (miss || !(am < aM)) {
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const int v = vbase + 32 * r;
            if (v < p.nV) out[(size_t)v * p.nU] = from_f32<TP>(0.f);
        }
        return;
    }
    const AxisSetup ax = axis_setup(sx, rx, am, aM, p.nX);
    const AxisSetup ay = axis_setup(sy, ry, am, aM, p.nY);
    const int ncells = 1 + (int)ax.ncross + (int)ay.ncross;
    const double Td = aM - am;
    const float T = (float)Td;
    const double P = (double)p.zpad;
    // ---- per-row z state, rows (2h, 2h+1) packed in .x/.y ----
    float2 zA[H], rz[H], nm[H], nQ[H], ntz0[H], sum[H], t0[H];
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const int v = min(vbase + 32 * r, p.nV - 1);
        const double pv = (double)(p.nV - 1 - v);
        const double szr = p.parallel ? fma(pv, F.dv[2], fma((double)u, F.du[2], F.s[2])) : F.s[2];
        double rzd = fma(pv, F.dv[2], fma((double)u, F.du[2], F.o[2])) - szr;
        if (fabs(rzd) < 0.001) rzd = 0.0;
        const double za = fma(am, rzd, szr) + P;   // z + pad at the xy entry
        const double zb = fma(Td, rzd, za);           // ... and at the xy exit
        const double lo = fmin(za, zb), hi = fmax(za, zb);
        bool live = hi > P && lo < P + (double)p.nZ;
        if (live && hi - lo > P - 1.5) {              // beyond the host's bound: not expected
            live = false;
            if (p.status) atomicOr(p.status, 2);
        }
        float zaf = (float)(P - 0.5), rzf = 0.f, m = 0.f, q = 0.f, tz = 0.f;
        if (live) {
            zaf = (float)za;
            rzf = (float)rzd;
            const float zs = __fadd_rz(zaf, kMagic) - kMagic;   // floor(zA) as the loop computes it
            if (rzd > 0.0) {
                q = zs + 1.f;
                tz = (float)(((double)zs + 1.0 - za) / rzd);
                m = (float)(1.0 / rzd);
            } else if (rzd < 0.0) {
                q = zs - 1.f;
                tz = (float)(((double)zs - za) / rzd);
                m = (float)(1.0 / rzd);
            }
        }
        const float t = __fadd_rz(zaf, kMagic);
        if (r & 1) {
            zA[r >> 1].y = zaf; rz[r >> 1].y = rzf; nm[r >> 1].y = -m; nQ[r >> 1].y = -(kMagic + q);
            ntz0[r >> 1].y = -tz; sum[r >> 1].y = 0.f; t0[r >> 1].y = t;
        } else {
            zA[r >> 1].x = zaf; rz[r >> 1].x = rzf; nm[r >> 1].x = -m; nQ[r >> 1].x = -(kMagic + q);
            ntz0[r >> 1].x = -tz; sum[r >> 1].x = 0.f; t0[r >> 1].x = t;
        }
    }
    const uintptr_t vb = (uintptr_t)p.vol_x - (uintptr_t)kMagicBits * sizeof(TV);
    const uintptr_t colb = (uintptr_t)(p.nZ + 2 * p.zpad) * sizeof(TV);
    int cidx = ax.i * p.nY + ay.i;
    const int dcx = ax.step * p.nY, dcy = ay.step;
    int remx = ax.rem, remy = ay.rem;
    float tx = ax.t0, ty = ay.t0, kx = 0.f, ky = 0.f;
    float a = 0.f;
    // Software pipeline over cells: front() of cell k+1 (its bounds, floors and the four loads
    // per row pair) is issued before back() of cell k (the accumulation), so the loads of one
    // cell are in flight while the previous one is summed.  Two state sets, A and B, alternate.
    struct Cell {
        float seg;
        float2 d[H], v0[H], v1[H];
    };
    auto front = [&](Cell& C) {
        const float b = fminf(fminf(tx, ty), T);
        const float2 b2 = pk(b);
        C.seg = b - a;
        const uintptr_t cb = vb + (uintptr_t)cidx * colb;
#pragma unroll
        for (int h = 0; h < H; ++h) {
            const float2 zf = __ffma2_rn(b2, rz[h], zA[h]);
            const float2 t1 = __fadd2_rz(zf, pk(kMagic));                       // kMagic + floor(z(b))
            const float2 kq = __fadd2_rn(t1, nQ[h]);                            // z_end - q, exact
            C.d[h] = __fadd2_rn(b2, __ffma2_rn(kq, nm[h], ntz0[h]));            // b - alpha_k
            C.v0[h] = pk(ldz<TV>(cb, t0[h].x), ldz<TV>(cb, t0[h].y));
            C.v1[h] = pk(ldz<TV>(cb, t1.x), ldz<TV>(cb, t1.y));
            t0[h] = t1;
        }
        a = b;
        const bool stepx = tx <= ty;
        cidx += stepx ? dcx : dcy;
        if (stepx) {
            kx += 1.f;
            tx = (--remx > 0) ? fmaf(kx, ax.dt, ax.t0) : kInf;
        } else {
            ky += 1.f;
            ty = (--remy > 0) ? fmaf(ky, ay.dt, ay.t0) : kInf;
        }
    };
    auto back = [&](const Cell& C) {
        const float2 seg2 = pk(C.seg);
#pragma unroll
        for (int h = 0; h < H; ++h) {
            sum[h] = __ffma2_rn(seg2, C.v0[h], sum[h]);
            sum[h] = __ffma2_rn(C.d[h], __ffma2_rn(C.v0[h], pk(-1.f), C.v1[h]), sum[h]);
        }
    };
    Cell A, B;
    front(A);
    int c = 1;
#pragma unroll 1
    while (true) {
        if (c >= ncells) { back(A); break; }
        front(B);
        back(A);
        if (++c >= ncells) { back(B); break; }
        front(A);
        back(B);
        ++c;
    }
    const double lxy = rx * rx * p.dVX * p.dVX + ry * ry * p.dVY * p.dVY;
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const int v = vbase + 32 * r;
        if (v < p.nV) {
            const double pv = (double)(p.nV - 1 - v);
            const double szr = p.parallel ? fma(pv, F.dv[2], fma((double)u, F.du[2], F.s[2])) : F.s[2];
            double rzd = fma(pv, F.dv[2], fma((double)u, F.du[2], F.o[2])) - szr;
            if (fabs(rzd) < 0.001) rzd = 0.0;
            const float len = (float)sqrt(lxy + rzd * rzd * p.dVZ * p.dVZ);
            const float sr = (r & 1) ? sum[r >> 1].y : sum[r >> 1].x;
            out[(size_t)v * p.nU] = from_f32<TP>(sr * len);
        }
    }
}

SiddonArgs make_args(TigrePlan* P, int a0) {
    SiddonArgs a{};
    a.frames = P->d_siddon;
    a.a0 = a0;
    a.nX = P->d.nX; a.nY = P->d.nY; a.nZ = P->d.nZ; a.nU = P->d.nU; a.nV = P->d.nV;
    a.dVX = P->d.dVX; a.dVY = P->d.dVY; a.dVZ = P->d.dVZ;
    a.zpad = 1;
    a.parallel = P->parallel ? 1 : 0;
    a.status = P->d_status;
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
        TIGRE_LAUNCHED();
    }
    return TIGRE_SUCCESS;
}

template <typename TV, typename TP, bool SINGLE>
static void launch_columns_r(const SiddonArgs& a, int rows_per_thread, dim3 grid, cudaStream_t st) {
    if (rows_per_thread == 4) siddon_columns_kernel<TV, TP, 4, SINGLE><<<grid, 128, 0, st>>>(a);
    else if (rows_per_thread == 2) siddon_columns_kernel<TV, TP, 2, SINGLE><<<grid, 128, 0, st>>>(a);
    else siddon_columns_kernel<TV, TP, 1, SINGLE><<<grid, 128, 0, st>>>(a);
}

template <typename TV, typename TP>
static void launch_columns_typed(const SiddonArgs& a, int rows_per_thread, bool single, dim3 grid, cudaStream_t st) {
    if (single) launch_columns_r<TV, TP, true>(a, rows_per_thread, grid, st);
    else launch_columns_r<TV, TP, false>(a, rows_per_thread, grid, st);
}

int launch_siddon_columns(TigrePlan* P, const void* vol_z, int vdt, void* proj, int pdt, int a0, int a1,
                          cudaStream_t st) {
    SiddonArgs a = make_args(P, a0);
    a.vol_x = vol_z;
    a.proj = proj;
    const int nv = P->d.nV;
    const int R = nv >= 512 ? 4 : (nv >= 128 ? 2 : 1);
    // z advance per xy segment <= slope: below 1 a segment crosses at most one z plane
    const bool single = P->column_slope_max < 0.5;
    const int na = a1 - a0;
    for (int c = 0; c < na; c += 65535) {
        SiddonArgs ac = a;
        ac.a0 = a0 + c;
        ac.proj = (char*)proj + (size_t)c * P->d.nU * P->d.nV * dtype_size(pdt);
        dim3 grid((P->d.nU + 3) / 4, std::min(65535, na - c), (nv + 32 * R - 1) / (32 * R));
        if (vdt == TIGRE_F32 && pdt == TIGRE_F32) launch_columns_typed<float, float>(ac, R, single, grid, st);
        else if (vdt == TIGRE_BF16 && pdt == TIGRE_BF16) launch_columns_typed<__nv_bfloat16, __nv_bfloat16>(ac, R, single, grid, st);
        else if (vdt == TIGRE_F16 && pdt == TIGRE_F16) launch_columns_typed<__half, __half>(ac, R, single, grid, st);
        else if (vdt == TIGRE_BF16 && pdt == TIGRE_F32) launch_columns_typed<__nv_bfloat16, float>(ac, R, single, grid, st);
        else if (vdt == TIGRE_F16 && pdt == TIGRE_F32) launch_columns_typed<__half, float>(ac, R, single, grid, st);
        else if (vdt == TIGRE_F32 && pdt == TIGRE_BF16) launch_columns_typed<float, __nv_bfloat16>(ac, R, single, grid, st);
        else if (vdt == TIGRE_F32 && pdt == TIGRE_F16) launch_columns_typed<float, __half>(ac, R, single, grid, st);
        else return fail(TIGRE_ERR_BAD_ASSERT, "unsupported dtype pair for Siddon");
        TIGRE_LAUNCHED();
    }
    return TIGRE_SUCCESS;
}

template <typename TV, typename TP>
static void launch_cells_typed(const SiddonArgs& a, int rows_per_thread, dim3 grid, cudaStream_t st) {
    if (rows_per_thread == 8) siddon_cells_kernel<TV, TP, 8><<<grid, 32 * kCellWarps, 0, st>>>(a);
    else if (rows_per_thread == 4) siddon_cells_kernel<TV, TP, 4><<<grid, 32 * kCellWarps, 0, st>>>(a);
    else siddon_cells_kernel<TV, TP, 2><<<grid, 32 * kCellWarps, 0, st>>>(a);
}

int launch_siddon_cells(TigrePlan* P, const void* vol_z, int vdt, void* proj, int pdt, int a0, int a1,
                        cudaStream_t st) {
    SiddonArgs a = make_args(P, a0);
    a.vol_x = vol_z;
    a.proj = proj;
    a.zpad = P->cells_zpad;
    const int nv = P->d.nV;
    // rows per thread: 8 (256 rows per warp, 4 resident blocks per SM) for tall detectors
    const int R = nv >= 512 ? 8 : (nv >= 256 ? 4 : 2);
    const int vtile = 64;   // flat between 32 and 128 views at 512^3 / 1024x768
    const int na = a1 - a0;
    const int nug = (P->d.nU + kCellWarps - 1) / kCellWarps, nbands = (nv + 32 * R - 1) / (32 * R);
    const long max_views = std::max(1L, (long)INT32_MAX / ((long)nug * nbands));
    for (long c = 0; c < na; c += max_views) {
        SiddonArgs ac = a;
        ac.a0 = a0 + (int)c;
        ac.proj = (char*)proj + (size_t)c * P->d.nU * P->d.nV * dtype_size(pdt);
        ac.grid_nug = nug;
        ac.grid_nviews = (int)std::min<long>(max_views, na - c);
        ac.grid_vtile = std::min(vtile, ac.grid_nviews);
        dim3 grid((unsigned)((long)nug * ac.grid_nviews * nbands));
        if (vdt == TIGRE_F32 && pdt == TIGRE_F32) launch_cells_typed<float, float>(ac, R, grid, st);
        else if (vdt == TIGRE_BF16 && pdt == TIGRE_BF16) launch_cells_typed<__nv_bfloat16, __nv_bfloat16>(ac, R, grid, st);
        else if (vdt == TIGRE_F16 && pdt == TIGRE_F16) launch_cells_typed<__half, __half>(ac, R, grid, st);
        else if (vdt == TIGRE_BF16 && pdt == TIGRE_F32) launch_cells_typed<__nv_bfloat16, float>(ac, R, grid, st);
        else if (vdt == TIGRE_F16 && pdt == TIGRE_F32) launch_cells_typed<__half, float>(ac, R, grid, st);
        else if (vdt == TIGRE_F32 && pdt == TIGRE_BF16) launch_cells_typed<float, __nv_bfloat16>(ac, R, grid, st);
        else if (vdt == TIGRE_F32 && pdt == TIGRE_F16) launch_cells_typed<float, __half>(ac, R, grid, st);
        else return fail(TIGRE_ERR_BAD_ASSERT, "unsupported dtype pair for Siddon");
        TIGRE_LAUNCHED();
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
        TIGRE_LAUNCHED();
    }
    return TIGRE_SUCCESS;
}

}  // namespace tigre
