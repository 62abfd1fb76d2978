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

#include <climits>
#include <type_traits>
#include <cmath>

#include "tigre_internal.h"

namespace tigre {
namespace {

struct InterpArgs {
    const void* vol_x;   // padded, (nZ+3, nY+3, nX+3)       (point sampling)
    const void* vol_y;   // padded, (nZ+3, nX+3, nY+3)
    const void* quad_x;  // corner quads of vol_x / vol_y   (trilinear sampling)
    const void* quad_y;
    void* proj;
    const FrameInterp* frames;
    int a0;
    int nX, nY, nZ, nU, nV;
    double dVX, dVY, dVZ, acc;
    int parallel;        // parallel beam: each pixel's source is s + u du + v dv
};

// one corner quad (fast axis x z 2x2 block) as floats
template <typename TV> __device__ __forceinline__ float4 ldq(const void* base, uint32_t i);
template <> __device__ __forceinline__ float4 ldq<float>(const void* base, uint32_t i) {
    return __ldg(reinterpret_cast<const float4*>(base) + i);
}
template <> __device__ __forceinline__ float4 ldq<__nv_bfloat16>(const void* base, uint32_t i) {
    const uint2 r = __ldg(reinterpret_cast<const uint2*>(base) + i);
    return make_float4(__uint_as_float(r.x << 16), __uint_as_float(r.x & 0xffff0000u), __uint_as_float(r.y << 16),
                       __uint_as_float(r.y & 0xffff0000u));
}
template <> __device__ __forceinline__ float4 ldq<__half>(const void* base, uint32_t i) {
    const uint2 r = __ldg(reinterpret_cast<const uint2*>(base) + i);
    const float2 a = __half22float2(*reinterpret_cast<const __half2*>(&r.x));
    const float2 b = __half22float2(*reinterpret_cast<const __half2*>(&r.y));
    return make_float4(a.x, a.y, b.x, b.y);
}

// trilinear value from the quads of rows o and o+1 (fractions along fast, z, other); FP32
// quads carry the fast-axis differences already (make_quads_kernel), 16-bit ones the corners
template <typename TV>
__device__ __forceinline__ float tri(const float4 q0, const float4 q1, float ff, float fz, float fo) {
    float a0, a1, b0, b1;
    if constexpr (std::is_same<TV, float>::value) {
        a0 = fmaf(ff, q0.y, q0.x), a1 = fmaf(ff, q0.w, q0.z);
        b0 = fmaf(ff, q1.y, q1.x), b1 = fmaf(ff, q1.w, q1.z);
    } else {
        a0 = fmaf(ff, q0.y - q0.x, q0.x), a1 = fmaf(ff, q0.w - q0.z, q0.z);
        b0 = fmaf(ff, q1.y - q1.x, q1.x), b1 = fmaf(ff, q1.w - q1.z, q1.z);
    }
    const float r0 = fmaf(fz, a1 - a0, a0), r1 = fmaf(fz, b1 - b0, b0);
    return fmaf(fo, r1 - r0, r0);
}

__device__ __forceinline__ float2 pk2(float a, float b) { return make_float2(a, b); }
__device__ __forceinline__ float2 pk2(float a) { return make_float2(a, a); }

// FP64 ray setup of detector pixel (u, v): source s, step vector vec and the last sample index
// (the reference's length, capped per view).
__device__ __forceinline__ double interp_setup(const InterpArgs& p, const FrameInterp& F, int u, int v, double (&s)[3],
                                               double (&vec)[3]) {
    const double pv = (double)(p.nV - 1 - v);
    double d[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        s[k] = p.parallel ? fma(pv, F.dv[k], fma((double)u, F.du[k], F.s[k])) : F.s[k];
        d[k] = fma(pv, F.dv[k], fma((double)u, F.du[k], F.o[k])) - s[k];
    }
    const double len = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
    double length = ceil(len / p.acc);
#pragma unroll
    for (int k = 0; k < 3; ++k) vec[k] = d[k] / length;
    if (F.cap < length) length = ceil(F.cap);
    return length;
}

// Number of samples of each ray strictly inside the open box (-1, n) per axis -- the samples
// whose trilinear footprint can be nonzero, the count of the oracle's interp_ray -- summed
// over the launch into *total (the algorithmic-bytes numerator of the interpolated roofline).
__global__ void __launch_bounds__(256) interp_count_kernel(InterpArgs p, unsigned long long* total) {
    const int u = blockIdx.x * 32 + threadIdx.x;
    const int la = blockIdx.y;
    const int v = blockIdx.z * blockDim.y + threadIdx.y;
    unsigned long long c = 0;
    if (u < p.nU && v < p.nV) {
        const FrameInterp& F = p.frames[p.a0 + la];
        double s[3], vec[3];
        const double length = interp_setup(p, F, u, v, s, vec);
        double lo = F.first_sample, hi = length;
        const int n[3] = {p.nX, p.nY, p.nZ};
        bool empty = false;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            if (vec[k] != 0.0) {
                const double ta = (-1.0 - s[k]) / vec[k], tb = ((double)n[k] - s[k]) / vec[k];
                lo = fmax(lo, floor(fmin(ta, tb)) + 1.0);
                hi = fmin(hi, ceil(fmax(ta, tb)) - 1.0);
            } else if (s[k] <= -1.0 || s[k] >= (double)n[k]) {
                empty = true;
            }
        }
        if (!empty && lo <= hi) c = (unsigned long long)(hi - lo + 1.0);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) c += __shfl_down_sync(0xffffffffu, c, o);
    if ((threadIdx.x & 31) == 0 && c) atomicAdd(total, c);
}

template <typename TV, typename TP, bool NEAREST>
__global__ void __launch_bounds__(256) interp_kernel(InterpArgs p) {
    // grid: detector column groups fastest, then views, then bands of detector rows, so the
    // z-slab of the volume that one band of rows crosses stays L2-resident across all views
    const int u0 = blockIdx.x * 32 + threadIdx.x;
    const int la = blockIdx.y;
    const int v = blockIdx.z * blockDim.y + threadIdx.y;
    if (v >= p.nV) return;   // a warp is one detector row: uniform
    const bool in_u = u0 < p.nU;
    const int u = in_u ? u0 : p.nU - 1;
    const FrameInterp& F = p.frames[p.a0 + la];
    double s[3], vec[3];
    const double length = interp_setup(p, F, u, v, s, vec);
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
    const bool live = in_u && !empty && lo <= hi;
    // The lanes of a warp walk one global sample index i from the warp's smallest first
    // sample: at each step their samples sit at the same fraction of neighbouring rays, so
    // the warp's gathers stay compact.  A lane's samples before its own first one lie outside
    // the volume (beyond the first-sample cap of the view they are not taken at all, and lo
    // is never below it), clamp to the zero pads and add nothing.
    const int i0 = __reduce_min_sync(0xffffffffu, live ? (int)lo : INT_MAX);
    if (!in_u) return;
    const size_t oidx = ((size_t)la * p.nV + v) * (size_t)p.nU + u;
    if (!live) {
        ((TP*)p.proj)[oidx] = from_f32<TP>(0.f);
        return;
    }
    const int first = NEAREST ? (int)lo : i0;
    const int nsamp = (int)hi - first + 1;
    // padded coordinates (+1) of the first sample
    const float q0x = (float)(fma(vec[0], (double)first, s[0]) + 1.0);
    const float q0y = (float)(fma(vec[1], (double)first, s[1]) + 1.0);
    const float q0z = (float)(fma(vec[2], (double)first, s[2]) + 1.0);
    const float vx = (float)vec[0], vy = (float)vec[1], vz = (float)vec[2];
    const float mx = (float)(p.nX + 1), my = (float)(p.nY + 1), mz = (float)(p.nZ + 1);
    const int XP = p.nX + 3, YP = p.nY + 3;
    const int layout = F.layout;
    const TV* vol = (const TV*)(layout ? p.vol_y : p.vol_x);
    const int sx = layout ? YP : 1;
    const int sy = layout ? 1 : XP;
    const int sz = XP * YP;
    float sum = 0.f;
    if (NEAREST) {
#pragma unroll 2
        for (int k = 0; k < nsamp; ++k) {
            const float kf = (float)k;
            const float qx = fminf(fmaxf(fmaf(kf, vx, q0x), 0.f), mx);
            const float qy = fminf(fmaxf(fmaf(kf, vy, q0y), 0.f), my);
            const float qz = fminf(fmaxf(fmaf(kf, vz, q0z), 0.f), mz);
            const int ix = (int)(qx + 0.5f), iy = (int)(qy + 0.5f), iz = (int)(qz + 0.5f);
            sum += ldg_f<TV>(vol + ix * sx + iy * sy + iz * sz);
        }
    } else {
        // Trilinear from corner quads: with f the fast axis of this view's layout and o the
        // other one, a sample is two vector loads (rows o and o+1).  Two samples per step in
        // packed FP32x2.  Floors by a round-toward-zero add of 1.5*2^23 (the clamped
        // coordinates are >= 0); the float bits then index the quads directly:
        // index = bf + bo*FP + bz*FP*OP - 0x4B400000*(1 + FP + FP*OP) (32-bit wrap).
        constexpr float M = 12582912.0f;
        const float q0f = layout ? q0y : q0x, q0o = layout ? q0x : q0y;
        const float vf = layout ? vy : vx, vo = layout ? vx : vy;
        const float mf = layout ? my : mx, mo = layout ? mx : my;
        const uint32_t FP = (uint32_t)(layout ? YP : XP), OP = (uint32_t)(layout ? XP : YP);
        const uint32_t PL = FP * OP;
        const uint32_t bias = 0u - 0x4B400000u * (1u + FP + PL);
        const void* quads = layout ? p.quad_y : p.quad_x;
        const float2 vf2 = pk2(vf), vo2 = pk2(vo), vz2 = pk2(vz);
        const float2 q0f2 = pk2(q0f), q0o2 = pk2(q0o), q0z2 = pk2(q0z);
        float2 kk = pk2(0.f, 1.f);
        float sa = 0.f, sb = 0.f;
        // Consecutive samples are a fraction of a voxel apart and often share their trilinear
        // cell: the corner quads of the previous sample are kept and reloaded only when the
        // cell index changes (a lane that skips a load adds no L1 traffic).
        uint32_t pidx = 0xffffffffu;
        float4 p0 = make_float4(0.f, 0.f, 0.f, 0.f), p1 = p0;
        int k = 0;
#pragma unroll 1
        for (; k + 1 < nsamp; k += 2) {
            float2 qf = __ffma2_rn(kk, vf2, q0f2), qo = __ffma2_rn(kk, vo2, q0o2), qz = __ffma2_rn(kk, vz2, q0z2);
            kk = __fadd2_rn(kk, pk2(2.f));
            qf.x = fminf(fmaxf(qf.x, 0.f), mf); qf.y = fminf(fmaxf(qf.y, 0.f), mf);
            qo.x = fminf(fmaxf(qo.x, 0.f), mo); qo.y = fminf(fmaxf(qo.y, 0.f), mo);
            qz.x = fminf(fmaxf(qz.x, 0.f), mz); qz.y = fminf(fmaxf(qz.y, 0.f), mz);
            const float2 tf = __fadd2_rz(qf, pk2(M)), to = __fadd2_rz(qo, pk2(M)), tz = __fadd2_rz(qz, pk2(M));
            const float2 ff = __ffma2_rn(__fadd2_rn(tf, pk2(-M)), pk2(-1.f), qf);
            const float2 fo = __ffma2_rn(__fadd2_rn(to, pk2(-M)), pk2(-1.f), qo);
            const float2 fz = __ffma2_rn(__fadd2_rn(tz, pk2(-M)), pk2(-1.f), qz);
            const uint32_t ia = __float_as_uint(tf.x) + __float_as_uint(to.x) * FP + __float_as_uint(tz.x) * PL + bias;
            const uint32_t ib = __float_as_uint(tf.y) + __float_as_uint(to.y) * FP + __float_as_uint(tz.y) * PL + bias;
            if (ia != pidx) {
                p0 = ldq<TV>(quads, ia);
                p1 = ldq<TV>(quads, ia + FP);
            }
            sa += tri<TV>(p0, p1, ff.x, fz.x, fo.x);
            if (ib != ia) {
                p0 = ldq<TV>(quads, ib);
                p1 = ldq<TV>(quads, ib + FP);
            }
            sb += tri<TV>(p0, p1, ff.y, fz.y, fo.y);
            pidx = ib;
        }
        sum = sa + sb;
        if (k < nsamp) {   // odd count: last sample
            const float kf = (float)k;
            const float qf = fminf(fmaxf(fmaf(kf, vf, q0f), 0.f), mf);
            const float qo = fminf(fmaxf(fmaf(kf, vo, q0o), 0.f), mo);
            const float qz = fminf(fmaxf(fmaf(kf, vz, q0z), 0.f), mz);
            const float tf = __fadd_rz(qf, M), to = __fadd_rz(qo, M), tz = __fadd_rz(qz, M);
            const uint32_t i = __float_as_uint(tf) + __float_as_uint(to) * FP + __float_as_uint(tz) * PL + bias;
            sum += tri<TV>(ldq<TV>(quads, i), ldq<TV>(quads, i + FP), qf - (tf - M), qz - (tz - M), qo - (to - M));
        }
    }
    const double dl = sqrt(vec[0] * p.dVX * vec[0] * p.dVX + vec[1] * p.dVY * vec[1] * p.dVY +
                           vec[2] * p.dVZ * vec[2] * p.dVZ);
    ((TP*)p.proj)[oidx] = from_f32<TP>(sum * (float)dl);
}

// Hardware-texture variant (TIGRE_OPT_INTERP_TEXTURE): the same samples, each one tex3D fetch
// with the texture unit's linear filter from an FP32 3-D array, border 0, texel centres at +0.5
// -- the reference's own sampling (ray_interpolated_projection.cu:193-199, texture set up at
// :549-603).  The filter weights are the texture unit's 8-bit fractions, so results differ
// from the exact trilinear kernel by up to ~2^-9 relative per sample.
template <typename TP>
__global__ void __launch_bounds__(256) interp_tex_kernel(InterpArgs p, cudaTextureObject_t tex) {
    const int u0 = blockIdx.x * 32 + threadIdx.x;
    const int la = blockIdx.y;
    const int v = blockIdx.z * blockDim.y + threadIdx.y;
    if (v >= p.nV || u0 >= p.nU) return;
    const int u = u0;
    const FrameInterp& F = p.frames[p.a0 + la];
    double s[3], vec[3];
    const double length = interp_setup(p, F, u, v, s, vec);
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
    const int first = (int)lo;
    const int nsamp = (int)hi - first + 1;
    // texture coordinates of the first sample (texel i spans [i, i+1), centre i + 0.5)
    const float qx = (float)(fma(vec[0], (double)first, s[0]) + 0.5);
    const float qy = (float)(fma(vec[1], (double)first, s[1]) + 0.5);
    const float qz = (float)(fma(vec[2], (double)first, s[2]) + 0.5);
    const float vx = (float)vec[0], vy = (float)vec[1], vz = (float)vec[2];
    float sa = 0.f, sb = 0.f;
    int k = 0;
#pragma unroll 2
    for (; k + 1 < nsamp; k += 2) {
        const float ka = (float)k, kb = (float)(k + 1);
        sa += tex3D<float>(tex, fmaf(ka, vx, qx), fmaf(ka, vy, qy), fmaf(ka, vz, qz));
        sb += tex3D<float>(tex, fmaf(kb, vx, qx), fmaf(kb, vy, qy), fmaf(kb, vz, qz));
    }
    if (k < nsamp) {
        const float ka = (float)k;
        sa += tex3D<float>(tex, fmaf(ka, vx, qx), fmaf(ka, vy, qy), fmaf(ka, vz, qz));
    }
    const double dl = sqrt(vec[0] * p.dVX * vec[0] * p.dVX + vec[1] * p.dVY * vec[1] * p.dVY +
                           vec[2] * p.dVZ * vec[2] * p.dVZ);
    ((TP*)p.proj)[oidx] = from_f32<TP>((sa + sb) * (float)dl);
}

template <typename TV, typename TP>
void launch_typed(const InterpArgs& a, bool nearest, dim3 grid, dim3 block, cudaStream_t st) {
    if (nearest) interp_kernel<TV, TP, true><<<grid, block, 0, st>>>(a);
    else interp_kernel<TV, TP, false><<<grid, block, 0, st>>>(a);
}

}  // namespace

int launch_interp_count(TigrePlan* P, int a0, int a1, unsigned long long* d_total, cudaStream_t st) {
    InterpArgs a{};
    a.frames = P->d_interp;
    a.nX = P->d.nX; a.nY = P->d.nY; a.nZ = P->d.nZ; a.nU = P->d.nU; a.nV = P->d.nV;
    a.dVX = P->d.dVX; a.dVY = P->d.dVY; a.dVZ = P->d.dVZ; a.acc = P->d.accuracy;
    a.parallel = P->parallel ? 1 : 0;
    const int rows = 8;
    dim3 block(32, rows);
    dim3 grid((P->d.nU + 31) / 32, 1, (P->d.nV + rows - 1) / rows);
    TIGRE_CUDA(cudaMemsetAsync(d_total, 0, sizeof(unsigned long long), st));
    for (int c = 0; c < a1 - a0; c += 65535) {
        InterpArgs ac = a;
        ac.a0 = a0 + c;
        grid.y = std::min(65535, a1 - a0 - c);
        interp_count_kernel<<<grid, block, 0, st>>>(ac, d_total);
        TIGRE_LAUNCHED();
    }
    return TIGRE_SUCCESS;
}

int launch_interp(TigrePlan* P, const void* vol_x, const void* vol_y, const void* quad_x, const void* quad_y, int vdt,
                  void* proj, int pdt, int a0, int a1, cudaStream_t st) {
    InterpArgs a{};
    a.vol_x = vol_x; a.vol_y = vol_y; a.quad_x = quad_x; a.quad_y = quad_y; a.frames = P->d_interp;
    a.nX = P->d.nX; a.nY = P->d.nY; a.nZ = P->d.nZ; a.nU = P->d.nU; a.nV = P->d.nV;
    a.dVX = P->d.dVX; a.dVY = P->d.dVY; a.dVZ = P->d.dVZ; a.acc = P->d.accuracy;
    a.parallel = P->parallel ? 1 : 0;
    const bool nearest = P->d.accuracy > 1.0;
    const int rows = 8;
    dim3 block(32, rows);
    dim3 grid((P->d.nU + 31) / 32, 1, (P->d.nV + rows - 1) / rows);
    const int na = a1 - a0;
    for (int c = 0; c < na; c += 65535) {
        InterpArgs ac = a;
        ac.a0 = a0 + c;
        ac.proj = (char*)proj + (size_t)c * P->d.nU * P->d.nV * dtype_size(pdt);
        grid.y = std::min(65535, na - c);
        if (vdt == TIGRE_F32 && pdt == TIGRE_F32) launch_typed<float, float>(ac, nearest, grid, block, st);
        else if (vdt == TIGRE_BF16 && pdt == TIGRE_BF16)
            launch_typed<__nv_bfloat16, __nv_bfloat16>(ac, nearest, grid, block, st);
        else if (vdt == TIGRE_F16 && pdt == TIGRE_F16) launch_typed<__half, __half>(ac, nearest, grid, block, st);
        else if (vdt == TIGRE_BF16 && pdt == TIGRE_F32) launch_typed<__nv_bfloat16, float>(ac, nearest, grid, block, st);
        else if (vdt == TIGRE_F16 && pdt == TIGRE_F32) launch_typed<__half, float>(ac, nearest, grid, block, st);
        else if (vdt == TIGRE_F32 && pdt == TIGRE_BF16) launch_typed<float, __nv_bfloat16>(ac, nearest, grid, block, st);
        else if (vdt == TIGRE_F32 && pdt == TIGRE_F16) launch_typed<float, __half>(ac, nearest, grid, block, st);
        else return fail(TIGRE_ERR_BAD_ASSERT, "unsupported dtype pair for interpolated projection");
        TIGRE_LAUNCHED();
    }
    return TIGRE_SUCCESS;
}

}  // namespace tigre

namespace tigre {

// The plan's FP32 3-D array and linear-filter texture object, sized to the volume (made once
// per plan, reused by every call), filled from d_vol (FP32, (nZ, nY, nX)) on stream st.
int interp_texture(TigrePlan* P, const float* d_vol, cudaStream_t st, unsigned long long* tex_out) {
    const Dims& d = P->d;
    if (!P->tex_array) {
        cudaChannelFormatDesc ch = cudaCreateChannelDesc<float>();
        TIGRE_CUDA(cudaMalloc3DArray(&P->tex_array, &ch, make_cudaExtent(d.nX, d.nY, d.nZ)));
        cudaResourceDesc rd{};
        rd.resType = cudaResourceTypeArray;
        rd.res.array.array = P->tex_array;
        cudaTextureDesc td{};
        td.addressMode[0] = td.addressMode[1] = td.addressMode[2] = cudaAddressModeBorder;
        td.filterMode = cudaFilterModeLinear;
        td.readMode = cudaReadModeElementType;
        td.normalizedCoords = 0;
        cudaTextureObject_t t = 0;
        TIGRE_CUDA(cudaCreateTextureObject(&t, &rd, &td, nullptr));
        P->tex_obj = t;
    }
    cudaMemcpy3DParms cp{};
    cp.srcPtr = make_cudaPitchedPtr(const_cast<float*>(d_vol), (size_t)d.nX * sizeof(float), d.nX, d.nY);
    cp.dstArray = P->tex_array;
    cp.extent = make_cudaExtent(d.nX, d.nY, d.nZ);
    cp.kind = cudaMemcpyDeviceToDevice;
    TIGRE_CUDA(cudaMemcpy3DAsync(&cp, st));
    *tex_out = (unsigned long long)P->tex_obj;
    return TIGRE_SUCCESS;
}

int launch_interp_tex(TigrePlan* P, unsigned long long tex, void* proj, int pdt, int a0, int a1, cudaStream_t st) {
    InterpArgs a{};
    a.frames = P->d_interp;
    a.nX = P->d.nX; a.nY = P->d.nY; a.nZ = P->d.nZ; a.nU = P->d.nU; a.nV = P->d.nV;
    a.dVX = P->d.dVX; a.dVY = P->d.dVY; a.dVZ = P->d.dVZ; a.acc = P->d.accuracy;
    a.parallel = P->parallel ? 1 : 0;
    const int rows = 8;
    dim3 block(32, rows);
    dim3 grid((P->d.nU + 31) / 32, 1, (P->d.nV + rows - 1) / rows);
    const int na = a1 - a0;
    for (int c = 0; c < na; c += 65535) {
        InterpArgs ac = a;
        ac.a0 = a0 + c;
        ac.proj = (char*)proj + (size_t)c * P->d.nU * P->d.nV * dtype_size(pdt);
        grid.y = std::min(65535, na - c);
        if (pdt == TIGRE_F32) interp_tex_kernel<float><<<grid, block, 0, st>>>(ac, (cudaTextureObject_t)tex);
        else if (pdt == TIGRE_BF16) interp_tex_kernel<__nv_bfloat16><<<grid, block, 0, st>>>(ac, (cudaTextureObject_t)tex);
        else interp_tex_kernel<__half><<<grid, block, 0, st>>>(ac, (cudaTextureObject_t)tex);
        TIGRE_LAUNCHED();
    }
    return TIGRE_SUCCESS;
}

}  // namespace tigre
