// POCS total-variation descent, sm_100a.
//
// One step of pocs_tv (Common/CUDA/GD_TV.cu:440-597) is
//     g = grad TV(f)                                  (gradientTV, :117-143)
//     f <- f - alpha * g / sqrt(sum(g^2) + 1e-7)      (:556-597)
// The reference runs gradientTV, a device copy, two reduction kernels, a host
// synchronisation and three element-wise kernels per step (~48 B/voxel).
// Here a step is two passes and no host round trip (~12 B/voxel):
//   pass 1  tv_tiled_kernel<kTvOutNorm>    stencil -> g, sum g^2 (FP64, one atomic per block)
//   pass 2  tv_tiled_kernel<kTvOutUpdate>  stencil again -> g, writes f - alpha g / |g|,
//                             reading |g|^2 from device memory (ping-pong buffers)
// g is recomputed rather than stored: the stencil is cheap, the bytes are not.
//
// Boundary rule of the single-device reference call: the image sits between
// zero slices in z (its zeroed halo buffer, GD_TV.cu:380-393 and 447-461);
// along x and y a difference whose neighbour is outside is 0 (gradient(), :91-115),
// and the terms of neighbours beyond the last x / y index vanish.

#include <cmath>
#include <cstdlib>
#include <mutex>
#include <string>
#include <type_traits>

#include "tigre_internal.h"

namespace tigre {
namespace {

struct TVDims {
    int nx, ny, nz;
};

// Voxels (x, y, z < nzr) of the per-voxel kernels: blocks stride over (y, z) rows, threads over
// x, so no thread divides a linear index; i is the linear index of (x, y, z).
#define TV_FOR_EACH_VOXEL(d, nzr, x, y, z, i)                                                     \
    for (long row_ = blockIdx.x; row_ < (long)(d).ny * (nzr); row_ += gridDim.x) {               \
        const int y = (int)(row_ % (d).ny), z = (int)(row_ / (d).ny);                             \
        for (int x = threadIdx.x; x < (d).nx; x += blockDim.x) {                                   \
            const size_t i = ((size_t)z * (d).ny + y) * (d).nx + x;
#define TV_END_FOR_EACH_VOXEL \
    }                         \
    }

int grid_rows(const TVDims& d, int nzr) { return (int)std::min<long>((long)d.ny * nzr, 148 * 16); }

__device__ __forceinline__ float fget(const float* __restrict__ f, const TVDims& d, int x, int y, int z) {
    return (z >= 0 && z < d.nz) ? __ldg(f + ((size_t)z * d.ny + y) * d.nx + x) : 0.f;
}

__device__ __forceinline__ double block_sum(double v) {
    __shared__ double red[32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) red[wid] = v;
    __syncthreads();
    v = 0.0;
    if (wid == 0) {
        const int nw = (blockDim.x + 31) >> 5;
        v = lane < nw ? red[lane] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    }
    return v;
}

// ---- tiled gradientTV: the POCS passes and the autograd gradient ----
//
// A block owns a 32 x 8 tile of (x, y) columns and marches down a chunk of kTvZC slices.
// Per slice it stages f with a one-voxel x/y halo in shared memory and computes, at every
// tile point and at the tile's +x column and +y row, the backward differences (dz, dy, dx)
// and r = 1 / (sqrt(dz^2 + dy^2 + dx^2) + 1e-8) of gradientTV (GD_TV.cu:117-143).  The
// gradient at (x, y, z) (dftv, GD_TV.cu:135-140) is then
//     (dz + dy + dx) r  -  dx(x+1) r(x+1)  -  dy(y+1) r(y+1)  -  dz(z+1) r(z+1),
// with each norm evaluated once instead of four times and each voxel read from global memory
// once per slice (plus the halo), with no integer division per voxel.  The differences are
// the reference's exactly; r uses the hardware reciprocal square root and reciprocal, so each
// term carries a relative error of a few 1e-7 against the reference's IEEE divisions.
// Zero-filled staging reproduces the boundary rule: the zero slices below z = 0 and above
// z = nz - 1, and zero differences across the -x / -y faces.
//
// Pipeline: staged slices live in a ring of three buffers and the (dy, dx, r) planes in two,
// so one barrier per slice suffices; each thread fetches its staged elements three slices
// ahead into registers, so global loads overlap the arithmetic of the slices before them.
constexpr int kTvTX = 32, kTvZC = 32;   // tile width; slices per chunk (tile height: 8 rows per thread row)
constexpr int kTvFX = kTvTX + 2;         // staged f: x0-1 .. x0+32 (and y0-1 .. y0+TY)
constexpr int kTvQX = kTvTX + 1;         // difference points: x0 .. x0+32 (and y0 .. y0+TY)
constexpr int kTvOutNorm = 0, kTvOutUpdate = 1, kTvOutGrad = 2;

struct TvTiles {
    int tx, ty, tz, ntiles;
};

TvTiles tv_tiles(const TVDims& d, int rows) {
    const int TY = 8 * rows;
    TvTiles t{(d.nx + kTvTX - 1) / kTvTX, (d.ny + TY - 1) / TY, (d.nz + kTvZC - 1) / kTvZC, 0};
    t.ntiles = t.tx * t.ty * t.tz;
    return t;
}

int tv_tiled_grid(const TvTiles& t) { return std::min(t.ntiles, 148 * 8); }

// rows of the tile each thread owns (1: 32 x 8 tiles, 2: 32 x 16); TIGRE_B200_TV_ROWS overrides
int tv_rows() {
    const char* e = std::getenv("TIGRE_B200_TV_ROWS");
    return (e && std::atoi(e) == 1) ? 1 : (e && std::atoi(e) == 2) ? 2 : 2;
}

// 1 / (sqrt(s) + eps) for s >= 0
__device__ __forceinline__ float tv_rnorm(float s) {
    const float q = s > 0.f ? s * rsqrtf(s) : 0.f;
    return __fdividef(1.f, q + 1e-8f);
}

// OUT: kTvOutNorm adds sum g^2 (FP64, one atomic per block) into *sums; kTvOutUpdate writes
// o = f - alpha g / sqrt(*sums + 1e-7) (GD_TV.cu:556-597); kTvOutGrad writes o = g.
// ROWS: tile rows per thread; the tile is 32 x (8 ROWS) columns.
template <int OUT, int ROWS>
__global__ void __launch_bounds__(256, ROWS == 1 ? 4 : 3) tv_tiled_kernel(const float* __restrict__ f, float* __restrict__ o, TVDims d,
                                                       TvTiles T, double* __restrict__ sums, float alpha) {
    constexpr int TY = 8 * ROWS, FY = TY + 2, QY = TY + 1;
    constexpr int FS = FY * kTvFX;            // one staged slice
    constexpr int NS = (FS + 255) / 256;      // staged elements per thread and slice
    __shared__ float F[3 * FS];
    // dy, dx and r of a staged slice (dz is needed only at a thread's own columns: registers)
    __shared__ float Qy[2][QY][kTvQX], Qx[2][QY][kTvQX], Qr[2][QY][kTvQX];
    const int tid = threadIdx.x, lx = tid & 31, ly = tid >> 5;
    float scale = 0.f;
    if (OUT == kTvOutUpdate) scale = (float)((double)alpha / sqrt(*sums + 1e-7));
    const int plane = d.nx * d.ny;   // the host keeps nx * ny * nz below 2^31
    // the +x column (qx = 32, qy = 0..TY) and the +y row (qy = TY) of difference points
    const bool extra = tid < QY + kTvTX;
    const int eqx = tid < QY ? kTvTX : tid - QY, eqy = tid < QY ? tid : TY;
    double acc = 0.0;
    for (int t = blockIdx.x; t < T.ntiles; t += gridDim.x) {
        const int bx = t % T.tx, rt = t / T.tx;
        const int by = rt % T.ty, bz = rt / T.ty;
        const int x0 = bx * kTvTX, y0 = by * TY, z0 = bz * kTvZC;
        const int zend = min(z0 + kTvZC, d.nz);   // output slices z0 .. zend-1; slice zend supplies dz(z+1)
        // thread tid stages elements k = tid + 256 j (k < FS) of every slice; their in-slice
        // offsets are fixed per tile (-1 outside the volume: zero)
        int off[NS];
#pragma unroll
        for (int j = 0; j < NS; ++j) {
            const int k = tid + 256 * j;
            const int fy = k / kTvFX, fx = k - fy * kTvFX;
            const int xx = x0 - 1 + fx, yy = y0 - 1 + fy;
            off[j] = (k < FS && xx >= 0 && xx < d.nx && yy >= 0 && yy < d.ny) ? yy * d.nx + xx : -1;
        }
        auto fetch = [&](int zz, float (&v)[NS]) {
            const bool zin = zz >= 0 && zz < d.nz;
#pragma unroll
            for (int j = 0; j < NS; ++j) v[j] = (zin && off[j] >= 0) ? __ldg(f + (zz * plane + off[j])) : 0.f;
        };
        auto put = [&](int slot, const float (&v)[NS]) {
#pragma unroll
            for (int j = 0; j < NS; ++j)
                if (j + 1 < NS || tid + 256 * j < FS) F[slot * FS + tid + 256 * j] = v[j];
        };
        // differences and reciprocal norm at point (qx, qy) of slice slot sc over slice slot sp
        auto qpoint = [&](int qx, int qy, int sc, int sp, float& dz, float& dy, float& dx) {
            const int k = (qy + 1) * kTvFX + qx + 1;
            const float c = F[sc * FS + k];
            dz = c - F[sp * FS + k];
            dy = y0 + qy > 0 ? c - F[sc * FS + k - kTvFX] : 0.f;
            dx = x0 + qx > 0 ? c - F[sc * FS + k - 1] : 0.f;
            return tv_rnorm(dz * dz + dy * dy + dx * dx);
        };
        const int x = x0 + lx;
        bool inside[ROWS];
        int own[ROWS];
#pragma unroll
        for (int q = 0; q < ROWS; ++q) {
            const int y = y0 + ly + 8 * q;
            inside[q] = x < d.nx && y < d.ny;
            own[q] = y * d.nx + x;
        }
        // R[j]: registers holding a fetched slice; at relative step j the slice zz + 1 is in
        // R[(j + 1) % 3] and slice zz + 3 is fetched into R[j % 3]
        float R[3][NS];
        fetch(z0 - 1, R[0]);
        put(0, R[0]);
        fetch(z0, R[0]);
        put(1, R[0]);
        fetch(z0 + 1, R[1]);
        fetch(z0 + 2, R[2]);
        __syncthreads();
        float part[ROWS], fown[ROWS];
#pragma unroll
        for (int q = 0; q < ROWS; ++q) part[q] = fown[q] = 0.f;
        // one slice: slots (SP, SC, SN) hold slices zz - 1, zz, zz + 1; QB is the difference buffer
        auto step = [&](int zz, auto SPc, auto SCc, auto SNc, auto QBc, auto RPc) {
            constexpr int SP = decltype(SPc)::value, SC = decltype(SCc)::value, SN = decltype(SNc)::value;
            constexpr int QB = decltype(QBc)::value, RP = decltype(RPc)::value;
            if (zz + 1 <= zend) put(SN, R[RP]);
            if (zz + 3 <= zend) fetch(zz + 3, R[(RP + 2) % 3]);
            float dz[ROWS], r[ROWS], dy[ROWS], dx[ROWS];
#pragma unroll
            for (int q = 0; q < ROWS; ++q) {
                const int qy = ly + 8 * q;
                r[q] = qpoint(lx, qy, SC, SP, dz[q], dy[q], dx[q]);
                Qy[QB][qy][lx] = dy[q]; Qx[QB][qy][lx] = dx[q]; Qr[QB][qy][lx] = r[q];
            }
            if (extra) {
                float a, b, c;
                const float m = qpoint(eqx, eqy, SC, SP, a, b, c);
                Qy[QB][eqy][eqx] = b; Qx[QB][eqy][eqx] = c; Qr[QB][eqy][eqx] = m;
            }
            __syncthreads();
#pragma unroll
            for (int q = 0; q < ROWS; ++q) {
                const int qy = ly + 8 * q;
                if (zz > z0 && inside[q]) {   // slice zz-1 is complete with its +z neighbour's term
                    const float g = part[q] - dz[q] * r[q];
                    if (OUT == kTvOutNorm) acc += (double)g * (double)g;
                    else {
                        const int i = (zz - 1) * plane + own[q];
                        o[i] = OUT == kTvOutUpdate ? fmaf(-scale, g, fown[q]) : g;
                    }
                }
                if (zz < zend && inside[q]) {
                    float g = (dz[q] + dy[q] + dx[q]) * r[q];
                    if (x + 1 < d.nx) g -= Qx[QB][qy][lx + 1] * Qr[QB][qy][lx + 1];
                    if (y0 + qy + 1 < d.ny) g -= Qy[QB][qy + 1][lx] * Qr[QB][qy + 1][lx];
                    part[q] = g;
                    fown[q] = F[SC * FS + (qy + 1) * kTvFX + lx + 1];
                }
            }
        };
        using I0 = std::integral_constant<int, 0>;
        using I1 = std::integral_constant<int, 1>;
        using I2 = std::integral_constant<int, 2>;
        // six relative steps bring the three slots, two buffers and three register sets back to
        // their starting assignment
        for (int zb = z0; zb <= zend; zb += 6) {
            step(zb, I0{}, I1{}, I2{}, I0{}, I1{});
            if (zb + 1 > zend) break;
            step(zb + 1, I1{}, I2{}, I0{}, I1{}, I2{});
            if (zb + 2 > zend) break;
            step(zb + 2, I2{}, I0{}, I1{}, I0{}, I0{});
            if (zb + 3 > zend) break;
            step(zb + 3, I0{}, I1{}, I2{}, I1{}, I1{});
            if (zb + 4 > zend) break;
            step(zb + 4, I1{}, I2{}, I0{}, I0{}, I2{});
            if (zb + 5 > zend) break;
            step(zb + 5, I2{}, I0{}, I1{}, I1{}, I0{});
        }
        __syncthreads();   // the next tile restages the ring
    }
    if (OUT == kTvOutNorm) {
        acc = block_sum(acc);
        if (threadIdx.x == 0) atomicAdd(sums, acc);
    }
}

// launch one tiled pass with the tile shape of tv_rows()
template <int OUT>
void launch_tv_tiled(const float* f, float* o, const TVDims& d, double* sums, float alpha, cudaStream_t st) {
    const int rows = tv_rows();
    const TvTiles T = tv_tiles(d, rows);
    if (rows == 2) tv_tiled_kernel<OUT, 2><<<tv_tiled_grid(T), 256, 0, st>>>(f, o, d, T, sums, alpha);
    else tv_tiled_kernel<OUT, 1><<<tv_tiled_grid(T), 256, 0, st>>>(f, o, d, T, sums, alpha);
}

// sum_i |grad f_i| over the voxels and the zero halo slice above the last one
// (whose gradient norm is |f(x,y,nz-1)|); its derivative is the gradient of tv_tiled_kernel.
__global__ void __launch_bounds__(256) tv_value_kernel(const float* __restrict__ f, TVDims d, double* __restrict__ out) {
    double s = 0.0;
    TV_FOR_EACH_VOXEL(d, d.nz + 1, x, y, z, i) {
        (void)i;
        if (z == d.nz) {
            s += fabs((double)fget(f, d, x, y, z - 1));
            continue;
        }
        const float c = fget(f, d, x, y, z);
        const float d0 = c - fget(f, d, x, y, z - 1);
        const float d1 = y > 0 ? c - fget(f, d, x, y - 1, z) : 0.f;
        const float d2 = x > 0 ? c - fget(f, d, x - 1, y, z) : 0.f;
        s += sqrt((double)d0 * d0 + (double)d1 * d1 + (double)d2 * d2);
    }
    TV_END_FOR_EACH_VOXEL
    s = block_sum(s);
    if (threadIdx.x == 0) atomicAdd(out, s);
}

// ---- adaptive-weighted TV (aw_pocs_tv) and PICCS (piccs_tv) ----
//
// Both reuse the backward-difference stencil of gradientTV with two changes:
// * AwTV (GD_AwTV.cu:117-158): every difference component d_c carries the weight
//   w_c = exp(-(d_c / delta)^2), in the numerators and inside the norms;
// * PICCS (PICCS.cu:117-154, :274-380) runs on the bare image (no halo slices: a z
//   difference whose neighbour is outside is 0, like x and y) and descends along
//   (1 - ratio) grad TV(f) + ratio grad TV(f - prior), with 1e-6 (not 1e-8) added to each norm.
// A step is again two passes (norm, then update), with the gradient recomputed.

struct TVStep {
    const float* prior;   // PICCS prior image (same layout as f)
    float inv_delta;      // AwTV: 1 / delta
    float ratio;          // PICCS: weight of the prior term
    double norm_eps;      // added to sum(g^2) before the square root
    float grad_eps;       // added to every gradient norm: 1e-8 (GD_AwTV.cu:131), 1e-6 (PICCS.cu:149)
};

template <bool HALO, bool AW, typename Rd>
__device__ __forceinline__ float tv_stencil(const Rd& rd, const TVDims& d, int x, int y, int z, float idl, float eps) {
    auto val = [&](int xx, int yy, int zz) -> float { return (zz >= 0 && zz < d.nz) ? rd(xx, yy, zz) : 0.f; };
    auto wt = [&](float v) -> float {
        if (!AW) return 1.f;
        const float t = v * idl;
        return expf(-(t * t));
    };
    // |grad| with weights: sqrt(w0 a0^2 + w1 a1^2 + w2 a2^2) + eps
    auto nrm = [&](float a0, float a1, float a2, float w0, float w1, float w2) {
        return sqrtf(w0 * a0 * a0 + w1 * a1 * a1 + w2 * a2 * a2) + eps;
    };
    const bool zlow = HALO || z > 0;
    const float c = val(x, y, z);
    const float d0 = zlow ? c - val(x, y, z - 1) : 0.f;
    const float d1 = y > 0 ? c - val(x, y - 1, z) : 0.f;
    const float d2 = x > 0 ? c - val(x - 1, y, z) : 0.f;
    const float w0 = wt(d0), w1 = wt(d1), w2 = wt(d2);
    float g = (w0 * d0 + w1 * d1 + w2 * d2) / nrm(d0, d1, d2, w0, w1, w2);
    if (x + 1 < d.nx) {   // neighbour (x+1): its x difference involves f(x)
        const float n = val(x + 1, y, z);
        const float e0 = zlow ? n - val(x + 1, y, z - 1) : 0.f;
        const float e1 = y > 0 ? n - val(x + 1, y - 1, z) : 0.f;
        const float e2 = n - c;
        const float v2 = wt(e2);
        g -= v2 * e2 / nrm(e0, e1, e2, wt(e0), wt(e1), v2);
    }
    if (y + 1 < d.ny) {
        const float n = val(x, y + 1, z);
        const float e0 = zlow ? n - val(x, y + 1, z - 1) : 0.f;
        const float e1 = n - c;
        const float e2 = x > 0 ? n - val(x - 1, y + 1, z) : 0.f;
        const float v1 = wt(e1);
        g -= v1 * e1 / nrm(e0, e1, e2, wt(e0), v1, wt(e2));
    }
    if (HALO || z + 1 < d.nz) {   // neighbour (z+1); with the halo, above the last slice it is 0
        const float n = val(x, y, z + 1);
        const float e0 = n - c;
        const float e1 = y > 0 ? n - val(x, y - 1, z + 1) : 0.f;
        const float e2 = x > 0 ? n - val(x - 1, y, z + 1) : 0.f;
        const float v0 = wt(e0);
        g -= v0 * e0 / nrm(e0, e1, e2, v0, wt(e1), wt(e2));
    }
    return g;
}

constexpr int kTvAw = 1, kTvPiccs = 2;

template <int KIND>
__device__ __forceinline__ float tv_step_grad(const float* __restrict__ f, const TVDims& d, const TVStep& s, int x,
                                              int y, int z) {
    auto rf = [&](int xx, int yy, int zz) { return __ldg(f + ((size_t)zz * d.ny + yy) * d.nx + xx); };
    if (KIND == kTvAw) return tv_stencil<true, true>(rf, d, x, y, z, s.inv_delta, s.grad_eps);
    auto rdiff = [&](int xx, int yy, int zz) {
        const size_t i = ((size_t)zz * d.ny + yy) * d.nx + xx;
        return __ldg(f + i) - __ldg(s.prior + i);
    };
    const float ga = tv_stencil<false, false>(rf, d, x, y, z, 0.f, s.grad_eps);
    const float gb = tv_stencil<false, false>(rdiff, d, x, y, z, 0.f, s.grad_eps);
    return fmaf(1.f - s.ratio, ga, s.ratio * gb);
}

template <int KIND>
__global__ void __launch_bounds__(256) tv_step_norm_kernel(const float* __restrict__ f, TVDims d, TVStep st,
                                                           double* __restrict__ out) {
    double s = 0.0;
    TV_FOR_EACH_VOXEL(d, d.nz, x, y, z, i) {
        (void)i;
        const float g = tv_step_grad<KIND>(f, d, st, x, y, z);
        s += (double)g * (double)g;
    }
    TV_END_FOR_EACH_VOXEL
    s = block_sum(s);
    if (threadIdx.x == 0) atomicAdd(out, s);
}

template <int KIND>
__global__ void __launch_bounds__(256) tv_step_update_kernel(const float* __restrict__ f, float* __restrict__ o,
                                                             TVDims d, TVStep st, const double* __restrict__ sumsq,
                                                             float alpha) {
    const float scale = (float)((double)alpha / sqrt(*sumsq + st.norm_eps));
    TV_FOR_EACH_VOXEL(d, d.nz, x, y, z, i) {
        const float g = tv_step_grad<KIND>(f, d, st, x, y, z);
        o[i] = fmaf(-scale, g, __ldg(f + i));
    }
    TV_END_FOR_EACH_VOXEL
}

}  // namespace
}  // namespace tigre

using namespace tigre;

extern "C" {

int tigre_tv_gradient(const void* d_img, int dtype, float* d_grad, long nx, long ny, long nz, void* stream) {
    if (dtype != TIGRE_F32) return fail(TIGRE_ERR_BAD_ASSERT, "TV kernels take float32 volumes");
    if (nx <= 0 || ny <= 0 || nz <= 0 || !d_img || !d_grad) return fail(TIGRE_ERR_BAD_ASSERT, "bad TV arguments");
    TVDims d{(int)nx, (int)ny, (int)nz};
    launch_tv_tiled<kTvOutGrad>((const float*)d_img, d_grad, d, nullptr, 0.f, (cudaStream_t)stream);
    TIGRE_LAUNCHED();
    return TIGRE_SUCCESS;
}

int tigre_tv_value(const void* d_img, int dtype, long nx, long ny, long nz, double* d_out, void* stream) {
    if (dtype != TIGRE_F32) return fail(TIGRE_ERR_BAD_ASSERT, "TV kernels take float32 volumes");
    if (nx <= 0 || ny <= 0 || nz <= 0 || !d_img || !d_out) return fail(TIGRE_ERR_BAD_ASSERT, "bad TV arguments");
    TVDims d{(int)nx, (int)ny, (int)nz};
    tv_value_kernel<<<grid_rows(d, d.nz + 1), 256, 0, (cudaStream_t)stream>>>((const float*)d_img, d, d_out);
    TIGRE_LAUNCHED();
    return TIGRE_SUCCESS;
}

// In-place POCS-TV.  d_work: nx*ny*nz floats of caller scratch; 8 bytes of
// reduction scratch are taken from the stream-ordered allocator.
int tigre_tv_pocs(void* d_img, int dtype, long nx, long ny, long nz, float alpha, int max_iter, float* d_work,
                  void* stream) {
    if (dtype != TIGRE_F32) return fail(TIGRE_ERR_BAD_ASSERT, "TV kernels take float32 volumes");
    if (nx <= 0 || ny <= 0 || nz <= 0 || !d_img || !d_work || max_iter < 0)
        return fail(TIGRE_ERR_BAD_ASSERT, "bad TV arguments");
    if ((double)nx * ny * nz >= 2147483647.0) return fail(TIGRE_ERR_BAD_ASSERT, "volume too large");
    cudaStream_t st = (cudaStream_t)stream;
    TVDims d{(int)nx, (int)ny, (int)nz};
    const size_t n = (size_t)nx * ny * nz;
    double* sums = nullptr;
    TIGRE_CUDA(cudaMallocAsync(&sums, sizeof(double) * (size_t)std::max(max_iter, 1), st));
    TIGRE_CUDA(cudaMemsetAsync(sums, 0, sizeof(double) * (size_t)std::max(max_iter, 1), st));
    float* cur = (float*)d_img;
    float* nxt = d_work;
    for (int it = 0; it < max_iter; ++it) {
        launch_tv_tiled<kTvOutNorm>(cur, nullptr, d, sums + it, 0.f, st);
        launch_tv_tiled<kTvOutUpdate>(cur, nxt, d, sums + it, alpha, st);
        std::swap(cur, nxt);
    }
    if (cur != (float*)d_img) TIGRE_CUDA(cudaMemcpyAsync(d_img, cur, n * sizeof(float), cudaMemcpyDeviceToDevice, st));
    TIGRE_CUDA(cudaFreeAsync(sums, st));
    TIGRE_CUDA(cudaGetLastError());
    note_launches(2ull * (unsigned long long)max_iter);
    return TIGRE_SUCCESS;
}

}  // extern "C"

// Shared driver of the weighted / prior TV descents: ping-pong between d_img and d_work.
template <int KIND>
static int tv_descent(void* d_img, long nx, long ny, long nz, float alpha, int max_iter, const TVStep& stp,
                      float* d_work, cudaStream_t st) {
    TVDims d{(int)nx, (int)ny, (int)nz};
    const size_t n = (size_t)nx * ny * nz;
    double* sums = nullptr;
    TIGRE_CUDA(cudaMallocAsync(&sums, sizeof(double) * (size_t)std::max(max_iter, 1), st));
    TIGRE_CUDA(cudaMemsetAsync(sums, 0, sizeof(double) * (size_t)std::max(max_iter, 1), st));
    float* cur = (float*)d_img;
    float* nxt = d_work;
    for (int it = 0; it < max_iter; ++it) {
        tv_step_norm_kernel<KIND><<<grid_rows(d, d.nz), 256, 0, st>>>(cur, d, stp, sums + it);
        tv_step_update_kernel<KIND><<<grid_rows(d, d.nz), 256, 0, st>>>(cur, nxt, d, stp, sums + it, alpha);
        std::swap(cur, nxt);
    }
    if (cur != (float*)d_img) TIGRE_CUDA(cudaMemcpyAsync(d_img, cur, n * sizeof(float), cudaMemcpyDeviceToDevice, st));
    TIGRE_CUDA(cudaFreeAsync(sums, st));
    TIGRE_CUDA(cudaGetLastError());
    note_launches(2ull * (unsigned long long)max_iter);
    return TIGRE_SUCCESS;
}

extern "C" {

// In-place adaptive-weighted TV descent (aw_pocs_tv, GD_AwTV.cu:276-720): per step
//   g = grad AwTV(f);  f <- f - alpha g / sqrt(sum g^2 + 1e-7).
int tigre_tv_aw_pocs(void* d_img, int dtype, long nx, long ny, long nz, float alpha, int max_iter, float delta,
                    float* d_work, void* stream) {
    if (dtype != TIGRE_F32) return fail(TIGRE_ERR_BAD_ASSERT, "TV kernels take float32 volumes");
    if (nx <= 0 || ny <= 0 || nz <= 0 || !d_img || !d_work || max_iter < 0)
        return fail(TIGRE_ERR_BAD_ASSERT, "bad TV arguments");
    if ((double)nx * ny * nz >= 2147483647.0) return fail(TIGRE_ERR_BAD_ASSERT, "volume too large");
    if (!(delta != 0.f) || !std::isfinite(delta)) return fail(TIGRE_ERR_BAD_ASSERT, "AwTV: delta must be finite and nonzero");
    const TVStep stp{nullptr, 1.f / delta, 0.f, 1e-7, 1e-8f};
    return tv_descent<kTvAw>(d_img, nx, ny, nz, alpha, max_iter, stp, d_work, (cudaStream_t)stream);
}

// In-place PICCS TV descent (piccs_tv, PICCS.cu:274-380): per step
//   g = (1 - ratio) grad TV(f) + ratio grad TV(f - prior);  f <- f - alpha g / sqrt(sum g^2).
int tigre_tv_piccs(void* d_img, const void* d_prior, int dtype, long nx, long ny, long nz, float alpha, float ratio,
                   int max_iter, float* d_work, void* stream) {
    if (dtype != TIGRE_F32) return fail(TIGRE_ERR_BAD_ASSERT, "TV kernels take float32 volumes");
    if (nx <= 0 || ny <= 0 || nz <= 0 || !d_img || !d_prior || !d_work || max_iter < 0)
        return fail(TIGRE_ERR_BAD_ASSERT, "bad TV arguments");
    if ((double)nx * ny * nz >= 2147483647.0) return fail(TIGRE_ERR_BAD_ASSERT, "volume too large");
    const TVStep stp{(const float*)d_prior, 0.f, ratio, 0.0, 1e-6f};
    return tv_descent<kTvPiccs>(d_img, nx, ny, nz, alpha, max_iter, stp, d_work, (cudaStream_t)stream);
}

}  // extern "C"

// POCS-TV that allocates nothing.
//
// Who needs it: a caller whose process has handed all free device memory to another
// allocator (a framework's caching pool, a service run under a fixed memory cap) gets
// no memory from cudaMallocAsync, and a caller inside a fixed-latency loop must not
// enter the allocator at all, since allocation can block on locks or on the device.
// For those callers the only scratch of tigre_tv_pocs besides d_work -- one FP64 norm
// sum per iteration -- lives here in a fixed array of this module's device memory.
//
// Limits and sharing: the array holds kTvPocsStaticMaxIter sums, so max_iter above it
// is rejected.  Every call on a device uses the same array, and the first max_iter
// entries must be zero when a call's first kernel runs: each call clears them on its
// stream before use.  Calls that overlap in time on one device (other streams, other
// host threads) therefore race on the sums and must be serialised by the caller.
// The first call on each device looks up the array's address with that device
// current and caches it; make that first call before any stream capture.
constexpr int kTvPocsStaticMaxIter = 4096;   // 32 KiB
static __device__ __align__(256) double g_tv_pocs_sums[kTvPocsStaticMaxIter];

namespace {
constexpr int kMaxDevices = 256;
std::mutex g_tv_pocs_sums_mu;
double* g_tv_pocs_sums_addr[kMaxDevices] = {};

// Address of g_tv_pocs_sums on the current device (looked up once per device).
int tv_pocs_static_sums(double** out) {
    int dev = 0;
    TIGRE_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) return fail(TIGRE_ERR_BAD_ASSERT, "device index out of range");
    std::lock_guard<std::mutex> lk(g_tv_pocs_sums_mu);
    if (!g_tv_pocs_sums_addr[dev]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_tv_pocs_sums);
        if (e != cudaSuccess || !p) return cuda_fail(e, "cudaGetSymbolAddress(g_tv_pocs_sums)");
        g_tv_pocs_sums_addr[dev] = (double*)p;
    }
    *out = g_tv_pocs_sums_addr[dev];
    return TIGRE_SUCCESS;
}
}  // namespace

extern "C" int tigre_tv_pocs_noalloc(void* d_img, int dtype, long nx, long ny, long nz, float alpha, int max_iter,
                                     float* d_work, void* stream) {
    if (dtype != TIGRE_F32) return fail(TIGRE_ERR_BAD_ASSERT, "TV kernels take float32 volumes");
    if (nx <= 0 || ny <= 0 || nz <= 0 || !d_img || !d_work || max_iter < 0)
        return fail(TIGRE_ERR_BAD_ASSERT, "bad TV arguments");
    if ((double)nx * ny * nz >= 2147483647.0) return fail(TIGRE_ERR_BAD_ASSERT, "volume too large");
    if (max_iter > kTvPocsStaticMaxIter)
        return fail(TIGRE_ERR_BAD_ASSERT, "tigre_tv_pocs_noalloc: max_iter " + std::to_string(max_iter) +
                                              " exceeds its fixed scratch of " +
                                              std::to_string(kTvPocsStaticMaxIter) + " iterations");
    double* sums = nullptr;
    if (int rc = tv_pocs_static_sums(&sums)) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    TVDims d{(int)nx, (int)ny, (int)nz};
    const size_t n = (size_t)nx * ny * nz;
    if (max_iter > 0) TIGRE_CUDA(cudaMemsetAsync(sums, 0, sizeof(double) * (size_t)max_iter, st));
    float* cur = (float*)d_img;
    float* nxt = d_work;
    for (int it = 0; it < max_iter; ++it) {
        launch_tv_tiled<kTvOutNorm>(cur, nullptr, d, sums + it, 0.f, st);
        launch_tv_tiled<kTvOutUpdate>(cur, nxt, d, sums + it, alpha, st);
        std::swap(cur, nxt);
    }
    if (cur != (float*)d_img) TIGRE_CUDA(cudaMemcpyAsync(d_img, cur, n * sizeof(float), cudaMemcpyDeviceToDevice, st));
    TIGRE_CUDA(cudaGetLastError());
    note_launches(2ull * (unsigned long long)max_iter);
    return TIGRE_SUCCESS;
}
