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

struct TVStep {
    const float* prior;   // PICCS prior image (same layout as f)
    float inv_delta;      // AwTV: 1 / delta
    float ratio;          // PICCS: weight of the prior term
    double norm_eps;      // added to sum(g^2) before the square root
    float grad_eps;       // added to every gradient norm: 1e-8 (GD_AwTV.cu:131), 1e-6 (PICCS.cu:149)
};

constexpr int kTvPocs = 0, kTvAw = 1, kTvPiccs = 2;

// ---- tiled gradientTV: POCS-TV, AwTV and PICCS passes and the autograd gradient ----
//
// A block owns a 32 x (8 ROWS) tile of (x, y) columns and marches down a chunk of kTvZC
// slices.  Per slice it stages f with a one-voxel x/y halo in shared memory and computes, at
// every tile point and at the tile's +x column and +y row, the backward differences
// (dz, dy, dx), their weighted forms (nz, ny, nx) and r = 1 / (sqrt(nz dz + ny dy + nx dx) + eps)
// -- unweighted for POCS-TV (gradientTV, GD_TV.cu:117-143), with w = exp(-(d / delta)^2) per
// component for AwTV (GD_AwTV.cu:117-158).  The gradient at (x, y, z) (dftv, GD_TV.cu:135-140)
// is then
//     (nz + ny + nx) r  -  nx(x+1) r(x+1)  -  ny(y+1) r(y+1)  -  nz(z+1) r(z+1),
// each norm and weight evaluated once per voxel instead of four times, each voxel read from
// global memory once per slice (plus the halo), and no integer division per voxel.  The
// differences are the reference's exactly; r uses the hardware reciprocal square root and
// reciprocal, so each term carries a relative error of a few 1e-7 against the reference's
// IEEE divisions.  Zero-filled staging reproduces the boundary rules: the zero slices below
// z = 0 and above z = nz - 1 (POCS-TV, AwTV), zero differences across the -x / -y faces.
// PICCS (PICCS.cu:117-154) runs on the bare image (no z difference at z = 0, no +z term at the
// last slice, eps 1e-6) and stages two fields, f and f - prior, for
// g = (1 - ratio) grad TV(f) + ratio grad TV(f - prior).
//
// Pipeline: staged slices live in a ring of three buffers and the (ny, nx, r) planes in two,
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

// rows of the tile each thread owns (1: 32 x 8 tiles, 2: 32 x 16).  PICCS, with two staged
// fields, uses one row.
int tv_rows(int kind) { return kind == kTvPiccs ? 1 : 2; }

// 1 / (sqrt(s) + eps) for s >= 0
__device__ __forceinline__ float tv_rnorm(float s, float eps) {
    const float q = s > 0.f ? s * rsqrtf(s) : 0.f;
    return __fdividef(1.f, q + eps);
}

// OUT: kTvOutNorm adds sum g^2 (FP64, one atomic per block) into *sums; kTvOutUpdate writes
// o = f - alpha g / sqrt(*sums + st.norm_eps) (GD_TV.cu:556-597); kTvOutGrad writes o = g.
// ROWS: tile rows per thread.  KIND: kTvPocs, kTvAw or kTvPiccs.
template <int OUT, int ROWS, int KIND>
__global__ void __launch_bounds__(256, ROWS == 1 ? 4 : 3) tv_tiled_kernel(const float* __restrict__ f,
                                                                           float* __restrict__ o, TVDims d, TvTiles T,
                                                                           TVStep st, double* __restrict__ sums,
                                                                           float alpha) {
    constexpr bool HALO = KIND != kTvPiccs;
    constexpr int NF = KIND == kTvPiccs ? 2 : 1;   // staged fields: f (and f - prior)
    constexpr int TY = 8 * ROWS, FY = TY + 2, QY = TY + 1;
    constexpr int FS = FY * kTvFX;            // one staged slice of one field
    constexpr int NS = (FS + 255) / 256;      // staged elements per thread, slice and field
    __shared__ float F[NF * 3 * FS];
    // ny, nx and r of a staged slice (nz is needed only at a thread's own columns: registers)
    __shared__ float Qy[NF][2][QY][kTvQX], Qx[NF][2][QY][kTvQX], Qr[NF][2][QY][kTvQX];
    const int tid = threadIdx.x, lx = tid & 31, ly = tid >> 5;
    const float eps = st.grad_eps, idl = st.inv_delta;
    float scale = 0.f;
    if (OUT == kTvOutUpdate) scale = (float)((double)alpha / sqrt(*sums + st.norm_eps));
    const int plane = d.nx * d.ny;   // the host keeps nx * ny * nz below 2^31
    // the +x column (qx = 32, qy = 0..TY) and the +y row (qy = TY) of difference points
    const bool extra = tid < QY + kTvTX;
    const int eqx = tid < QY ? kTvTX : tid - QY, eqy = tid < QY ? tid : TY;
    double acc = 0.0;
    for (int t = blockIdx.x; t < T.ntiles; t += gridDim.x) {
        const int bx = t % T.tx, rt = t / T.tx;
        const int by = rt % T.ty, bz = rt / T.ty;
        const int x0 = bx * kTvTX, y0 = by * TY, z0 = bz * kTvZC;
        const int zend = min(z0 + kTvZC, d.nz);   // output slices z0 .. zend-1; slice zend supplies the +z term
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
        auto fetch = [&](int zz, float (&v)[NF][NS]) {
            const bool zin = zz >= 0 && zz < d.nz;
#pragma unroll
            for (int j = 0; j < NS; ++j) {
                const bool ok = zin && off[j] >= 0;
                const int i = zz * plane + off[j];
                v[0][j] = ok ? __ldg(f + i) : 0.f;
                if (NF == 2) v[NF - 1][j] = ok ? __ldg(f + i) - __ldg(st.prior + i) : 0.f;
            }
        };
        auto put = [&](int slot, const float (&v)[NF][NS]) {
#pragma unroll
            for (int c = 0; c < NF; ++c)
#pragma unroll
                for (int j = 0; j < NS; ++j)
                    if (j + 1 < NS || tid + 256 * j < FS) F[(c * 3 + slot) * FS + tid + 256 * j] = v[c][j];
        };
        // weighted differences and reciprocal norm at point (qx, qy) of field c, slice slot sc
        // over slot sp; zlow: the slice has a z difference (always with the zero halo slices)
        auto qpoint = [&](int c, int qx, int qy, int sc, int sp, bool zlow, float& wz, float& wy, float& wx) {
            const int k = (qy + 1) * kTvFX + qx + 1;
            const float* Fc = F + (c * 3 + sc) * FS;
            const float v = Fc[k];
            const float dz = zlow ? v - F[(c * 3 + sp) * FS + k] : 0.f;
            const float dy = y0 + qy > 0 ? v - Fc[k - kTvFX] : 0.f;
            const float dx = x0 + qx > 0 ? v - Fc[k - 1] : 0.f;
            if (KIND == kTvAw) {
                const float tz = dz * idl, ty = dy * idl, tx = dx * idl;
                wz = expf(-(tz * tz)) * dz;
                wy = expf(-(ty * ty)) * dy;
                wx = expf(-(tx * tx)) * dx;
            } else {
                wz = dz; wy = dy; wx = dx;
            }
            return tv_rnorm(wz * dz + wy * dy + wx * dx, eps);
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
        float R[3][NF][NS];
        fetch(z0 - 1, R[0]);
        put(0, R[0]);
        fetch(z0, R[0]);
        put(1, R[0]);
        fetch(z0 + 1, R[1]);
        fetch(z0 + 2, R[2]);
        __syncthreads();
        float part[NF][ROWS], fown[ROWS];
#pragma unroll
        for (int q = 0; q < ROWS; ++q) {
            fown[q] = 0.f;
#pragma unroll
            for (int c = 0; c < NF; ++c) part[c][q] = 0.f;
        }
        // one slice: slots (SP, SC, SN) hold slices zz - 1, zz, zz + 1; QB is the difference buffer
        auto step = [&](int zz, auto SPc, auto SCc, auto SNc, auto QBc, auto RPc) {
            constexpr int SP = decltype(SPc)::value, SC = decltype(SCc)::value, SN = decltype(SNc)::value;
            constexpr int QB = decltype(QBc)::value, RP = decltype(RPc)::value;
            if (zz + 1 <= zend) put(SN, R[RP]);
            if (zz + 3 <= zend) fetch(zz + 3, R[(RP + 2) % 3]);
            const bool zlow = HALO || zz > 0;
            float wz[NF][ROWS], r[NF][ROWS], wy[NF][ROWS], wx[NF][ROWS];
#pragma unroll
            for (int c = 0; c < NF; ++c) {
#pragma unroll
                for (int q = 0; q < ROWS; ++q) {
                    const int qy = ly + 8 * q;
                    r[c][q] = qpoint(c, lx, qy, SC, SP, zlow, wz[c][q], wy[c][q], wx[c][q]);
                    Qy[c][QB][qy][lx] = wy[c][q]; Qx[c][QB][qy][lx] = wx[c][q]; Qr[c][QB][qy][lx] = r[c][q];
                }
                if (extra) {
                    float a, b, e;
                    const float m = qpoint(c, eqx, eqy, SC, SP, zlow, a, b, e);
                    Qy[c][QB][eqy][eqx] = b; Qx[c][QB][eqy][eqx] = e; Qr[c][QB][eqy][eqx] = m;
                }
            }
            __syncthreads();
            // without the halo there is no +z neighbour above the last slice
            const bool zterm = HALO || zz < d.nz;
#pragma unroll
            for (int q = 0; q < ROWS; ++q) {
                const int qy = ly + 8 * q;
                if (zz > z0 && inside[q]) {   // slice zz-1 is complete with its +z neighbour's term
                    float gc[NF];
#pragma unroll
                    for (int c = 0; c < NF; ++c) gc[c] = zterm ? part[c][q] - wz[c][q] * r[c][q] : part[c][q];
                    const float g = NF == 2 ? fmaf(1.f - st.ratio, gc[0], st.ratio * gc[NF - 1]) : gc[0];
                    if (OUT == kTvOutNorm) acc += (double)g * (double)g;
                    else {
                        const int i = (zz - 1) * plane + own[q];
                        o[i] = OUT == kTvOutUpdate ? fmaf(-scale, g, fown[q]) : g;
                    }
                }
                if (zz < zend && inside[q]) {
#pragma unroll
                    for (int c = 0; c < NF; ++c) {
                        float g = (wz[c][q] + wy[c][q] + wx[c][q]) * r[c][q];
                        if (x + 1 < d.nx) g -= Qx[c][QB][qy][lx + 1] * Qr[c][QB][qy][lx + 1];
                        if (y0 + qy + 1 < d.ny) g -= Qy[c][QB][qy + 1][lx] * Qr[c][QB][qy + 1][lx];
                        part[c][q] = g;
                    }
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

// launch one tiled pass with the tile shape of tv_rows(KIND)
template <int OUT, int KIND>
void launch_tv_tiled(const float* f, float* o, const TVDims& d, const TVStep& st, double* sums, float alpha,
                     cudaStream_t s) {
    const int rows = tv_rows(KIND);
    const TvTiles T = tv_tiles(d, rows);
    if constexpr (KIND != kTvPiccs) {
        if (rows == 2) {
            tv_tiled_kernel<OUT, 2, KIND><<<tv_tiled_grid(T), 256, 0, s>>>(f, o, d, T, st, sums, alpha);
            return;
        }
    }
    tv_tiled_kernel<OUT, 1, KIND><<<tv_tiled_grid(T), 256, 0, s>>>(f, o, d, T, st, sums, alpha);
}

// POCS-TV step parameters (GD_TV.cu): no prior, no weights, 1e-7 under the norm, 1e-8 per gradient
constexpr TVStep kPocsStep{nullptr, 0.f, 0.f, 1e-7, 1e-8f};

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

}  // namespace
}  // namespace tigre

using namespace tigre;

extern "C" {

int tigre_tv_gradient(const void* d_img, int dtype, float* d_grad, long nx, long ny, long nz, void* stream) {
    if (dtype != TIGRE_F32) return fail(TIGRE_ERR_BAD_ASSERT, "TV kernels take float32 volumes");
    if (nx <= 0 || ny <= 0 || nz <= 0 || !d_img || !d_grad) return fail(TIGRE_ERR_BAD_ASSERT, "bad TV arguments");
    TVDims d{(int)nx, (int)ny, (int)nz};
    launch_tv_tiled<kTvOutGrad, kTvPocs>((const float*)d_img, d_grad, d, kPocsStep, nullptr, 0.f, (cudaStream_t)stream);
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
    TIGRE_NVTX("tigre_tv_pocs");
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
        launch_tv_tiled<kTvOutNorm, kTvPocs>(cur, nullptr, d, kPocsStep, sums + it, 0.f, st);
        launch_tv_tiled<kTvOutUpdate, kTvPocs>(cur, nxt, d, kPocsStep, sums + it, alpha, st);
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
        launch_tv_tiled<kTvOutNorm, KIND>(cur, nullptr, d, stp, sums + it, 0.f, st);
        launch_tv_tiled<kTvOutUpdate, KIND>(cur, nxt, d, stp, sums + it, alpha, st);
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
    TIGRE_NVTX("tigre_tv_aw_pocs");
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
    TIGRE_NVTX("tigre_tv_piccs");
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
// current and caches it; make that first call before any stream capture.  A device
// reset invalidates the cached address: tigre_release_cache() forgets it, and the
// next call looks it up again.
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

namespace tigre {
void forget_static_addresses() {
    std::lock_guard<std::mutex> lk(g_tv_pocs_sums_mu);
    for (auto& a : g_tv_pocs_sums_addr) a = nullptr;
}
}  // namespace tigre

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
        launch_tv_tiled<kTvOutNorm, kTvPocs>(cur, nullptr, d, kPocsStep, sums + it, 0.f, st);
        launch_tv_tiled<kTvOutUpdate, kTvPocs>(cur, nxt, d, kPocsStep, sums + it, alpha, st);
        std::swap(cur, nxt);
    }
    if (cur != (float*)d_img) TIGRE_CUDA(cudaMemcpyAsync(d_img, cur, n * sizeof(float), cudaMemcpyDeviceToDevice, st));
    TIGRE_CUDA(cudaGetLastError());
    note_launches(2ull * (unsigned long long)max_iter);
    return TIGRE_SUCCESS;
}
