// Working layouts of the projectors.
//
// The caller's volume is (z, y, x), x fastest.  A warp of rays covers 32
// neighbouring detector columns; when those columns step mostly along y (view
// angles near 0 or pi) the rays of the warp sit at 32 consecutive y, so a
// y-fastest copy (z, x, y) turns their gathers into one or two cache lines per
// warp load.  make_layout builds either copy, optionally zero-padded
// (pad_lo/pad_hi voxels per side) so that interpolation needs no bounds tests.
// pad_projections builds the zero-bordered projection stack of the
// backprojector (1 pixel before, 2 after, in u and v).

#include <type_traits>

#include "tigre_internal.h"

namespace tigre {
namespace {

constexpr int TILE = 32;

// layout 0: dst (Z', Y', X') x fastest;  layout 1: dst (Z', X', Y') y fastest.
// Primed extents are n + pad_lo + pad_hi; source coordinate = dst - pad_lo.
template <typename T, int LAYOUT>
__global__ void make_layout_kernel(const T* __restrict__ src, T* __restrict__ dst, int nX, int nY, int nZ, int plo,
                                   int phi) {
    __shared__ T tile[TILE][TILE + 1];
    const int XP = nX + plo + phi, YP = nY + plo + phi;
    const int zp = blockIdx.z;
    const int z = zp - plo;
    const bool zin = z >= 0 && z < nZ;
    // tile origin in (yp, xp)
    const int xp0 = blockIdx.x * TILE, yp0 = blockIdx.y * TILE;
    const size_t plane_src = (size_t)nX * nY;
    // load: threads along x for coalesced reads
    for (int j = threadIdx.y; j < TILE; j += blockDim.y) {
        const int yp = yp0 + j, xp = xp0 + threadIdx.x;
        const int y = yp - plo, x = xp - plo;
        T v = from_f32<T>(0.f);
        if (zin && x >= 0 && x < nX && y >= 0 && y < nY) v = src[(size_t)z * plane_src + (size_t)y * nX + x];
        tile[j][threadIdx.x] = v;
    }
    __syncthreads();
    if (LAYOUT == 0) {
        for (int j = threadIdx.y; j < TILE; j += blockDim.y) {
            const int yp = yp0 + j, xp = xp0 + threadIdx.x;
            if (yp < YP && xp < XP) dst[((size_t)zp * YP + yp) * XP + xp] = tile[j][threadIdx.x];
        }
    } else {
        // write transposed: threads along y
        for (int j = threadIdx.y; j < TILE; j += blockDim.y) {
            const int xp = xp0 + j, yp = yp0 + threadIdx.x;
            if (yp < YP && xp < XP) dst[((size_t)zp * XP + xp) * YP + yp] = tile[threadIdx.x][j];
        }
    }
}

// z-fastest copy with P zero slices before and after each z-run: dst (X, Y, Z+2P),
// dst[(x*Y + y)*(Z+2P) + zp] = src(z = zp-P, y, x), zero where zp-P is outside [0, Z).
// One y per block row of the grid; a 32x32 (zp, x) tile goes through shared memory.
template <typename Ts, typename T>
__global__ void make_zfast_kernel(const Ts* __restrict__ src, T* __restrict__ dst, int nX, int nY, int nZ, int P) {
    __shared__ T tile[TILE][TILE + 1];
    const int ZP = nZ + 2 * P;
    const int zp0 = blockIdx.x * TILE, x0 = blockIdx.y * TILE, y = blockIdx.z;
    for (int j = threadIdx.y; j < TILE; j += blockDim.y) {
        const int zp = zp0 + j, x = x0 + threadIdx.x, z = zp - P;
        T v = from_f32<T>(0.f);
        if (z >= 0 && z < nZ && x < nX) v = from_f32<T>(to_f32<Ts>(src[((size_t)z * nY + y) * nX + x]));
        tile[j][threadIdx.x] = v;
    }
    __syncthreads();
    for (int j = threadIdx.y; j < TILE; j += blockDim.y) {
        const int x = x0 + j, zp = zp0 + threadIdx.x;
        if (x < nX && zp < ZP) dst[((size_t)x * nY + y) * ZP + zp] = tile[threadIdx.x][j];
    }
}

// Corner quads for the interpolated projector: from a padded copy (layout 0: x fastest,
// layout 1: y fastest; F = padded fast extent, O = padded other extent, Z = padded z extent),
// element i = (p[i], p[i+1], p[i+F*O], p[i+1+F*O]) -- the fast-axis x z 2x2 corner block of
// a trilinear sample, read as one vector load.  Corners past the last fast or z index are 0
// (no sample has its base there).  FP32 quads hold the fast-axis differences instead of the
// second corners, (p[i], p[i+1] - p[i], p[i+F*O], p[i+1+F*O] - p[i+F*O]), rounded to FP32 as
// the sampler's own subtraction would be: each fast-axis lerp is then one FMA, with the same
// result.
template <typename T>
struct Quad4 { T v[4]; };

template <typename Ts, typename T>
__global__ void make_quads_kernel(const Ts* __restrict__ pad, Quad4<T>* __restrict__ dst, int F, int O, int Z) {
    const long plane = (long)F * O, total = plane * Z;
    auto cv = [](Ts v) { return from_f32<T>(to_f32<Ts>(v)); };
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
        const int f = (int)(i % F);
        const long zp = i / plane;
        const bool f1 = f + 1 < F, z1 = zp + 1 < Z;
        Quad4<T> q;
        q.v[0] = cv(pad[i]);
        q.v[1] = f1 ? cv(pad[i + 1]) : from_f32<T>(0.f);
        q.v[2] = z1 ? cv(pad[i + plane]) : from_f32<T>(0.f);
        q.v[3] = (f1 && z1) ? cv(pad[i + plane + 1]) : from_f32<T>(0.f);
        if constexpr (std::is_same<T, float>::value) {
            q.v[1] = __fsub_rn(q.v[1], q.v[0]);
            q.v[3] = __fsub_rn(q.v[3], q.v[2]);
        }
        dst[i] = q;
    }
}

template <typename T>
__global__ void pad_projections_kernel(const T* __restrict__ src, T* __restrict__ dst, int nV, int nU, long total) {
    const long pitch = bp_pitch(nU), rows = bp_rows(nV);
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
        const long a = i / (pitch * rows);
        const long rem = i - a * pitch * rows;
        const int r = (int)(rem / pitch), c = (int)(rem - (long)r * pitch);
        const int v = r - 1, u = c - 1;
        T val = from_f32<T>(0.f);
        if (v >= 0 && v < nV && u >= 0 && u < nU) val = src[(a * nV + v) * (long)nU + u];
        dst[i] = val;
    }
}

template <typename Ts, typename T>
__global__ void repitch_kernel(const Ts* __restrict__ src, T* __restrict__ dst, int nU, int pitch, long rows) {
    const long total = rows * pitch;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
        const long r = i / pitch;
        const int c = (int)(i - r * pitch);
        dst[i] = c < nU ? from_f32<T>(to_f32<Ts>(src[r * nU + c])) : from_f32<T>(0.f);
    }
}

}  // namespace

int launch_repitch_projections(const void* src, int dtype, void* dst, int nA, int nV, int nU, int pitch,
                               cudaStream_t st) {
    const long rows = (long)nA * nV;
    const long want = (rows * pitch + 255) / 256;
    const int grid = (int)std::min<long>(want, 148L * 32);
    TIGRE_DISPATCH_DTYPE(dtype, T, { repitch_kernel<T, T><<<grid, 256, 0, st>>>((const T*)src, (T*)dst, nU, pitch, rows); });
    TIGRE_LAUNCHED();
    return TIGRE_SUCCESS;
}

// 16-bit projections widened to FP32 on the way (exact), same pitching as above
int launch_repitch_projections_f32(const void* src, int dtype, float* dst, int nA, int nV, int nU, int pitch,
                                   cudaStream_t st) {
    const long rows = (long)nA * nV;
    const long want = (rows * pitch + 255) / 256;
    const int grid = (int)std::min<long>(want, 148L * 32);
    TIGRE_DISPATCH_DTYPE(dtype, T, { repitch_kernel<T, float><<<grid, 256, 0, st>>>((const T*)src, dst, nU, pitch, rows); });
    TIGRE_LAUNCHED();
    return TIGRE_SUCCESS;
}

int launch_make_layout(const void* src, int dtype, void* dst, int nX, int nY, int nZ, int layout, int pad_lo,
                       int pad_hi, cudaStream_t st) {
    const int p = pad_lo + pad_hi;
    dim3 block(TILE, 8);
    dim3 grid((nX + p + TILE - 1) / TILE, (nY + p + TILE - 1) / TILE, nZ + p);
    TIGRE_DISPATCH_DTYPE(dtype, T, {
        if (layout == 0)
            make_layout_kernel<T, 0><<<grid, block, 0, st>>>((const T*)src, (T*)dst, nX, nY, nZ, pad_lo, pad_hi);
        else
            make_layout_kernel<T, 1><<<grid, block, 0, st>>>((const T*)src, (T*)dst, nX, nY, nZ, pad_lo, pad_hi);
    });
    TIGRE_LAUNCHED();
    return TIGRE_SUCCESS;
}

int launch_make_zfast(const void* src, int dtype, void* dst, int nX, int nY, int nZ, int zpad, cudaStream_t st) {
    dim3 block(TILE, 8);
    dim3 grid((nZ + 2 * zpad + TILE - 1) / TILE, (nX + TILE - 1) / TILE, nY);
    TIGRE_DISPATCH_DTYPE(dtype, T, {
        make_zfast_kernel<T, T><<<grid, block, 0, st>>>((const T*)src, (T*)dst, nX, nY, nZ, zpad);
    });
    TIGRE_LAUNCHED();
    return TIGRE_SUCCESS;
}

// FP32 z-fast copy of a volume of any storage type (16-bit values widen exactly)
int launch_make_zfast_f32(const void* src, int dtype, float* dst, int nX, int nY, int nZ, int zpad, cudaStream_t st) {
    dim3 block(TILE, 8);
    dim3 grid((nZ + 2 * zpad + TILE - 1) / TILE, (nX + TILE - 1) / TILE, nY);
    TIGRE_DISPATCH_DTYPE(dtype, T, {
        make_zfast_kernel<T, float><<<grid, block, 0, st>>>((const T*)src, dst, nX, nY, nZ, zpad);
    });
    TIGRE_LAUNCHED();
    return TIGRE_SUCCESS;
}

int launch_make_quads(const void* pad, int dtype, void* dst, int nX, int nY, int nZ, int layout, cudaStream_t st) {
    const int F = (layout ? nY : nX) + 3, O = (layout ? nX : nY) + 3, Z = nZ + 3;
    const long total = (long)F * O * Z;
    const int grid = (int)std::min<long>((total + 255) / 256, 148L * 32);
    TIGRE_DISPATCH_DTYPE(dtype, T, {
        make_quads_kernel<T, T><<<grid, 256, 0, st>>>((const T*)pad, (Quad4<T>*)dst, F, O, Z);
    });
    TIGRE_LAUNCHED();
    return TIGRE_SUCCESS;
}

// FP32 corner quads from a padded copy of any storage type
int launch_make_quads_f32(const void* pad, int dtype, float* dst, int nX, int nY, int nZ, int layout, cudaStream_t st) {
    const int F = (layout ? nY : nX) + 3, O = (layout ? nX : nY) + 3, Z = nZ + 3;
    const long total = (long)F * O * Z;
    const int grid = (int)std::min<long>((total + 255) / 256, 148L * 32);
    TIGRE_DISPATCH_DTYPE(dtype, T, {
        make_quads_kernel<T, float><<<grid, 256, 0, st>>>((const T*)pad, (Quad4<float>*)dst, F, O, Z);
    });
    TIGRE_LAUNCHED();
    return TIGRE_SUCCESS;
}

int launch_pad_projections(const void* src, int dtype, void* dst, int nA, int nV, int nU, cudaStream_t st) {
    const long total = (long)nA * bp_rows(nV) * bp_pitch(nU);
    const int block = 256;
    const long want = (total + block - 1) / block;
    const int grid = (int)std::min<long>(want, 148L * 32);
    TIGRE_DISPATCH_DTYPE(dtype, T, {
        pad_projections_kernel<T><<<grid, block, 0, st>>>((const T*)src, (T*)dst, nV, nU, total);
    });
    TIGRE_LAUNCHED();
    return TIGRE_SUCCESS;
}

}  // namespace tigre
