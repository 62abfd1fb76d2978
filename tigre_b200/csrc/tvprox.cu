// TV proximal operator (ROF denoising by a primal-dual iteration), sm_100a.
//
// Same iteration as tvdenoising (Common/CUDA/tv_proximal.cu:185-630) on one device:
//   u = f, p = 0; for i < maxIter:
//     tau2 = 0.3 + 0.02 i,  tau1 = (1/tau2) (1/6 - 5/(15 + i))
//     u <- (1 - tau1) u + tau1 (f + div(p) / lambda)          (update_u, :136-153)
//     q = p + tau2 grad(u);  p <- q / max(1, |q|)              (update_p, :156-181)
// with backward-difference divergence (p taken as 0 before index 0, :81-109) and
// forward-difference gradient (0 at the last index, :111-134), each divided by the spacing.
// The volume is iterated with one extra slice below and above in z, as the reference's
// single-device layout does (buffer_length = 1): the lower one holds slice 1 of the image,
// the upper one zeros (cpy_from_host, :672-692, writes its mirror slice where the image
// copy then lands), and both evolve with the rest.
//
// Layout here: f, u, px, py, pz as (nZ + 2, nY, nX) x-fastest arrays in one work buffer.
// Each update is one pass over the volume (blocks over rows, threads along x, neighbours
// through L1);
// a step moves ~52 bytes per voxel, so the operator is HBM bound.

#include <cmath>

#include "tigre_internal.h"

namespace tigre {
namespace {

struct ProxDims {
    int nx, ny, nzp;         // nzp = nZ + 2
    float idx, idy, idz;     // 1 / spacing
};

// Voxels of the (nzp, ny, nx) arrays: blocks stride over (y, z) rows, threads over x, so no
// thread divides a linear index; i is the linear index of (x, y, z).
#define PROX_FOR_EACH_VOXEL(d, x, y, z, i)                                                   \
    for (long row_ = blockIdx.x; row_ < (long)(d).ny * (d).nzp; row_ += gridDim.x) {        \
        const int y = (int)(row_ % (d).ny), z = (int)(row_ / (d).ny);                         \
        for (int x = threadIdx.x; x < (d).nx; x += blockDim.x) {                               \
            const long i = row_ * (d).nx + x;
#define PROX_END_FOR_EACH_VOXEL \
    }                           \
    }

__global__ void __launch_bounds__(256) prox_update_u(const float* __restrict__ f, const float* __restrict__ pz,
                                                     const float* __restrict__ py, const float* __restrict__ px,
                                                     float* __restrict__ u, float tau, float inv_lambda, ProxDims d) {
    const long plane = (long)d.nx * d.ny;
    PROX_FOR_EACH_VOXEL(d, x, y, z, i) {
        float div = z > 0 ? (pz[i] - pz[i - plane]) * d.idz : pz[i];
        div += y > 0 ? (py[i] - py[i - d.nx]) * d.idy : py[i];
        div += x > 0 ? (px[i] - px[i - 1]) * d.idx : px[i];
        u[i] = u[i] * (1.f - tau) + tau * (f[i] + inv_lambda * div);
    }
    PROX_END_FOR_EACH_VOXEL
}

__global__ void __launch_bounds__(256) prox_update_p(const float* __restrict__ u, float* __restrict__ pz,
                                                     float* __restrict__ py, float* __restrict__ px, float tau,
                                                     ProxDims d) {
    const long plane = (long)d.nx * d.ny;
    PROX_FOR_EACH_VOXEL(d, x, y, z, i) {
        const float c = u[i];
        const float gz = z + 1 < d.nzp ? (u[i + plane] - c) * d.idz : 0.f;
        const float gy = y + 1 < d.ny ? (u[i + d.nx] - c) * d.idy : 0.f;
        const float gx = x + 1 < d.nx ? (u[i + 1] - c) * d.idx : 0.f;
        const float q0 = pz[i] + tau * gz, q1 = py[i] + tau * gy, q2 = px[i] + tau * gx;
        const float nrm = fmaxf(1.f, sqrtf(q0 * q0 + q1 * q1 + q2 * q2));
        pz[i] = q0 / nrm;
        py[i] = q1 / nrm;
        px[i] = q2 / nrm;
    }
    PROX_END_FOR_EACH_VOXEL
}

int grid_for_prox(const ProxDims& d) {
    return (int)std::min<long>((long)d.ny * d.nzp, 148L * 16);
}

}  // namespace
}  // namespace tigre

using namespace tigre;

extern "C" {

long long tigre_tv_denoise_work_floats(long nx, long ny, long nz) {
    return 5LL * nx * ny * (nz + 2);
}

int tigre_tv_denoise(const float* d_src, float* d_dst, long nx, long ny, long nz, float lambda, const float* spacing,
                     int max_iter, float* d_work, void* stream) {
    TIGRE_NVTX("tigre_tv_denoise");
    if (!d_src || !d_dst || !d_work || nx <= 0 || ny <= 0 || nz <= 0 || max_iter < 0)
        return fail(TIGRE_ERR_BAD_ASSERT, "bad TV denoising arguments");
    if (!(lambda > 0.f)) return fail(TIGRE_ERR_BAD_ASSERT, "TV denoising: lambda must be positive");
    if ((double)nx * ny * (nz + 2) >= 9.0e18 / 5) return fail(TIGRE_ERR_BAD_ASSERT, "volume too large");
    const float sx = spacing ? spacing[0] : 1.f, sy = spacing ? spacing[1] : 1.f, sz = spacing ? spacing[2] : 1.f;
    if (!(sx > 0.f && sy > 0.f && sz > 0.f)) return fail(TIGRE_ERR_BAD_ASSERT, "TV denoising: spacing must be positive");
    cudaStream_t st = (cudaStream_t)stream;
    const long plane = nx * ny, n = plane * (nz + 2);
    float* f = d_work;
    float* u = f + n;
    float* pz = u + n;
    float* py = pz + n;
    float* px = py + n;
    // f: [image slice 1 | image | zeros] (zeros also for a single-slice image)
    TIGRE_CUDA(cudaMemsetAsync(f, 0, sizeof(float) * n, st));
    if (nz > 1) TIGRE_CUDA(cudaMemcpyAsync(f, d_src + plane, sizeof(float) * plane, cudaMemcpyDeviceToDevice, st));
    TIGRE_CUDA(cudaMemcpyAsync(f + plane, d_src, sizeof(float) * plane * nz, cudaMemcpyDeviceToDevice, st));
    TIGRE_CUDA(cudaMemcpyAsync(u, f, sizeof(float) * n, cudaMemcpyDeviceToDevice, st));
    TIGRE_CUDA(cudaMemsetAsync(pz, 0, sizeof(float) * n * 3, st));
    ProxDims d{(int)nx, (int)ny, (int)(nz + 2), 1.f / sx, 1.f / sy, 1.f / sz};
    const int grid = grid_for_prox(d);
    for (int i = 0; i < max_iter; ++i) {
        const float tau2 = 0.3f + 0.02f * (float)i;
        const float tau1 = (1.f / tau2) * ((1.f / 6.f) - (5.f / (15.f + (float)i)));
        prox_update_u<<<grid, 256, 0, st>>>(f, pz, py, px, u, tau1, 1.f / lambda, d);
        TIGRE_LAUNCHED();
        prox_update_p<<<grid, 256, 0, st>>>(u, pz, py, px, tau2, d);
        TIGRE_LAUNCHED();
    }
    TIGRE_CUDA(cudaMemcpyAsync(d_dst, u + plane, sizeof(float) * plane * nz, cudaMemcpyDeviceToDevice, st));
    return TIGRE_SUCCESS;
}

}  // extern "C"
