// FP64-accumulated reductions and fused CGLS vector updates.
//
// CGLS (Python/tigre/algorithms/krylov_subspace_algorithms.py:46-97) keeps its
// vectors in host numpy and its scalars alpha = gamma/|q|^2, beta = gamma'/gamma
// in host floats.  Here the vectors stay in HBM and the scalars in device
// FP64: each update reads its scalar pair from device memory, so an iteration
// needs no host synchronisation.

#include <cmath>

#include "tigre_internal.h"

namespace tigre {
namespace {

__device__ __forceinline__ double warp_block_sum(double v) {
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

template <typename T>
__global__ void __launch_bounds__(256) sumsq_kernel(const T* __restrict__ x, long n, double* __restrict__ out) {
    double s = 0.0;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        const double v = (double)to_f32<T>(x[i]);
        s = fma(v, v, s);
    }
    s = warp_block_sum(s);
    if (threadIdx.x == 0) atomicAdd(out, s);
}

__global__ void __launch_bounds__(256) dot_kernel(const float* __restrict__ x, const float* __restrict__ y, long n,
                                                  double* __restrict__ out) {
    double s = 0.0;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
        s = fma((double)x[i], (double)y[i], s);
    s = warp_block_sum(s);
    if (threadIdx.x == 0) atomicAdd(out, s);
}

// x += a p over the volume; r -= a q over the projections (and |r|^2 into rr)
__global__ void __launch_bounds__(256) cgls_step_kernel(float* __restrict__ x, const float* __restrict__ p, long nvol,
                                                        float* __restrict__ r, const float* __restrict__ q, long nproj,
                                                        const double* __restrict__ num, const double* __restrict__ den,
                                                        double* __restrict__ rr) {
    const double a = *num / *den;
    const float af = (float)a;
    const long stride = (long)gridDim.x * blockDim.x;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < nvol; i += stride) x[i] = fmaf(af, p[i], x[i]);
    double s = 0.0;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < nproj; i += stride) {
        const float v = fmaf(-af, q[i], r[i]);
        r[i] = v;
        s = fma((double)v, (double)v, s);
    }
    if (rr) {
        s = warp_block_sum(s);
        if (threadIdx.x == 0) atomicAdd(rr, s);
    }
}

__global__ void __launch_bounds__(256) cgls_dir_kernel(float* __restrict__ p, const float* __restrict__ s, long n,
                                                       const double* __restrict__ num, const double* __restrict__ den) {
    const float b = (float)(*num / *den);
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
        p[i] = fmaf(b, p[i], s[i]);
}

template <typename TS, typename TD>
__global__ void convert_kernel(const TS* __restrict__ s, TD* __restrict__ d, long n) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
        d[i] = from_f32<TD>(to_f32<TS>(s[i]));
}

int grid_for(long n) {
    const long want = (n + 255) / 256;
    return (int)std::max<long>(1, std::min<long>(want, 148 * 8));
}

}  // namespace
}  // namespace tigre

using namespace tigre;

extern "C" {

int tigre_sumsq(const void* d_x, int dtype, long n, double* d_out, void* stream) {
    if (n < 0 || (!d_x && n) || !d_out) return fail(TIGRE_ERR_BAD_ASSERT, "bad sumsq arguments");
    if (n == 0) return TIGRE_SUCCESS;
    cudaStream_t st = (cudaStream_t)stream;
    TIGRE_DISPATCH_DTYPE(dtype, T, { sumsq_kernel<T><<<grid_for(n), 256, 0, st>>>((const T*)d_x, n, d_out); });
    TIGRE_LAUNCHED();
    return TIGRE_SUCCESS;
}

int tigre_dot(const float* d_x, const float* d_y, long n, double* d_out, void* stream) {
    if (n < 0 || !d_out) return fail(TIGRE_ERR_BAD_ASSERT, "bad dot arguments");
    if (n == 0) return TIGRE_SUCCESS;
    dot_kernel<<<grid_for(n), 256, 0, (cudaStream_t)stream>>>(d_x, d_y, n, d_out);
    TIGRE_LAUNCHED();
    return TIGRE_SUCCESS;
}

int tigre_cgls_step(float* d_x, const float* d_p, long nvol, float* d_r, const float* d_q, long nproj,
                    const double* d_num, const double* d_den, double* d_rr, void* stream) {
    if (nvol < 0 || nproj < 0 || !d_num || !d_den) return fail(TIGRE_ERR_BAD_ASSERT, "bad cgls_step arguments");
    cgls_step_kernel<<<grid_for(std::max(nvol, nproj)), 256, 0, (cudaStream_t)stream>>>(d_x, d_p, nvol, d_r, d_q,
                                                                                        nproj, d_num, d_den, d_rr);
    TIGRE_LAUNCHED();
    return TIGRE_SUCCESS;
}

int tigre_cgls_direction(float* d_p, const float* d_s, long n, const double* d_num, const double* d_den,
                         void* stream) {
    if (n < 0 || !d_num || !d_den) return fail(TIGRE_ERR_BAD_ASSERT, "bad cgls_direction arguments");
    cgls_dir_kernel<<<grid_for(n), 256, 0, (cudaStream_t)stream>>>(d_p, d_s, n, d_num, d_den);
    TIGRE_LAUNCHED();
    return TIGRE_SUCCESS;
}

int tigre_convert(const void* d_src, int sdt, void* d_dst, int ddt, long n, void* stream) {
    if (n < 0) return fail(TIGRE_ERR_BAD_ASSERT, "bad convert arguments");
    if (n == 0) return TIGRE_SUCCESS;
    cudaStream_t st = (cudaStream_t)stream;
    TIGRE_DISPATCH_DTYPE(sdt, TS, {
        TIGRE_DISPATCH_DTYPE(ddt, TD, {
            convert_kernel<TS, TD><<<grid_for(n), 256, 0, st>>>((const TS*)d_src, (TD*)d_dst, n);
        });
    });
    TIGRE_LAUNCHED();
    return TIGRE_SUCCESS;
}

}  // extern "C"
