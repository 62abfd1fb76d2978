// The glue of the warm-start U-Net's inference pass, fused so that each step is one pass over
// HBM (channels-last BF16 activations, FP32 arithmetic):
//   tigre_unet_pool2      2x2x2 average pooling                  (read 8 voxels, write 1)
//   tigre_unet_up_concat  nearest 2x upsampling of the deeper level concatenated with the skip
//                         connection along channels              (one write of the decoder input)
//   tigre_unet_conv_in    the first 3x3x3 convolution (one input channel, FP32 volume rounded to
//                         BF16 on the fly, FP32 accumulation, bias, ReLU)
//   tigre_unet_conv_out   the last 3x3x3 convolution (one output channel) rounded to BF16 as the
//                         convolution output is, plus the residual input volume, FP32 out
// The network's other convolutions are the tensor-core kernels of conv3d*.cu.

#include <cuda_bf16.h>

#include <algorithm>

#include "tigre_internal.h"

namespace tigre {
namespace {

int grid_for(long n) { return (int)std::min<long>((n + 255) / 256, 148L * 32); }

__device__ __forceinline__ void bf8_to_f(const uint4 v, float (&f)[8]) {
    const uint32_t w[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        f[2 * i] = __uint_as_float(w[i] << 16);
        f[2 * i + 1] = __uint_as_float(w[i] & 0xffff0000u);
    }
}

__device__ __forceinline__ uint4 f_to_bf8(const float (&f)[8]) {
    uint32_t w[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const __nv_bfloat162 h = __floats2bfloat162_rn(f[2 * i], f[2 * i + 1]);
        w[i] = *reinterpret_cast<const uint32_t*>(&h);
    }
    return make_uint4(w[0], w[1], w[2], w[3]);
}

// y[z][y][x][c] = mean of x over the 2x2x2 block; one thread per (voxel, 8 channels)
__global__ void pool2_kernel(const uint4* __restrict__ x, uint4* __restrict__ y, int D, int H, int W, int C8) {
    const int d = D / 2, h = H / 2, w = W / 2;
    const long total = (long)d * h * w * C8;
    for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < total; e += (long)gridDim.x * blockDim.x) {
        const int c = (int)(e % C8);
        long v = e / C8;
        const int ox = (int)(v % w), oy = (int)((v / w) % h), oz = (int)(v / ((long)w * h));
        float s[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            const int iz = 2 * oz + (k >> 2), iy = 2 * oy + ((k >> 1) & 1), ix = 2 * ox + (k & 1);
            float f[8];
            bf8_to_f(__ldg(x + (((long)iz * H + iy) * W + ix) * C8 + c), f);
#pragma unroll
            for (int j = 0; j < 8; ++j) s[j] += f[j];
        }
#pragma unroll
        for (int j = 0; j < 8; ++j) s[j] *= 0.125f;
        y[e] = f_to_bf8(s);
    }
}

// out[z][y][x][0:Ca] = low[z/2][y/2][x/2][:], out[z][y][x][Ca:Ca+Cb] = skip[z][y][x][:]
__global__ void up_concat_kernel(const uint4* __restrict__ low, int Ca8, const uint4* __restrict__ skip, int Cb8,
                                 uint4* __restrict__ out, int D, int H, int W) {
    const int C8 = Ca8 + Cb8;
    const long total = (long)D * H * W * C8;
    for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < total; e += (long)gridDim.x * blockDim.x) {
        const int c = (int)(e % C8);
        const long v = e / C8;
        uint4 val;
        if (c < Ca8) {
            const int x = (int)(v % W), y = (int)((v / W) % H), z = (int)(v / ((long)W * H));
            val = __ldg(low + ((((long)(z >> 1) * (H >> 1) + (y >> 1)) * (W >> 1) + (x >> 1)) * Ca8 + c));
        } else {
            val = __ldg(skip + v * Cb8 + (c - Ca8));
        }
        out[e] = val;
    }
}

// first convolution: one input channel (vol, FP32, rounded to BF16), Cout <= 32 outputs
template <int COUT>
__global__ void __launch_bounds__(256) conv_in_kernel(const float* __restrict__ vol, const __nv_bfloat16* __restrict__ w,
                                                      const float* __restrict__ b, __nv_bfloat16* __restrict__ y,
                                                      int D, int H, int W, int relu) {
    __shared__ float sw[27][COUT];
    __shared__ float sb[COUT];
    for (int i = threadIdx.x; i < 27 * COUT; i += blockDim.x) sw[i % 27][i / 27] = __bfloat162float(w[i]);
    for (int i = threadIdx.x; i < COUT; i += blockDim.x) sb[i] = b ? b[i] : 0.f;
    __syncthreads();
    const long total = (long)D * H * W;
    for (long v = blockIdx.x * (long)blockDim.x + threadIdx.x; v < total; v += (long)gridDim.x * blockDim.x) {
        const int x = (int)(v % W), yy = (int)((v / W) % H), z = (int)(v / ((long)W * H));
        float acc[COUT];
#pragma unroll
        for (int c = 0; c < COUT; ++c) acc[c] = sb[c];
#pragma unroll
        for (int t = 0; t < 27; ++t) {
            const int sx = x + t % 3 - 1, sy = yy + (t / 3) % 3 - 1, sz = z + t / 9 - 1;
            float in = 0.f;
            if (sx >= 0 && sx < W && sy >= 0 && sy < H && sz >= 0 && sz < D)
                in = __bfloat162float(__float2bfloat16(__ldg(vol + ((long)sz * H + sy) * W + sx)));
#pragma unroll
            for (int c = 0; c < COUT; ++c) acc[c] = fmaf(sw[t][c], in, acc[c]);
        }
#pragma unroll
        for (int q = 0; q < COUT / 8; ++q) {
            float f[8];
#pragma unroll
            for (int j = 0; j < 8; ++j) f[j] = relu ? fmaxf(acc[8 * q + j], 0.f) : acc[8 * q + j];
            reinterpret_cast<uint4*>(y + v * COUT)[q] = f_to_bf8(f);
        }
    }
}

// last convolution: CIN input channels -> 1, rounded to BF16, plus the residual volume (FP32)
template <int CIN>
__global__ void __launch_bounds__(256) conv_out_kernel(const __nv_bfloat16* __restrict__ x,
                                                       const __nv_bfloat16* __restrict__ w, float b,
                                                       const float* __restrict__ vol, float* __restrict__ out, int D,
                                                       int H, int W) {
    __shared__ float sw[27 * CIN];
    for (int i = threadIdx.x; i < 27 * CIN; i += blockDim.x) sw[i] = __bfloat162float(w[i]);
    __syncthreads();
    const long total = (long)D * H * W;
    for (long v = blockIdx.x * (long)blockDim.x + threadIdx.x; v < total; v += (long)gridDim.x * blockDim.x) {
        const int xx = (int)(v % W), yy = (int)((v / W) % H), z = (int)(v / ((long)W * H));
        float acc = b;
#pragma unroll 3
        for (int t = 0; t < 27; ++t) {
            const int sx = xx + t % 3 - 1, sy = yy + (t / 3) % 3 - 1, sz = z + t / 9 - 1;
            if (sx < 0 || sx >= W || sy < 0 || sy >= H || sz < 0 || sz >= D) continue;
            const uint4* src = reinterpret_cast<const uint4*>(x + (((long)sz * H + sy) * W + sx) * CIN);
#pragma unroll
            for (int q = 0; q < CIN / 8; ++q) {
                float f[8];
                bf8_to_f(__ldg(src + q), f);
#pragma unroll
                for (int j = 0; j < 8; ++j) acc = fmaf(sw[t * CIN + 8 * q + j], f[j], acc);
            }
        }
        out[v] = vol[v] + __bfloat162float(__float2bfloat16(acc));
    }
}

bool aligned16(const void* p) { return ((uintptr_t)p & 15) == 0; }

}  // namespace
}  // namespace tigre

using namespace tigre;

extern "C" {

int tigre_unet_pool2(const void* d_x, void* d_y, long D, long H, long W, long C, void* stream) {
    if (!d_x || !d_y || D <= 0 || H <= 0 || W <= 0 || D % 2 || H % 2 || W % 2 || C <= 0 || C % 8 ||
        !aligned16(d_x) || !aligned16(d_y))
        return fail(TIGRE_ERR_BAD_ASSERT, "unet pool2: even sizes, C % 8 == 0 and 16-byte aligned buffers");
    const long n = (D / 2) * (H / 2) * (W / 2) * (C / 8);
    pool2_kernel<<<grid_for(n), 256, 0, (cudaStream_t)stream>>>((const uint4*)d_x, (uint4*)d_y, (int)D, (int)H, (int)W,
                                                              (int)(C / 8));
    TIGRE_LAUNCHED();
    return TIGRE_SUCCESS;
}

int tigre_unet_up_concat(const void* d_low, long Ca, const void* d_skip, long Cb, void* d_out, long D, long H, long W,
                         void* stream) {
    if (!d_low || !d_skip || !d_out || D % 2 || H % 2 || W % 2 || D <= 0 || H <= 0 || W <= 0 || Ca % 8 || Cb % 8 ||
        Ca <= 0 || Cb <= 0 || !aligned16(d_low) || !aligned16(d_skip) || !aligned16(d_out))
        return fail(TIGRE_ERR_BAD_ASSERT, "unet up_concat: even sizes, channels % 8 == 0, 16-byte aligned buffers");
    const long n = D * H * W * ((Ca + Cb) / 8);
    up_concat_kernel<<<grid_for(n), 256, 0, (cudaStream_t)stream>>>((const uint4*)d_low, (int)(Ca / 8),
                                                                  (const uint4*)d_skip, (int)(Cb / 8), (uint4*)d_out,
                                                                  (int)D, (int)H, (int)W);
    TIGRE_LAUNCHED();
    return TIGRE_SUCCESS;
}

int tigre_unet_conv_in(const float* d_vol, const void* d_w, const float* d_b, void* d_y, long D, long H, long W,
                       long Cout, int relu, void* stream) {
    if (!d_vol || !d_w || !d_y || D <= 0 || H <= 0 || W <= 0 || !aligned16(d_y))
        return fail(TIGRE_ERR_BAD_ASSERT, "unet conv_in: bad arguments");
    const long n = D * H * W;
    cudaStream_t st = (cudaStream_t)stream;
    const __nv_bfloat16* w = (const __nv_bfloat16*)d_w;
    __nv_bfloat16* y = (__nv_bfloat16*)d_y;
    if (Cout == 8) conv_in_kernel<8><<<grid_for(n), 256, 0, st>>>(d_vol, w, d_b, y, (int)D, (int)H, (int)W, relu);
    else if (Cout == 16) conv_in_kernel<16><<<grid_for(n), 256, 0, st>>>(d_vol, w, d_b, y, (int)D, (int)H, (int)W, relu);
    else if (Cout == 32) conv_in_kernel<32><<<grid_for(n), 256, 0, st>>>(d_vol, w, d_b, y, (int)D, (int)H, (int)W, relu);
    else return fail(TIGRE_ERR_BAD_ASSERT, "unet conv_in: Cout must be 8, 16 or 32");
    TIGRE_LAUNCHED();
    return TIGRE_SUCCESS;
}

int tigre_unet_conv_out(const void* d_x, long Cin, const void* d_w, float b, const float* d_vol, float* d_out, long D,
                        long H, long W, void* stream) {
    if (!d_x || !d_w || !d_vol || !d_out || D <= 0 || H <= 0 || W <= 0 || !aligned16(d_x))
        return fail(TIGRE_ERR_BAD_ASSERT, "unet conv_out: bad arguments");
    const long n = D * H * W;
    cudaStream_t st = (cudaStream_t)stream;
    const __nv_bfloat16* x = (const __nv_bfloat16*)d_x;
    const __nv_bfloat16* w = (const __nv_bfloat16*)d_w;
    if (Cin == 8) conv_out_kernel<8><<<grid_for(n), 256, 0, st>>>(x, w, b, d_vol, d_out, (int)D, (int)H, (int)W);
    else if (Cin == 16) conv_out_kernel<16><<<grid_for(n), 256, 0, st>>>(x, w, b, d_vol, d_out, (int)D, (int)H, (int)W);
    else if (Cin == 32) conv_out_kernel<32><<<grid_for(n), 256, 0, st>>>(x, w, b, d_vol, d_out, (int)D, (int)H, (int)W);
    else return fail(TIGRE_ERR_BAD_ASSERT, "unet conv_out: Cin must be 8, 16 or 32");
    TIGRE_LAUNCHED();
    return TIGRE_SUCCESS;
}

}  // extern "C"
