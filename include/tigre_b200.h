/*
 * tigre_b200.h -- C ABI of libtigre_b200.so, the sm_100a projector pair.
 *
 * Two layers of entry points live in the same shared library:
 *
 *  1. Drop-in host-pointer calls with the reference's argument meaning and
 *     error codes.  Each replaces one reference function of TIGRE's
 *     Common/CUDA layer (cited per declaration).  They take host pointers,
 *     block until the result is in host memory, and return 0 on success or a
 *     code of Common/CUDA/errors.hpp:1-7 (they never exit the process, unlike
 *     the reference's mexErrMsgIdAndTxt, TIGRE_common.cpp:13-16).
 *     C++ callers that bind the reference's exact C++ signatures (the unmodified
 *     Cython _Ax/_Atb/_minTV extensions) use include/tigre_b200_compat.hpp,
 *     whose functions are exported by the same library.
 *
 *  2. A device-resident API (plan + device pointers + CUDA stream) used by the
 *     Python package for algorithms, autograd and benchmarks.  It has no
 *     counterpart in the reference, whose every call copies host<->device.
 *
 * All pointers are plain pointers; streams are passed as void* (cudaStream_t).
 */
#ifndef TIGRE_B200_H
#define TIGRE_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Error codes, values of Common/CUDA/errors.hpp:1-7. */
#define TIGRE_SUCCESS 0
#define TIGRE_ERR_CUDA 1
#define TIGRE_ERR_NO_CAPABLE_DEVICES 2
#define TIGRE_ERR_NO_FREE_DEVICES 3
#define TIGRE_ERR_BAD_ASSERT 4
#define TIGRE_ERR_ASSERT_FAIL 5

/* Storage types accepted by the device API (arithmetic is always FP32, geometry FP64). */
#define TIGRE_F32 0
#define TIGRE_BF16 1
#define TIGRE_F16 2

/* Projector / backprojector selectors. */
#define TIGRE_PROJ_SIDDON 0
#define TIGRE_PROJ_INTERPOLATED 1
#define TIGRE_BACKPROJ_FDK 0
#define TIGRE_BACKPROJ_MATCHED 1

/* Rounding of FP32 results into 16-bit storage (tigre_sart_update). */
#define TIGRE_ROUND_NEAREST 0
#define TIGRE_ROUND_STOCHASTIC 1

/*
 * Per-call geometry: field-for-field the layout of `struct Geometry`
 * (Common/CUDA/types_TIGRE.hpp:48-85).  Per-angle arrays have nangles entries.
 * Axes are in the C convention: X fastest, detector U fastest.
 */
typedef struct TigreGeometry {
    int nVoxelX, nVoxelY, nVoxelZ;
    float sVoxelX, sVoxelY, sVoxelZ;
    float dVoxelX, dVoxelY, dVoxelZ;
    float *offOrigX, *offOrigY, *offOrigZ;
    float *DSO;
    int nDetecU, nDetecV;
    float sDetecU, sDetecV;
    float dDetecU, dDetecV;
    float *offDetecU, *offDetecV;
    float *DSD;
    float *dRoll;
    float *dPitch;
    float *dYaw;
    float unitX, unitY, unitZ;
    float alpha, theta, psi;
    float *COR;
    float maxLength;
    float accuracy;
} TigreGeometry;

/* Text of the last error raised on the calling thread ("" if none). */
const char* tigre_last_error(void);
/* Library version (major*100 + minor). */
int tigre_version(void);
/* Number of kernels this library has launched in this process, on all devices. */
unsigned long long tigre_launch_count(void);

/* ---------------------------------------------------------------------------
 * 1. Drop-in host-pointer entry points.
 *    gpu_ids/n_gpus: device list of the reference's GpuIds (Common/CUDA/GpuIds.hpp);
 *    this build runs on gpu_ids[0] (n_gpus == 0 means device 0).
 * ------------------------------------------------------------------------- */

/* Siddon ray-driven cone-beam projection.  Replaces siddon_ray_projection
 * (Common/CUDA/Siddon_projection.hpp:54, Siddon_projection.cu:271).
 * img: (nVoxelZ, nVoxelY, nVoxelX) float32; result[i]: projection i, (nDetecV, nDetecU);
 * angles: (nangles, 3) ZYZ Euler angles. */
int tigre_siddon_ray_projection(const float* img, const TigreGeometry* geo, float* const* result,
                                const float* angles, int nangles, const int* gpu_ids, int n_gpus);

/* Interpolated (fixed-step trilinear) cone-beam projection.  Replaces
 * interpolation_projection (Common/CUDA/ray_interpolated_projection.hpp:55,
 * ray_interpolated_projection.cu:211). */
int tigre_interpolation_projection(const float* img, const TigreGeometry* geo, float* const* result,
                                   const float* angles, int nangles, const int* gpu_ids, int n_gpus);

/* FDK-weighted voxel backprojection.  Replaces voxel_backprojection
 * (Common/CUDA/voxel_backprojection.hpp:52, voxel_backprojection.cu:293).
 * projections: (nangles, nDetecV, nDetecU); result: (nVoxelZ, nVoxelY, nVoxelX), overwritten. */
int tigre_voxel_backprojection(const float* projections, const TigreGeometry* geo, float* result,
                               const float* angles, int nangles, const int* gpu_ids, int n_gpus);

/* Matched voxel backprojection (weight L^3/(DSD*|S-x|^2), scaled by dV/dDetArea).
 * Replaces voxel_backprojection2 (Common/CUDA/voxel_backprojection2.hpp:57,
 * voxel_backprojection2.cu:318). */
int tigre_voxel_backprojection2(const float* projections, const TigreGeometry* geo, float* result,
                                const float* angles, int nangles, const int* gpu_ids, int n_gpus);

/* POCS total-variation descent: maxIter steps of img -= alpha*g/|g|, g = grad TV(img).
 * Replaces pocs_tv (Common/CUDA/GD_TV.hpp:58, GD_TV.cu:255).  image_size = {nX, nY, nZ}.
 * Unlike the reference it does not reset the device at the end. */
int tigre_pocs_tv(const float* img, float* dst, float alpha, const long* image_size, int max_iter,
                  const int* gpu_ids, int n_gpus);

/* Adaptive-weighted TV descent: as tigre_pocs_tv with each difference component weighted by
 * exp(-(d/delta)^2).  Replaces aw_pocs_tv (Common/CUDA/GD_AwTV.hpp:58, GD_AwTV.cu:276), the
 * operator behind tigre.utilities.AwminTV (_AwminTV.pyx). */
int tigre_aw_pocs_tv(const float* img, float* dst, float alpha, const long* image_size, int max_iter, float delta,
                     const int* gpu_ids, int n_gpus);

/* PICCS TV descent: maxIter steps of img -= alpha*g/|g| with
 * g = (1-ratio) grad TV(img) + ratio grad TV(img - prior), one-sided differences at every face.
 * Replaces piccs_tv (Common/CUDA/PICCS.hpp:58, PICCS.cu:274), behind
 * tigre.utilities.minPICCS (_minPICCS.pyx).  As the reference, |g| has no epsilon: a
 * constant image and prior give NaN. */
int tigre_piccs_tv(const float* img, const float* prior, float* dst, float alpha, float ratio, const long* image_size,
                   int max_iter, const int* gpu_ids, int n_gpus);

/* TV denoising by the primal-dual iteration of tvdenoising (Common/CUDA/tv_proximal.hpp,
 * tv_proximal.cu:185), the operator behind tigre.utilities.im3ddenoise (_tv_proximal.pyx).
 * src, dst: (nZ, nY, nX) float32 host arrays; image_size = {nX, nY, nZ}; spacing = {dX, dY, dZ}. */
int tigre_tvdenoising(const float* src, float* dst, float lambda, const float* spacing, const long* image_size,
                      int max_iter, const int* gpu_ids, int n_gpus);

/* Poisson noise out[i] = Poisson(in[i]), plus N(mu, sigma) when gaussian != 0, on n host floats.
 * Replaces poisson_1d / poisson_gaussian_1d (Common/CUDA/RandomNumberGenerator.hpp,
 * RandomNumberGenerator.cu), behind tigre.utilities.CTnoise.add.  Counter-based: the result
 * depends only on seed and element index (the reference's curand stream cannot be reproduced;
 * the C++ compat symbols pass the reference's fixed seed 1234). */
int tigre_noise_1d(const float* in, long long n, int gaussian, float mu, float sigma, unsigned long long seed,
                   float* out, const int* gpu_ids, int n_gpus);

/* Parallel-beam projection and backprojection.  Replace siddon_ray_projection_parallel
 * (Common/CUDA/Siddon_projection_parallel.hpp, Siddon_projection_parallel.cu:270),
 * interpolation_projection_parallel (ray_interpolated_projection_parallel.hpp,
 * ray_interpolated_projection_parallel.cu:195) and voxel_backprojection_parallel
 * (voxel_backprojection_parallel.hpp, voxel_backprojection_parallel.cu), called by
 * _Ax.pyx:85-87 and _Atb.pyx:75.  Same arguments as the cone-beam calls. */
int tigre_siddon_ray_projection_parallel(const float* img, const TigreGeometry* geo, float* const* result,
                                         const float* angles, int nangles, const int* gpu_ids, int n_gpus);
int tigre_interpolation_projection_parallel(const float* img, const TigreGeometry* geo, float* const* result,
                                            const float* angles, int nangles, const int* gpu_ids, int n_gpus);
int tigre_voxel_backprojection_parallel(const float* projections, const TigreGeometry* geo, float* result,
                                        const float* angles, int nangles, const int* gpu_ids, int n_gpus);

/* ---------------------------------------------------------------------------
 * 2. Device-resident API (no counterpart in the reference).
 * ------------------------------------------------------------------------- */

/* A plan holds the FP64 per-angle geometry (uploaded once) and reusable device
 * scratch for the working layouts of one geometry.  Plans are not thread-safe:
 * use one plan per host thread / stream. */
typedef struct TigrePlan TigrePlan;

int tigre_plan_create(const TigreGeometry* geo, const float* angles, int nangles, int device, TigrePlan** plan);
/* As tigre_plan_create; flags: TIGRE_PLAN_PARALLEL for a parallel-beam geometry (the frames
 * of the reference's *_parallel functions; tigre_ax / tigre_atb then project and backproject
 * in parallel beam, and the backprojector type is ignored, as in the reference). */
#define TIGRE_PLAN_PARALLEL 1
int tigre_plan_create_ex(const TigreGeometry* geo, const float* angles, int nangles, int device, int flags,
                         TigrePlan** plan);
void tigre_plan_destroy(TigrePlan* plan);
/* Bytes of device scratch currently held by the plan. */
long long tigre_plan_scratch_bytes(const TigrePlan* plan);
/* Synchronises the plan's device and returns its kernel status word (0 = ok; bit 0:
 * a bounded wait inside a kernel expired, results of that call are invalid; bit 1: the
 * cell-interval Siddon kernel met a ray outside the z bound computed at plan time and
 * wrote 0 for it).  reset != 0 clears it. */
#define TIGRE_STATUS_WAIT_EXPIRED 1
#define TIGRE_STATUS_RAY_DROPPED 2
int tigre_plan_status(TigrePlan* plan, int reset);

/* Forward projection of d_vol (nZ,nY,nX) into d_proj ((angle_end-angle_begin), nV, nU)
 * for plan angles [angle_begin, angle_end).  projector: TIGRE_PROJ_*. */
int tigre_ax(TigrePlan* plan, const void* d_vol, int vol_dtype, void* d_proj, int proj_dtype, int projector,
             int angle_begin, int angle_end, void* stream);

/* Backprojection of d_proj ((angle_end-angle_begin), nV, nU) into d_vol (overwritten).
 * backprojector: TIGRE_BACKPROJ_*. */
int tigre_atb(TigrePlan* plan, const void* d_proj, int proj_dtype, void* d_vol, int vol_dtype, int backprojector,
              int angle_begin, int angle_end, void* stream);

/* As tigre_atb; accumulate != 0 adds into d_vol instead of overwriting it (lets a caller
 * stream the views in chunks). */
int tigre_atb_ex(TigrePlan* plan, const void* d_proj, int proj_dtype, void* d_vol, int vol_dtype, int backprojector,
                 int angle_begin, int angle_end, int accumulate, void* stream);

/* Frees the device buffers and plans that the host entry points keep between calls, and
 * forgets the device addresses of this library's fixed device arrays (call it after a
 * cudaDeviceReset before the next call into the library). */
void tigre_release_cache(void);

/* Library options (no counterpart in the reference).  They select kernel variants for
 * diagnosis and testing, set how the host entry points move data, or make one launch fail
 * in a controlled way for the failure-detection tests.  Options read when a plan is
 * created (SIDDON_KERNEL, BP_BOX, BP_KERNEL) apply to plans created afterwards; the host
 * entry points keep plans between calls, so call tigre_release_cache() after changing
 * one.  tigre_set_option returns the previous value (or -1 with TIGRE_ERR_BAD_ASSERT in
 * tigre_last_error for an unknown option). */
#define TIGRE_OPT_SIDDON_KERNEL 1    /* 0 auto; 1 stepped column kernel instead of the cell-interval one; 2 the generic per-ray kernel */
#define TIGRE_OPT_BP_BOX 2           /* 0 auto; else (BU << 16) | BV: the staged backprojector's patch box */
#define TIGRE_OPT_BP_KERNEL 3        /* 0 auto; 1 the plain global-load backprojector instead of the TMA-staged one */
#define TIGRE_OPT_HOST_CHUNK_VIEWS 4 /* 0 auto (~192 MB of projections); else views per host<->device chunk */
#define TIGRE_OPT_HOST_STAGING 5     /* -1 auto; else a bit mask of the copies staged through pinned buffers:
                                        1 volume uploads, 2 volume downloads, 4 backprojector chunk uploads,
                                        8 backprojector volume download */
#define TIGRE_OPT_BP_SKIP_COPY 6     /* -1 off; else the staged backprojector issues no copy for this view index
                                        of every launch, so the wait for it runs out: the kernel then sets the
                                        plan status and the call returns TIGRE_ERR_CUDA (failure-detection test) */
#define TIGRE_OPT_INTERP_TEXTURE 7    /* 0 exact trilinear (default); 1 the interpolated projector samples through
                                        the texture unit's linear filter (8-bit weights, ~2^-9 relative per
                                        sample, as the reference's texture path) */
long long tigre_set_option(int option, long long value);
long long tigre_get_option(int option);

/* Sum over all rays of the number of Siddon voxel segments (FP64 ray setup only,
 * no traversal); the algorithmic-bytes count of the Siddon roofline. */
int tigre_siddon_count_segments(TigrePlan* plan, int angle_begin, int angle_end, unsigned long long* d_total,
                                void* stream);
/* Sum over all rays of the number of interpolated samples strictly inside the volume's open
 * box (-1, n) per axis, i.e. those whose trilinear footprint can be nonzero (FP64 ray setup of
 * ray_interpolated_projection.cu:153-199, no sampling); the algorithmic-bytes count of the
 * interpolated projector's roofline. */
int tigre_interp_count_samples(TigrePlan* plan, int angle_begin, int angle_end, unsigned long long* d_total,
                               void* stream);

/* POCS-TV on a device volume, in place: max_iter steps of GD_TV.cu:440-597.
 * d_work: caller scratch of nx*ny*nz floats (same dtype as d_img is not required: FP32). */
int tigre_tv_pocs(void* d_img, int dtype, long nx, long ny, long nz, float alpha, int max_iter, float* d_work,
                  void* stream);
/* As tigre_tv_pocs, but allocates no device memory (no counterpart in the reference).
 * The per-iteration norm sums live in a fixed 32 KiB device array of the library, so
 * max_iter <= 4096 (larger values return TIGRE_ERR_BAD_ASSERT).  All calls on a device
 * share that array: calls that overlap in time on one device race and must be
 * serialised by the caller.  The first call on each device looks up the array's
 * address with that device current; make it before any stream capture.  After a
 * cudaDeviceReset the cached address is stale: call tigre_release_cache() first, which
 * makes the next call look it up again. */
int tigre_tv_pocs_noalloc(void* d_img, int dtype, long nx, long ny, long nz, float alpha, int max_iter,
                          float* d_work, void* stream);
/* Device counterparts of tigre_aw_pocs_tv and tigre_piccs_tv, in place on d_img; d_work:
 * nx*ny*nz floats of caller scratch; d_prior: the prior image (FP32, same layout). */
int tigre_tv_aw_pocs(void* d_img, int dtype, long nx, long ny, long nz, float alpha, int max_iter, float delta,
                     float* d_work, void* stream);
int tigre_tv_piccs(void* d_img, const void* d_prior, int dtype, long nx, long ny, long nz, float alpha, float ratio,
                   int max_iter, float* d_work, void* stream);
/* Device TV denoising (same iteration as tigre_tvdenoising) of d_src into d_dst (may alias);
 * d_work: tigre_tv_denoise_work_floats(nx, ny, nz) floats of caller scratch. */
long long tigre_tv_denoise_work_floats(long nx, long ny, long nz);
int tigre_tv_denoise(const float* d_src, float* d_dst, long nx, long ny, long nz, float lambda, const float* spacing,
                     int max_iter, float* d_work, void* stream);
/* TV gradient (GD_TV.cu:117-143, single-device boundary rule) into d_grad (FP32). */
int tigre_tv_gradient(const void* d_img, int dtype, float* d_grad, long nx, long ny, long nz, void* stream);
/* TV value sum_i |grad f_i| consistent with tigre_tv_gradient; added into *d_out (FP64). */
int tigre_tv_value(const void* d_img, int dtype, long nx, long ny, long nz, double* d_out, void* stream);

/* SART-family volume update in place: d_x[z][j] <- max(d_x + (lambda / d_v[j]) * d_bp[z][j], 0)
 * for z < nz, j < nyx (the clip only when noneg), the update of IterativeReconAlg.update_image
 * (Python/tigre/algorithms/iterative_recon_alg.py:389-401) with the clip of art_data_minimizing
 * (:344-345) in one pass.  d_x: storage dtype; d_bp: FP32 backprojection; d_v: FP32 plane of nyx
 * weights.  FP32 arithmetic in the reference's operation order.  rounding: TIGRE_ROUND_NEAREST, or
 * TIGRE_ROUND_STOCHASTIC for 16-bit storage (Philox4x32-10 bits from (seed, step, voxel); FP32
 * storage ignores it). */
int tigre_sart_update(void* d_x, int dtype, const float* d_bp, const float* d_v, float lambda, int noneg,
                      long long nz, long long nyx, int rounding, unsigned long long seed, unsigned long long step,
                      void* stream);

/* Device noise (same generator as tigre_noise_1d); d_in and d_out may alias. */
int tigre_add_noise(const float* d_in, float* d_out, long long n, int gaussian, float mu, float sigma,
                    unsigned long long seed, void* stream);
/* Raw Philox4x32-10 blocks: d_out[4j..4j+3] = philox(counter = {j, counter_hi}, key = seed) for
 * j < nblocks (64-bit halves little-endian); d_out 16-byte aligned.  The generator behind the noise. */
int tigre_philox4x32(unsigned int* d_out, long long nblocks, unsigned long long counter_hi, unsigned long long seed,
                     void* stream);

/* 3x3x3 convolutions of the learned CGLS warm start (no reference counterpart): BF16
 * channels-last activations x[D][H][W][C], weights w[Cout][27*Cin] (tap (dz*3+dy)*3+dx major,
 * channel minor), zero padding 1, FP32 accumulation on the tensor cores.  d_col: scratch of
 * tigre_conv3d_col_elems(D, H, W, Cin) BF16 elements (d_dcol: as many floats). */
long long tigre_conv3d_col_elems(long D, long H, long W, long C);
/* Forward path of tigre_conv3d_fwd (and of the data gradient): 3 (default) the tcgen05 halo-tile
 * kernel -- one TMA load of a zero-padded input tile per 16 input channels, the 27 taps as
 * shifted shared-memory operand descriptors, TMEM accumulators -- wherever Cin % 16 == 0,
 * Cout % 16 == 0 (<= 192), W % 8 == 0 and H % 16 == 0, else mode 2; when Cin % 8 == 0 and
 * Cout % 16 == 0: 0 the warp-level implicit GEMM, 1 the tcgen05 implicit GEMM with per-step
 * gathers, 2 that kernel for narrow layers (Cin <= 16 or Cout == 16) and the warp-level one
 * otherwise.  Returns the old mode. */
int tigre_conv3d_set_tcgen05(int mode);
/* Synchronises the current device and returns the tensor-core convolution kernels' status word
 * (0 ok; TIGRE_STATUS_WAIT_EXPIRED: a bounded wait ran out and that output tile was not
 * written); reset != 0 clears it.  -1 if it cannot be read. */
int tigre_conv3d_status(int reset);
int tigre_conv3d_fwd(const void* d_x, const void* d_w, const float* d_bias, void* d_y_bf16, float* d_y_f32, long D,
                     long H, long W, long Cin, long Cout, int relu, void* d_col, void* stream);
int tigre_conv3d_bwd_data(const void* d_dy, const void* d_w, float* d_dx, long D, long H, long W, long Cin, long Cout,
                          float* d_dcol, void* stream);
int tigre_conv3d_bwd_weight(const void* d_x, const void* d_dy, float* d_dw, long D, long H, long W, long Cin,
                            long Cout, void* d_col, void* stream);

/* Fused steps of the warm-start U-Net's inference pass (no reference counterpart), BF16
 * channels-last activations with FP32 arithmetic; buffers 16-byte aligned.
 * pool2: y (D/2, H/2, W/2, C) = 2x2x2 mean of x (D, H, W, C); even sizes, C % 8 == 0.
 * up_concat: out (D, H, W, Ca + Cb) = [nearest 2x upsampling of low (D/2, H/2, W/2, Ca), skip].
 * conv_in: the first 3x3x3 convolution, one input channel: y (D, H, W, Cout) BF16 from the FP32
 *   volume rounded to BF16, weights w[Cout][27] BF16, bias FP32 (may be NULL), ReLU if relu;
 *   Cout 8, 16 or 32.
 * conv_out: the last 3x3x3 convolution, one output channel: out = vol + bf16(conv(x) + b) (FP32),
 *   weights w[27 Cin] BF16; Cin 8, 16 or 32. */
int tigre_unet_pool2(const void* d_x, void* d_y, long D, long H, long W, long C, void* stream);
int tigre_unet_up_concat(const void* d_low, long Ca, const void* d_skip, long Cb, void* d_out, long D, long H, long W,
                         void* stream);
int tigre_unet_conv_in(const float* d_vol, const void* d_w, const float* d_b, void* d_y, long D, long H, long W,
                       long Cout, int relu, void* stream);
int tigre_unet_conv_out(const void* d_x, long Cin, const void* d_w, float b, const float* d_vol, float* d_out, long D,
                        long H, long W, void* stream);

/* FP64 reductions and fused CGLS updates (device scalars, no host round trip). */
int tigre_sumsq(const void* d_x, int dtype, long n, double* d_out, void* stream);          /* *d_out += sum x^2 */
int tigre_dot(const float* d_x, const float* d_y, long n, double* d_out, void* stream);    /* *d_out += sum x*y */
/* x += a*p; r -= a*q; *d_rr += |r|^2, with a = (*d_num)/(*d_den). */
int tigre_cgls_step(float* d_x, const float* d_p, long nvol, float* d_r, const float* d_q, long nproj,
                    const double* d_num, const double* d_den, double* d_rr, void* stream);
/* p = s + (*d_num / *d_den) * p */
int tigre_cgls_direction(float* d_p, const float* d_s, long n, const double* d_num, const double* d_den,
                         void* stream);

/* Type conversion between storage types (for the reduced-precision paths). */
int tigre_convert(const void* d_src, int src_dtype, void* d_dst, int dst_dtype, long n, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* TIGRE_B200_H */
