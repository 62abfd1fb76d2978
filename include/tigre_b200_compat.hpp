// tigre_b200_compat.hpp -- the reference's own C++ entry points, exported by
// libtigre_b200.so with the exact signatures (and therefore the same mangled
// symbols) that TIGRE's Cython extensions bind:
//
//   Common/CUDA/Siddon_projection.hpp:54          siddon_ray_projection
//   Common/CUDA/ray_interpolated_projection.hpp:55 interpolation_projection
//   Common/CUDA/voxel_backprojection.hpp:52       voxel_backprojection
//   Common/CUDA/voxel_backprojection2.hpp:57      voxel_backprojection2
//   Common/CUDA/GD_TV.hpp:58                      pocs_tv
//   Common/CUDA/GD_AwTV.hpp:58                    aw_pocs_tv
//   Common/CUDA/PICCS.hpp:58                      piccs_tv
//   Common/CUDA/tv_proximal.hpp:52                tvdenoising
//   Common/CUDA/RandomNumberGenerator.hpp         poisson_1d, poisson_gaussian_1d
//   and the *_parallel symbols referenced by _Ax.pyx:21-26 / _Atb.pyx:21-22.
//
// `Geometry` and `GpuIds` here are declared with the field layout of
// Common/CUDA/types_TIGRE.hpp:48-85 and Common/CUDA/GpuIds.hpp:2-14 (the
// library only reads GpuIds' two data members and defines none of its
// methods, so the extension's own GpuIds.cpp keeps providing them).
// Include either this header or the reference's headers, never both.
#ifndef TIGRE_B200_COMPAT_HPP
#define TIGRE_B200_COMPAT_HPP

#include <cstddef>

#ifndef TYPES_CBCT
#define TYPES_CBCT
struct Geometry {
    int nVoxelX, nVoxelY, nVoxelZ;
    float sVoxelX, sVoxelY, sVoxelZ;
    float dVoxelX, dVoxelY, dVoxelZ;
    float *offOrigX, *offOrigY, *offOrigZ;
    float* DSO;
    int nDetecU, nDetecV;
    float sDetecU, sDetecV;
    float dDetecU, dDetecV;
    float *offDetecU, *offDetecV;
    float* DSD;
    float* dRoll;
    float* dPitch;
    float* dYaw;
    float unitX, unitY, unitZ;
    float alpha, theta, psi;
    float* COR;
    float maxLength;
    float accuracy;
};
#endif

#ifndef GPUIDS_H
#define GPUIDS_H
struct GpuIds {
    int* m_piDeviceIds;
    int m_iCount;
};
#endif

int siddon_ray_projection(float* img, Geometry geo, float** result, float const* const angles, int nangles,
                          const GpuIds& gpuids);
int siddon_ray_projection_parallel(float* img, Geometry geo, float** result, float const* const angles, int nangles,
                                   const GpuIds& gpuids);
int interpolation_projection(float* img, Geometry geo, float** result, float const* const angles, int nangles,
                             const GpuIds& gpuids);
int interpolation_projection_parallel(float* img, Geometry geo, float** result, float const* const angles,
                                      int nangles, const GpuIds& gpuids);
int voxel_backprojection(float* projections, Geometry geo, float* result, float const* const alphas, int nalpha,
                         const GpuIds& gpuids);
int voxel_backprojection2(float* projections, Geometry geo, float* result, float const* const alphas, int nalpha,
                          const GpuIds& gpuids);
int voxel_backprojection_parallel(float* projections, Geometry geo, float* result, float const* const alphas,
                                  int nalpha, const GpuIds& gpuids);
// The reference returns void here (and exits the process on an error); these report an error
// on stderr and fill dst (pfOut) with NaN, so that a failure cannot pass for a result.
void pocs_tv(float* img, float* dst, float alpha, const long* image_size, int maxIter, const GpuIds& gpuids);
// Common/CUDA/RandomNumberGenerator.hpp: Poisson (+ Gaussian) noise, seed 1234 on every call.
void poisson_1d(const float* pfIn, size_t uiLen, float* pfOut, const GpuIds& gpuids);
void poisson_gaussian_1d(const float* pfPoissonL, size_t uiLen, float fGaussMu, float fGaussSigma, float* pfOut,
                         GpuIds& gpuids);
// Common/CUDA/GD_AwTV.hpp:58 and PICCS.hpp:58; void like the reference, errors on stderr, dst NaN.
void aw_pocs_tv(float* img, float* dst, float alpha, const long* image_size, int maxIter, const float delta,
                const GpuIds& gpuids);
void piccs_tv(const float* img, const float* prior, float* dst, float alpha, float ratio, const long* image_size,
              int maxIter, const GpuIds& gpuids);
// Common/CUDA/tv_proximal.hpp:52: TV denoising (im3ddenoise); void like the reference, errors on stderr, dst NaN.
void tvdenoising(float* src, float* dst, float lambda, const float* spacing, const long* image_size, int maxIter,
                const GpuIds& gpuids);

#endif  // TIGRE_B200_COMPAT_HPP
