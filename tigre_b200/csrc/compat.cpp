// C++-linkage shims with the reference's exact signatures (see
// include/tigre_b200_compat.hpp), forwarding to the extern "C" entry points.
#include <cmath>
#include <cstdio>

#include "../../include/tigre_b200_compat.hpp"
#include "../../include/tigre_b200.h"

static_assert(sizeof(Geometry) == sizeof(TigreGeometry), "Geometry layout must match TigreGeometry");

namespace {
inline const TigreGeometry* as_c(const Geometry& g) { return reinterpret_cast<const TigreGeometry*>(&g); }

// The reference's void entry points have no error return (it exits the process instead,
// TIGRE_common.cpp:13-16).  Here a failure is printed and the output is filled with NaN, so
// that it cannot come back to the caller as plausible data.
void poison(float* dst, long long n) {
    if (!dst) return;
    for (long long i = 0; i < n; ++i) dst[i] = NAN;
}
long long volume(const long* image_size) {
    return image_size ? (long long)image_size[0] * image_size[1] * image_size[2] : 0;
}
}  // namespace

int siddon_ray_projection(float* img, Geometry geo, float** result, float const* const angles, int nangles,
                          const GpuIds& ids) {
    return tigre_siddon_ray_projection(img, as_c(geo), result, angles, nangles, ids.m_piDeviceIds, ids.m_iCount);
}

int siddon_ray_projection_parallel(float* img, Geometry geo, float** result, float const* const angles, int nangles,
                                   const GpuIds& ids) {
    return tigre_siddon_ray_projection_parallel(img, as_c(geo), result, angles, nangles, ids.m_piDeviceIds,
                                                ids.m_iCount);
}

int interpolation_projection(float* img, Geometry geo, float** result, float const* const angles, int nangles,
                             const GpuIds& ids) {
    return tigre_interpolation_projection(img, as_c(geo), result, angles, nangles, ids.m_piDeviceIds, ids.m_iCount);
}

int interpolation_projection_parallel(float* img, Geometry geo, float** result, float const* const angles,
                                      int nangles, const GpuIds& ids) {
    return tigre_interpolation_projection_parallel(img, as_c(geo), result, angles, nangles, ids.m_piDeviceIds,
                                                   ids.m_iCount);
}

int voxel_backprojection(float* projections, Geometry geo, float* result, float const* const alphas, int nalpha,
                         const GpuIds& ids) {
    return tigre_voxel_backprojection(projections, as_c(geo), result, alphas, nalpha, ids.m_piDeviceIds,
                                      ids.m_iCount);
}

int voxel_backprojection2(float* projections, Geometry geo, float* result, float const* const alphas, int nalpha,
                          const GpuIds& ids) {
    return tigre_voxel_backprojection2(projections, as_c(geo), result, alphas, nalpha, ids.m_piDeviceIds,
                                       ids.m_iCount);
}

int voxel_backprojection_parallel(float* projections, Geometry geo, float* result, float const* const alphas,
                                  int nalpha, const GpuIds& ids) {
    return tigre_voxel_backprojection_parallel(projections, as_c(geo), result, alphas, nalpha, ids.m_piDeviceIds,
                                               ids.m_iCount);
}

void pocs_tv(float* img, float* dst, float alpha, const long* image_size, int maxIter, const GpuIds& ids) {
    const int rc = tigre_pocs_tv(img, dst, alpha, image_size, maxIter, ids.m_piDeviceIds, ids.m_iCount);
    if (rc) {
        std::fprintf(stderr, "minimizeTV:POCS_TV: error %d: %s\n", rc, tigre_last_error());
        poison(dst, volume(image_size));
    }
}

void aw_pocs_tv(float* img, float* dst, float alpha, const long* image_size, int maxIter, const float delta,
                const GpuIds& ids) {
    const int rc = tigre_aw_pocs_tv(img, dst, alpha, image_size, maxIter, delta, ids.m_piDeviceIds, ids.m_iCount);
    if (rc) {
        std::fprintf(stderr, "minimizeAwTV:GD_AwTV: error %d: %s\n", rc, tigre_last_error());
        poison(dst, volume(image_size));
    }
}

void piccs_tv(const float* img, const float* prior, float* dst, float alpha, float ratio, const long* image_size,
              int maxIter, const GpuIds& ids) {
    const int rc =
        tigre_piccs_tv(img, prior, dst, alpha, ratio, image_size, maxIter, ids.m_piDeviceIds, ids.m_iCount);
    if (rc) {
        std::fprintf(stderr, "minimizeTV:PICCS_TV: error %d: %s\n", rc, tigre_last_error());
        poison(dst, volume(image_size));
    }
}

// RandomNumberGenerator.hpp: the reference seeds every call with 1234 (setup_kernel), so
// repeated calls on the same input give the same noise; so do these.
void poisson_1d(const float* pfIn, size_t uiLen, float* pfOut, const GpuIds& ids) {
    const int rc = tigre_noise_1d(pfIn, (long long)uiLen, 0, 0.f, 0.f, 1234ull, pfOut, ids.m_piDeviceIds, ids.m_iCount);
    if (rc) {
        std::fprintf(stderr, "RandomNumberGenerator: poisson_1d error %d: %s\n", rc, tigre_last_error());
        poison(pfOut, (long long)uiLen);
    }
}

void poisson_gaussian_1d(const float* pfPoissonL, size_t uiLen, float fGaussMu, float fGaussSigma, float* pfOut,
                         GpuIds& ids) {
    const int rc = tigre_noise_1d(pfPoissonL, (long long)uiLen, 1, fGaussMu, fGaussSigma, 1234ull, pfOut,
                                  ids.m_piDeviceIds, ids.m_iCount);
    if (rc) {
        std::fprintf(stderr, "RandomNumberGenerator: poisson_gaussian_1d error %d: %s\n", rc, tigre_last_error());
        poison(pfOut, (long long)uiLen);
    }
}

void tvdenoising(float* src, float* dst, float lambda, const float* spacing, const long* image_size, int maxIter,
                 const GpuIds& ids) {
    const int rc = tigre_tvdenoising(src, dst, lambda, spacing, image_size, maxIter, ids.m_piDeviceIds, ids.m_iCount);
    if (rc) {
        std::fprintf(stderr, "tvdenoising failed with code %d: %s\n", rc, tigre_last_error());
        poison(dst, volume(image_size));
    }
}
