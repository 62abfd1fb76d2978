// C++-linkage shims with the reference's exact signatures (see
// include/tigre_b200_compat.hpp), forwarding to the extern "C" entry points.
#include <cstdio>

#include "../../include/tigre_b200_compat.hpp"
#include "../../include/tigre_b200.h"

static_assert(sizeof(Geometry) == sizeof(TigreGeometry), "Geometry layout must match TigreGeometry");

namespace {
inline const TigreGeometry* as_c(const Geometry& g) { return reinterpret_cast<const TigreGeometry*>(&g); }
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
    if (rc) std::fprintf(stderr, "minimizeTV:POCS_TV: error %d: %s\n", rc, tigre_last_error());
}

void aw_pocs_tv(float* img, float* dst, float alpha, const long* image_size, int maxIter, const float delta,
                const GpuIds& ids) {
    const int rc = tigre_aw_pocs_tv(img, dst, alpha, image_size, maxIter, delta, ids.m_piDeviceIds, ids.m_iCount);
    if (rc) std::fprintf(stderr, "minimizeAwTV:GD_AwTV: error %d: %s\n", rc, tigre_last_error());
}

void piccs_tv(const float* img, const float* prior, float* dst, float alpha, float ratio, const long* image_size,
              int maxIter, const GpuIds& ids) {
    const int rc =
        tigre_piccs_tv(img, prior, dst, alpha, ratio, image_size, maxIter, ids.m_piDeviceIds, ids.m_iCount);
    if (rc) std::fprintf(stderr, "minimizeTV:PICCS_TV: error %d: %s\n", rc, tigre_last_error());
}

// RandomNumberGenerator.hpp: the reference seeds every call with 1234 (setup_kernel), so
// repeated calls on the same input give the same noise; so do these.
void poisson_1d(const float* pfIn, size_t uiLen, float* pfOut, const GpuIds& ids) {
    const int rc = tigre_noise_1d(pfIn, (long long)uiLen, 0, 0.f, 0.f, 1234ull, pfOut, ids.m_piDeviceIds, ids.m_iCount);
    if (rc) std::fprintf(stderr, "RandomNumberGenerator: poisson_1d error %d: %s\n", rc, tigre_last_error());
}

void poisson_gaussian_1d(const float* pfPoissonL, size_t uiLen, float fGaussMu, float fGaussSigma, float* pfOut,
                         GpuIds& ids) {
    const int rc = tigre_noise_1d(pfPoissonL, (long long)uiLen, 1, fGaussMu, fGaussSigma, 1234ull, pfOut,
                                  ids.m_piDeviceIds, ids.m_iCount);
    if (rc) std::fprintf(stderr, "RandomNumberGenerator: poisson_gaussian_1d error %d: %s\n", rc, tigre_last_error());
}

void tvdenoising(float* src, float* dst, float lambda, const float* spacing, const long* image_size, int maxIter,
                 const GpuIds& ids) {
    const int rc = tigre_tvdenoising(src, dst, lambda, spacing, image_size, maxIter, ids.m_piDeviceIds, ids.m_iCount);
    if (rc) std::fprintf(stderr, "tvdenoising failed with code %d: %s\n", rc, tigre_last_error());
}
