// extern "C" shim over the reference's own C++ entry points.
//
// TEST INFRASTRUCTURE ONLY.  oracle/build.py (build_ref) compiles this file together
// with the reference's CUDA sources (read in place from the TIGRE tree, never
// copied) into oracle/_ref/libref_{ax,atb,tv}.so, grouped exactly as the
// reference's own Python extensions group them (setup.py:347-433).  The
// wrappers take a single device id and build the GpuIds object the reference
// expects (Common/CUDA/GpuIds.hpp).  The reference calls exit(1) on any CUDA
// error (Common/CUDA/TIGRE_common.cpp:13-16), so callers must load these
// libraries in a child process (oracle/ref.py does).

#include <cstdlib>
#include "types_TIGRE.hpp"
#include "GpuIds.hpp"

#if defined(REF_AX)
#include "Siddon_projection.hpp"
#include "Siddon_projection_parallel.hpp"
#include "ray_interpolated_projection.hpp"
#include "ray_interpolated_projection_parallel.hpp"
#elif defined(REF_ATB)
#include "voxel_backprojection.hpp"
#include "voxel_backprojection2.hpp"
#include "voxel_backprojection_parallel.hpp"
#elif defined(REF_TV)
#include "GD_TV.hpp"
#elif defined(REF_PROX)
#include "tv_proximal.hpp"
#elif defined(REF_AWTV)
#include "GD_AwTV.hpp"
#elif defined(REF_PICCS)
#include "PICCS.hpp"
#endif

namespace {
struct OneGpu {
    GpuIds ids;
    explicit OneGpu(int dev) { ids.SetIds(1, &dev); }
};
}  // namespace

extern "C" {

#if defined(REF_AX)
// projector: 0 = Siddon (siddon_ray_projection, Siddon_projection.cu:271),
//            1 = interpolated (interpolation_projection, ray_interpolated_projection.cu:211),
//            2 = parallel Siddon (siddon_ray_projection_parallel),
//            3 = parallel interpolated (interpolation_projection_parallel)
int ref_ax(float* img, const Geometry* geo, float* out, const float* angles, int nangles, int projector, int dev) {
    OneGpu g(dev);
    const size_t npix = (size_t)geo->nDetecU * (size_t)geo->nDetecV;
    float** rows = (float**)std::malloc(sizeof(float*) * (size_t)nangles);
    if (!rows) return 1;
    for (int i = 0; i < nangles; ++i) rows[i] = out + npix * (size_t)i;
    int rc = 1;
    switch (projector) {
        case 0: rc = siddon_ray_projection(img, *geo, rows, angles, nangles, g.ids); break;
        case 1: rc = interpolation_projection(img, *geo, rows, angles, nangles, g.ids); break;
        case 2: rc = siddon_ray_projection_parallel(img, *geo, rows, angles, nangles, g.ids); break;
        case 3: rc = interpolation_projection_parallel(img, *geo, rows, angles, nangles, g.ids); break;
    }
    std::free(rows);
    return rc;
}
#elif defined(REF_ATB)
// backprojector: 0 = FDK (voxel_backprojection, voxel_backprojection.cu:293),
//                1 = matched (voxel_backprojection2, voxel_backprojection2.cu:318),
//                2 = parallel (voxel_backprojection_parallel)
int ref_atb(float* proj, const Geometry* geo, float* out, const float* angles, int nangles, int backprojector,
            int dev) {
    OneGpu g(dev);
    if (backprojector == 2) return voxel_backprojection_parallel(proj, *geo, out, angles, nangles, g.ids);
    return backprojector == 0 ? voxel_backprojection(proj, *geo, out, angles, nangles, g.ids)
                              : voxel_backprojection2(proj, *geo, out, angles, nangles, g.ids);
}
#elif defined(REF_TV)
// pocs_tv (GD_TV.cu:255); image_size = {nX, nY, nZ}.  Note that the reference
// ends this call with cudaDeviceReset().
int ref_pocs_tv(float* img, float* dst, float alpha, const long* image_size, int maxiter, int dev) {
    OneGpu g(dev);
    pocs_tv(img, dst, alpha, image_size, maxiter, g.ids);
    return 0;
}
#elif defined(REF_PROX)
// tvdenoising (tv_proximal.cu:185) with unit spacing, as _tv_proximal.pyx:52-55 passes it.
int ref_tvdenoise(float* img, float* dst, float lambda, const long* image_size, int maxiter, int dev) {
    OneGpu g(dev);
    const float spacing[3] = {1.f, 1.f, 1.f};
    tvdenoising(img, dst, lambda, spacing, image_size, maxiter, g.ids);
    return 0;
}
#elif defined(REF_AWTV)
// aw_pocs_tv (GD_AwTV.cu:276); image_size = {nX, nY, nZ}.
int ref_aw_pocs_tv(float* img, float* dst, float alpha, const long* image_size, int maxiter, float delta, int dev) {
    OneGpu g(dev);
    aw_pocs_tv(img, dst, alpha, image_size, maxiter, delta, g.ids);
    return 0;
}
#elif defined(REF_PICCS)
// piccs_tv (PICCS.cu:274); image_size = {nX, nY, nZ}; ends with cudaDeviceReset().
int ref_piccs_tv(float* img, float* prior, float* dst, float alpha, float ratio, const long* image_size, int maxiter,
                 int dev) {
    OneGpu g(dev);
    piccs_tv(img, prior, dst, alpha, ratio, image_size, maxiter, g.ids);
    return 0;
}
#endif

}  // extern "C"
