// Public entry points of libtigre_b200 (include/tigre_b200.h).
//
// Device API: tigre_ax / tigre_atb run one projector on device buffers, on the
// caller's stream, with plan-owned scratch for the working layouts.
//
// Host API: the drop-in replacements of the reference's host-pointer functions
// (siddon_ray_projection & co.).  Same argument meaning; the volume or the
// projection stack is uploaded once, the work is pipelined in view chunks so
// that device->host copies of one chunk overlap the kernels of the next, and
// errors come back as return codes instead of exit(1).

#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <mutex>

#include "tigre_internal.h"

using namespace tigre;

namespace {

struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev) {
        cudaGetDevice(&prev);
        if (prev != dev) cudaSetDevice(dev);
    }
    ~DeviceGuard() {
        int cur = -1;
        cudaGetDevice(&cur);
        if (prev >= 0 && cur != prev) cudaSetDevice(prev);
    }
};

int check_range(const TigrePlan* p, int a0, int a1) {
    if (!p) return fail(TIGRE_ERR_BAD_ASSERT, "null plan");
    if (a0 < 0 || a1 > p->d.nA || a0 >= a1) return fail(TIGRE_ERR_BAD_ASSERT, "angle range outside the plan");
    return TIGRE_SUCCESS;
}

void layouts_needed(const TigrePlan* p, int a0, int a1, bool& l0, bool& l1) {
    l0 = l1 = false;
    for (int i = a0; i < a1; ++i) (p->h_siddon[i].layout ? l1 : l0) = true;
}

}  // namespace

extern "C" {

int tigre_ax(TigrePlan* plan, const void* d_vol, int vdt, void* d_proj, int pdt, int projector, int a0, int a1,
             void* stream) {
    if (int rc = check_range(plan, a0, a1)) return rc;
    if (!d_vol || !d_proj) return fail(TIGRE_ERR_BAD_ASSERT, "null device pointer");
    if (!dtype_ok(vdt) || !dtype_ok(pdt)) return fail(TIGRE_ERR_BAD_ASSERT, "unsupported dtype");
    DeviceGuard g(plan->device);
    cudaStream_t st = (cudaStream_t)stream;
    const Dims& d = plan->d;
    bool l0, l1;
    layouts_needed(plan, a0, a1, l0, l1);
    const size_t es = dtype_size(vdt);
    int rc = TIGRE_SUCCESS;
    if (projector == TIGRE_PROJ_SIDDON && plan->columns) {
        void* s = plan_scratch(plan, (size_t)d.nX * d.nY * (d.nZ + 2) * es, st, &rc);
        if (rc) return rc;
        if ((rc = launch_make_zfast(d_vol, vdt, s, d.nX, d.nY, d.nZ, st))) return rc;
        return launch_siddon_columns(plan, s, vdt, d_proj, pdt, a0, a1, st);
    }
    if (projector == TIGRE_PROJ_SIDDON) {
        const void* vx = d_vol;
        const void* vy = nullptr;
        if (l1) {
            void* s = plan_scratch(plan, (size_t)d.nX * d.nY * d.nZ * es, st, &rc);
            if (rc) return rc;
            if ((rc = launch_make_layout(d_vol, vdt, s, d.nX, d.nY, d.nZ, 1, 0, 0, st))) return rc;
            vy = s;
        }
        return launch_siddon(plan, vx, vy, vdt, d_proj, pdt, a0, a1, st);
    }
    if (projector == TIGRE_PROJ_INTERPOLATED) {
        const size_t padded = (size_t)(d.nX + 3) * (d.nY + 3) * (d.nZ + 3) * es;
        char* s = (char*)plan_scratch(plan, padded * 2, st, &rc);
        if (rc) return rc;
        void* vx = s;
        void* vy = s + padded;
        if (l0 && (rc = launch_make_layout(d_vol, vdt, vx, d.nX, d.nY, d.nZ, 0, 1, 2, st))) return rc;
        if (l1 && (rc = launch_make_layout(d_vol, vdt, vy, d.nX, d.nY, d.nZ, 1, 1, 2, st))) return rc;
        return launch_interp(plan, vx, vy, vdt, d_proj, pdt, a0, a1, st);
    }
    return fail(TIGRE_ERR_BAD_ASSERT, "unknown projector");
}

int tigre_atb(TigrePlan* plan, const void* d_proj, int pdt, void* d_vol, int vdt, int backprojector, int a0, int a1,
              void* stream) {
    if (int rc = check_range(plan, a0, a1)) return rc;
    if (!d_vol || !d_proj) return fail(TIGRE_ERR_BAD_ASSERT, "null device pointer");
    if (!dtype_ok(vdt) || !dtype_ok(pdt)) return fail(TIGRE_ERR_BAD_ASSERT, "unsupported dtype");
    if (backprojector != TIGRE_BACKPROJ_FDK && backprojector != TIGRE_BACKPROJ_MATCHED)
        return fail(TIGRE_ERR_BAD_ASSERT, "unknown backprojector");
    DeviceGuard g(plan->device);
    cudaStream_t st = (cudaStream_t)stream;
    const Dims& d = plan->d;
    const int na = a1 - a0;
    int rc = TIGRE_SUCCESS;
    if (bp_tma_supported(plan, pdt)) {
        const int align = 16 / (int)dtype_size(pdt);
        if (d.nU % align == 0 && ((uintptr_t)d_proj % 16) == 0)
            return launch_backproject_tma(plan, d_proj, d.nU, pdt, d_vol, vdt,
                                          backprojector == TIGRE_BACKPROJ_MATCHED, a0, a1, st);
        const int pitch = (d.nU + align - 1) / align * align;
        void* s = plan_scratch(plan, (size_t)na * d.nV * pitch * dtype_size(pdt), st, &rc);
        if (rc) return rc;
        if ((rc = launch_repitch_projections(d_proj, pdt, s, na, d.nV, d.nU, pitch, st))) return rc;
        return launch_backproject_tma(plan, s, pitch, pdt, d_vol, vdt, backprojector == TIGRE_BACKPROJ_MATCHED, a0,
                                      a1, st);
    }
    void* s = plan_scratch(plan, (size_t)na * bp_rows(d.nV) * bp_pitch(d.nU) * dtype_size(pdt), st, &rc);
    if (rc) return rc;
    if ((rc = launch_pad_projections(d_proj, pdt, s, na, d.nV, d.nU, st))) return rc;
    return launch_backproject(plan, s, pdt, d_vol, vdt, backprojector == TIGRE_BACKPROJ_MATCHED, a0, a1, st);
}

int tigre_siddon_count_segments(TigrePlan* plan, int a0, int a1, unsigned long long* d_total, void* stream) {
    if (int rc = check_range(plan, a0, a1)) return rc;
    if (!d_total) return fail(TIGRE_ERR_BAD_ASSERT, "null output");
    DeviceGuard g(plan->device);
    return launch_siddon_count(plan, a0, a1, d_total, (cudaStream_t)stream);
}

}  // extern "C"

// ---------------------------------------------------------------- host API --

namespace {

int pick_device(const int* ids, int n, int* dev) {
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0)
        return fail(TIGRE_ERR_NO_CAPABLE_DEVICES, "There are no available device(s) that support CUDA");
    *dev = (n > 0 && ids) ? ids[0] : 0;
    if (*dev < 0 || *dev >= count) return fail(TIGRE_ERR_NO_CAPABLE_DEVICES, "requested GPU id does not exist");
    return TIGRE_SUCCESS;
}

struct HostCall {
    TigrePlan* plan = nullptr;
    cudaStream_t st = nullptr, st2 = nullptr;
    cudaEvent_t ev[2] = {nullptr, nullptr};
    std::vector<void*> bufs;
    ~HostCall() {
        if (st) cudaStreamSynchronize(st);
        if (st2) cudaStreamSynchronize(st2);
        for (void* b : bufs) cudaFree(b);
        for (auto& e : ev)
            if (e) cudaEventDestroy(e);
        if (st) cudaStreamDestroy(st);
        if (st2) cudaStreamDestroy(st2);
        if (plan) tigre_plan_destroy(plan);
    }
    int alloc(void** p, size_t bytes) {
        cudaError_t e = cudaMalloc(p, bytes);
        if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc");
        bufs.push_back(*p);
        return TIGRE_SUCCESS;
    }
};

int host_project(const float* img, const TigreGeometry* geo, float* const* result, const float* angles, int nangles,
                 const int* ids, int n, int projector) {
    if (!img || !geo || !result || !angles) return fail(TIGRE_ERR_BAD_ASSERT, "null argument");
    int dev = 0;
    if (int rc = pick_device(ids, n, &dev)) return rc;
    DeviceGuard g(dev);
    HostCall h;
    if (int rc = tigre_plan_create(geo, angles, nangles, dev, &h.plan)) return rc;
    const Dims& d = h.plan->d;
    TIGRE_CUDA(cudaStreamCreateWithFlags(&h.st, cudaStreamNonBlocking));
    TIGRE_CUDA(cudaStreamCreateWithFlags(&h.st2, cudaStreamNonBlocking));
    for (auto& e : h.ev) TIGRE_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    const size_t nvox = (size_t)d.nX * d.nY * d.nZ, npix = (size_t)d.nU * d.nV;
    void* dvol = nullptr;
    if (int rc = h.alloc(&dvol, nvox * sizeof(float))) return rc;
    TIGRE_CUDA(cudaMemcpyAsync(dvol, img, nvox * sizeof(float), cudaMemcpyHostToDevice, h.st));
    // view chunks of ~128 MB, double-buffered
    const int chunk = (int)std::max<size_t>(1, std::min<size_t>(nangles, (128u << 20) / (npix * sizeof(float))));
    void* buf[2];
    for (auto& b : buf)
        if (int rc = h.alloc(&b, (size_t)chunk * npix * sizeof(float))) return rc;
    int prev_a = -1, prev_n = 0, k = 0;
    for (int a = 0; a < nangles; a += chunk, ++k) {
        const int cnt = std::min(chunk, nangles - a);
        // the copy stream must have drained this buffer (chunk k-2) before it is rewritten
        TIGRE_CUDA(cudaStreamWaitEvent(h.st, h.ev[k % 2], 0));
        if (int rc = tigre_ax(h.plan, dvol, TIGRE_F32, buf[k % 2], TIGRE_F32, projector, a, a + cnt, h.st)) return rc;
        if (prev_a >= 0) {
            const int pb = (k - 1) % 2;
            for (int i = 0; i < prev_n; ++i)
                TIGRE_CUDA(cudaMemcpyAsync(result[prev_a + i], (char*)buf[pb] + (size_t)i * npix * sizeof(float),
                                           npix * sizeof(float), cudaMemcpyDeviceToHost, h.st2));
            TIGRE_CUDA(cudaEventRecord(h.ev[pb], h.st2));
        }
        // copies of this chunk wait for its kernel
        cudaEvent_t done;
        TIGRE_CUDA(cudaEventCreateWithFlags(&done, cudaEventDisableTiming));
        cudaEventRecord(done, h.st);
        cudaStreamWaitEvent(h.st2, done, 0);
        cudaEventDestroy(done);
        prev_a = a;
        prev_n = cnt;
    }
    if (prev_a >= 0) {
        const int pb = (k - 1) % 2;
        for (int i = 0; i < prev_n; ++i)
            TIGRE_CUDA(cudaMemcpyAsync(result[prev_a + i], (char*)buf[pb] + (size_t)i * npix * sizeof(float),
                                       npix * sizeof(float), cudaMemcpyDeviceToHost, h.st2));
    }
    TIGRE_CUDA(cudaStreamSynchronize(h.st2));
    TIGRE_CUDA(cudaStreamSynchronize(h.st));
    return TIGRE_SUCCESS;
}

int host_backproject(const float* proj, const TigreGeometry* geo, float* result, const float* angles, int nangles,
                     const int* ids, int n, int matched) {
    if (!proj || !geo || !result || !angles) return fail(TIGRE_ERR_BAD_ASSERT, "null argument");
    int dev = 0;
    if (int rc = pick_device(ids, n, &dev)) return rc;
    DeviceGuard g(dev);
    HostCall h;
    if (int rc = tigre_plan_create(geo, angles, nangles, dev, &h.plan)) return rc;
    const Dims& d = h.plan->d;
    TIGRE_CUDA(cudaStreamCreateWithFlags(&h.st, cudaStreamNonBlocking));
    const size_t nvox = (size_t)d.nX * d.nY * d.nZ, nproj = (size_t)nangles * d.nU * d.nV;
    void *dvol = nullptr, *dproj = nullptr;
    if (int rc = h.alloc(&dvol, nvox * sizeof(float))) return rc;
    if (int rc = h.alloc(&dproj, nproj * sizeof(float))) return rc;
    TIGRE_CUDA(cudaMemcpyAsync(dproj, proj, nproj * sizeof(float), cudaMemcpyHostToDevice, h.st));
    if (int rc = tigre_atb(h.plan, dproj, TIGRE_F32, dvol, TIGRE_F32,
                           matched ? TIGRE_BACKPROJ_MATCHED : TIGRE_BACKPROJ_FDK, 0, nangles, h.st))
        return rc;
    TIGRE_CUDA(cudaMemcpyAsync(result, dvol, nvox * sizeof(float), cudaMemcpyDeviceToHost, h.st));
    TIGRE_CUDA(cudaStreamSynchronize(h.st));
    if (tigre_plan_status(h.plan, 1) != 0) return fail(TIGRE_ERR_CUDA, "backprojection: a bounded wait expired");
    return TIGRE_SUCCESS;
}

}  // namespace

extern "C" {

int tigre_siddon_ray_projection(const float* img, const TigreGeometry* geo, float* const* result, const float* angles,
                                int nangles, const int* ids, int n) {
    return host_project(img, geo, result, angles, nangles, ids, n, TIGRE_PROJ_SIDDON);
}

int tigre_interpolation_projection(const float* img, const TigreGeometry* geo, float* const* result,
                                   const float* angles, int nangles, const int* ids, int n) {
    return host_project(img, geo, result, angles, nangles, ids, n, TIGRE_PROJ_INTERPOLATED);
}

int tigre_voxel_backprojection(const float* proj, const TigreGeometry* geo, float* result, const float* angles,
                               int nangles, const int* ids, int n) {
    return host_backproject(proj, geo, result, angles, nangles, ids, n, 0);
}

int tigre_voxel_backprojection2(const float* proj, const TigreGeometry* geo, float* result, const float* angles,
                                int nangles, const int* ids, int n) {
    return host_backproject(proj, geo, result, angles, nangles, ids, n, 1);
}

int tigre_pocs_tv(const float* img, float* dst, float alpha, const long* image_size, int max_iter, const int* ids,
                  int n) {
    if (!img || !dst || !image_size) return fail(TIGRE_ERR_BAD_ASSERT, "null argument");
    const long nx = image_size[0], ny = image_size[1], nz = image_size[2];
    if (nx <= 0 || ny <= 0 || nz <= 0) return fail(TIGRE_ERR_BAD_ASSERT, "bad image size");
    int dev = 0;
    if (int rc = pick_device(ids, n, &dev)) return rc;
    DeviceGuard g(dev);
    HostCall h;
    TIGRE_CUDA(cudaStreamCreateWithFlags(&h.st, cudaStreamNonBlocking));
    const size_t nvox = (size_t)nx * ny * nz;
    void *dimg = nullptr, *dwork = nullptr;
    if (int rc = h.alloc(&dimg, nvox * sizeof(float))) return rc;
    if (int rc = h.alloc(&dwork, nvox * sizeof(float))) return rc;
    TIGRE_CUDA(cudaMemcpyAsync(dimg, img, nvox * sizeof(float), cudaMemcpyHostToDevice, h.st));
    if (int rc = tigre_tv_pocs(dimg, TIGRE_F32, nx, ny, nz, alpha, max_iter, (float*)dwork, h.st)) return rc;
    TIGRE_CUDA(cudaMemcpyAsync(dst, dimg, nvox * sizeof(float), cudaMemcpyDeviceToHost, h.st));
    TIGRE_CUDA(cudaStreamSynchronize(h.st));
    return TIGRE_SUCCESS;
}

int tigre_siddon_ray_projection_parallel(const float*, const TigreGeometry*, float* const*, const float*, int,
                                         const int*, int) {
    return fail(TIGRE_ERR_BAD_ASSERT, "parallel-beam projection is not provided by libtigre_b200");
}

int tigre_interpolation_projection_parallel(const float*, const TigreGeometry*, float* const*, const float*, int,
                                            const int*, int) {
    return fail(TIGRE_ERR_BAD_ASSERT, "parallel-beam projection is not provided by libtigre_b200");
}

int tigre_voxel_backprojection_parallel(const float*, const TigreGeometry*, float*, const float*, int, const int*,
                                        int) {
    return fail(TIGRE_ERR_BAD_ASSERT, "parallel-beam backprojection is not provided by libtigre_b200");
}

}  // extern "C"
