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
#include <thread>
#include <vector>

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

// Working copies of the volume that the forward projectors read, built once for a range of
// views and reused by every launch over sub-ranges of it (the host pipeline projects in view
// chunks).  Lives in the plan's scratch until the next plan_scratch call.
struct AxWork {
    enum Mode { CELLS, COLUMNS, GENERAL, INTERP, INTERP_TEX } mode = GENERAL;
    unsigned long long tex = 0;   // INTERP_TEX: texture object over the plan's 3-D array
    const void* vx = nullptr;
    const void* vy = nullptr;
    const void* qx = nullptr;
    const void* qy = nullptr;
    int vdt = TIGRE_F32;   // element type the kernels read
};

int ax_prepare(TigrePlan* plan, const void* d_vol, int vdt, int projector, int a0, int a1, cudaStream_t st,
               AxWork* w) {
    const Dims& d = plan->d;
    bool l0, l1;
    layouts_needed(plan, a0, a1, l0, l1);
    const size_t es = dtype_size(vdt);
    int rc = TIGRE_SUCCESS;
    w->vdt = vdt;
    if (projector == TIGRE_PROJ_SIDDON && plan->columns) {
        // z-fast working copy; the cell-interval kernel needs deeper zero pads
        const int zpad = plan->cells_zpad > 0 ? plan->cells_zpad : 1;
        if (plan->cells_zpad > 0 && vdt != TIGRE_F32) {
            // 16-bit storage: the working copy is built in FP32 (exact), so the cell kernel runs
            // its FP32 form and gives the same sums as on a widened volume
            float* sf = (float*)plan_scratch(plan, (size_t)d.nX * d.nY * (d.nZ + 2 * zpad) * sizeof(float), st, &rc);
            if (rc) return rc;
            if ((rc = launch_make_zfast_f32(d_vol, vdt, sf, d.nX, d.nY, d.nZ, zpad, st))) return rc;
            w->mode = AxWork::CELLS;
            w->vx = sf;
            w->vdt = TIGRE_F32;
            return TIGRE_SUCCESS;
        }
        void* s = plan_scratch(plan, (size_t)d.nX * d.nY * (d.nZ + 2 * zpad) * es, st, &rc);
        if (rc) return rc;
        if ((rc = launch_make_zfast(d_vol, vdt, s, d.nX, d.nY, d.nZ, zpad, st))) return rc;
        w->mode = plan->cells_zpad > 0 ? AxWork::CELLS : AxWork::COLUMNS;
        w->vx = s;
        return TIGRE_SUCCESS;
    }
    if (projector == TIGRE_PROJ_SIDDON) {
        w->mode = AxWork::GENERAL;
        w->vx = d_vol;
        if (l1) {
            void* s = plan_scratch(plan, (size_t)d.nX * d.nY * d.nZ * es, st, &rc);
            if (rc) return rc;
            if ((rc = launch_make_layout(d_vol, vdt, s, d.nX, d.nY, d.nZ, 1, 0, 0, st))) return rc;
            w->vy = s;
        }
        return TIGRE_SUCCESS;
    }
    if (projector == TIGRE_PROJ_INTERPOLATED && option(TIGRE_OPT_INTERP_TEXTURE) && d.accuracy <= 1.0) {
        // hardware trilinear: the volume goes into the plan's FP32 3-D array (16-bit storage is
        // widened first, exactly)
        const float* vf = (const float*)d_vol;
        if (vdt != TIGRE_F32) {
            float* s = (float*)plan_scratch(plan, (size_t)d.nX * d.nY * d.nZ * sizeof(float), st, &rc);
            if (rc) return rc;
            if ((rc = tigre_convert(d_vol, vdt, s, TIGRE_F32, (long)d.nX * d.nY * d.nZ, st))) return rc;
            vf = s;
        }
        w->mode = AxWork::INTERP_TEX;
        return interp_texture(plan, vf, st, &w->tex);
    }
    if (projector == TIGRE_PROJ_INTERPOLATED) {
        // zero-padded copies (1 before, 2 after), x- and/or y-fastest; trilinear sampling reads
        // corner quads built from them (4 values per element), point sampling the copies
        // (offsets rounded to 256 bytes: the quads are read as 8- or 16-byte vectors)
        w->mode = AxWork::INTERP;
        const size_t padded = ((size_t)(d.nX + 3) * (d.nY + 3) * (d.nZ + 3) * es + 255) / 256 * 256;
        const bool nearest = d.accuracy > 1.0;
        if (!nearest && vdt != TIGRE_F32) {
            // 16-bit storage: FP32 corner quads (exact widening) for the FP32 sampling kernel
            const size_t pf = ((size_t)(d.nX + 3) * (d.nY + 3) * (d.nZ + 3) * sizeof(float) + 255) / 256 * 256;
            char* s = (char*)plan_scratch(plan, padded + 8 * pf, st, &rc);
            if (rc) return rc;
            void* vx = s;
            float* qx = (float*)(s + padded);
            float* qy = (float*)(s + padded + 4 * pf);
            for (int l = 0; l < 2; ++l) {
                if (!(l ? l1 : l0)) continue;
                if ((rc = launch_make_layout(d_vol, vdt, vx, d.nX, d.nY, d.nZ, l, 1, 2, st))) return rc;
                if ((rc = launch_make_quads_f32(vx, vdt, l ? qy : qx, d.nX, d.nY, d.nZ, l, st))) return rc;
            }
            w->qx = qx;
            w->qy = qy;
            w->vdt = TIGRE_F32;
            return TIGRE_SUCCESS;
        }
        char* s = (char*)plan_scratch(plan, padded * (nearest ? 2 : 9), st, &rc);
        if (rc) return rc;
        void* vx = s;
        void* vy = s + padded;
        void* qx = nearest ? nullptr : s + padded;
        void* qy = nearest ? nullptr : s + 5 * padded;
        if (nearest) {
            if (l0 && (rc = launch_make_layout(d_vol, vdt, vx, d.nX, d.nY, d.nZ, 0, 1, 2, st))) return rc;
            if (l1 && (rc = launch_make_layout(d_vol, vdt, vy, d.nX, d.nY, d.nZ, 1, 1, 2, st))) return rc;
        } else {
            for (int l = 0; l < 2; ++l) {
                if (!(l ? l1 : l0)) continue;
                if ((rc = launch_make_layout(d_vol, vdt, vx, d.nX, d.nY, d.nZ, l, 1, 2, st))) return rc;
                if ((rc = launch_make_quads(vx, vdt, l ? qy : qx, d.nX, d.nY, d.nZ, l, st))) return rc;
            }
        }
        w->vx = vx;
        w->vy = vy;
        w->qx = qx;
        w->qy = qy;
        return TIGRE_SUCCESS;
    }
    return fail(TIGRE_ERR_BAD_ASSERT, "unknown projector");
}

int ax_launch(TigrePlan* plan, const AxWork& w, void* d_proj, int pdt, int a0, int a1, cudaStream_t st) {
    switch (w.mode) {
        case AxWork::CELLS: return launch_siddon_cells(plan, w.vx, w.vdt, d_proj, pdt, a0, a1, st);
        case AxWork::COLUMNS: return launch_siddon_columns(plan, w.vx, w.vdt, d_proj, pdt, a0, a1, st);
        case AxWork::GENERAL: return launch_siddon(plan, w.vx, w.vy, w.vdt, d_proj, pdt, a0, a1, st);
        case AxWork::INTERP_TEX: return launch_interp_tex(plan, w.tex, d_proj, pdt, a0, a1, st);
        default: return launch_interp(plan, w.vx, w.vy, w.qx, w.qy, w.vdt, d_proj, pdt, a0, a1, st);
    }
}

}  // namespace

extern "C" {

int tigre_ax(TigrePlan* plan, const void* d_vol, int vdt, void* d_proj, int pdt, int projector, int a0, int a1,
             void* stream) {
    TIGRE_NVTX("tigre_ax");
    if (int rc = check_range(plan, a0, a1)) return rc;
    if (!d_vol || !d_proj) return fail(TIGRE_ERR_BAD_ASSERT, "null device pointer");
    if (!dtype_ok(vdt) || !dtype_ok(pdt)) return fail(TIGRE_ERR_BAD_ASSERT, "unsupported dtype");
    DeviceGuard g(plan->device);
    cudaStream_t st = (cudaStream_t)stream;
    AxWork w;
    if (int rc = ax_prepare(plan, d_vol, vdt, projector, a0, a1, st, &w)) return rc;
    return ax_launch(plan, w, d_proj, pdt, a0, a1, st);
}

int tigre_atb(TigrePlan* plan, const void* d_proj, int pdt, void* d_vol, int vdt, int backprojector, int a0, int a1,
              void* stream) {
    return tigre_atb_ex(plan, d_proj, pdt, d_vol, vdt, backprojector, a0, a1, 0, stream);
}

int tigre_atb_ex(TigrePlan* plan, const void* d_proj, int pdt, void* d_vol, int vdt, int backprojector, int a0, int a1,
                 int accumulate, void* stream) {
    TIGRE_NVTX("tigre_atb");
    if (int rc = check_range(plan, a0, a1)) return rc;
    if (!d_vol || !d_proj) return fail(TIGRE_ERR_BAD_ASSERT, "null device pointer");
    if (!dtype_ok(vdt) || !dtype_ok(pdt)) return fail(TIGRE_ERR_BAD_ASSERT, "unsupported dtype");
    if (backprojector != TIGRE_BACKPROJ_FDK && backprojector != TIGRE_BACKPROJ_MATCHED)
        return fail(TIGRE_ERR_BAD_ASSERT, "unknown backprojector");
    // parallel beam has one backprojector (voxel_backprojection_parallel); its frames are
    // encoded for the FDK path (unit weight, no scale)
    if (plan->parallel) backprojector = TIGRE_BACKPROJ_FDK;
    DeviceGuard g(plan->device);
    cudaStream_t st = (cudaStream_t)stream;
    const Dims& d = plan->d;
    const int na = a1 - a0;
    int rc = TIGRE_SUCCESS;
    if (pdt != TIGRE_F32 && (vdt == TIGRE_F32 || vdt == TIGRE_BF16) && bp_tma_supported(plan, TIGRE_F32)) {
        // 16-bit projections: widened to FP32 (exact) into a pitched copy, then the FP32 patches
        const int pitch = (d.nU + 3) / 4 * 4;
        float* s = (float*)plan_scratch(plan, (size_t)na * d.nV * pitch * sizeof(float), st, &rc);
        if (rc) return rc;
        if ((rc = launch_repitch_projections_f32(d_proj, pdt, s, na, d.nV, d.nU, pitch, st))) return rc;
        return launch_backproject_tma(plan, s, pitch, TIGRE_F32, d_vol, vdt, backprojector == TIGRE_BACKPROJ_MATCHED,
                                      a0, a1, accumulate, st);
    }
    if (bp_tma_supported(plan, pdt)) {
        const int align = 16 / (int)dtype_size(pdt);
        if (d.nU % align == 0 && ((uintptr_t)d_proj % 16) == 0)
            return launch_backproject_tma(plan, d_proj, d.nU, pdt, d_vol, vdt,
                                          backprojector == TIGRE_BACKPROJ_MATCHED, a0, a1, accumulate, st);
        const int pitch = (d.nU + align - 1) / align * align;
        void* s = plan_scratch(plan, (size_t)na * d.nV * pitch * dtype_size(pdt), st, &rc);
        if (rc) return rc;
        if ((rc = launch_repitch_projections(d_proj, pdt, s, na, d.nV, d.nU, pitch, st))) return rc;
        return launch_backproject_tma(plan, s, pitch, pdt, d_vol, vdt, backprojector == TIGRE_BACKPROJ_MATCHED, a0,
                                      a1, accumulate, st);
    }
    void* s = plan_scratch(plan, (size_t)na * bp_rows(d.nV) * bp_pitch(d.nU) * dtype_size(pdt), st, &rc);
    if (rc) return rc;
    if ((rc = launch_pad_projections(d_proj, pdt, s, na, d.nV, d.nU, st))) return rc;
    return launch_backproject(plan, s, pdt, d_vol, vdt, backprojector == TIGRE_BACKPROJ_MATCHED, a0, a1, accumulate,
                              st);
}

int tigre_siddon_count_segments(TigrePlan* plan, int a0, int a1, unsigned long long* d_total, void* stream) {
    if (int rc = check_range(plan, a0, a1)) return rc;
    if (!d_total) return fail(TIGRE_ERR_BAD_ASSERT, "null output");
    DeviceGuard g(plan->device);
    return launch_siddon_count(plan, a0, a1, d_total, (cudaStream_t)stream);
}

int tigre_interp_count_samples(TigrePlan* plan, int a0, int a1, unsigned long long* d_total, void* stream) {
    if (int rc = check_range(plan, a0, a1)) return rc;
    if (!d_total) return fail(TIGRE_ERR_BAD_ASSERT, "null output");
    DeviceGuard g(plan->device);
    return launch_interp_count(plan, a0, a1, d_total, (cudaStream_t)stream);
}

}  // extern "C"

// ---------------------------------------------------------------- host API --
//
// Per device, the host entry points keep (a) the plans of the last few
// geometries, keyed by the bytes of the geometry and the angles, and (b) a
// small set of device buffers that only grow, so repeated calls on the same
// geometry allocate nothing and recompute no frames.  Calls on one device are
// serialised (the reference's host functions are not reentrant either).

namespace {

int pick_device(const int* ids, int n, int* dev) {
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0)
        return fail(TIGRE_ERR_NO_CAPABLE_DEVICES, "There are no available device(s) that support CUDA");
    *dev = (n > 0 && ids) ? ids[0] : 0;
    if (*dev < 0 || *dev >= count) return fail(TIGRE_ERR_NO_CAPABLE_DEVICES, "requested GPU id does not exist");
    return TIGRE_SUCCESS;
}

uint64_t fnv(uint64_t h, const void* p, size_t n) {
    const unsigned char* c = (const unsigned char*)p;
    for (size_t i = 0; i < n; ++i) h = (h ^ c[i]) * 1099511628211ull;
    return h;
}

uint64_t geometry_key(const TigreGeometry* g, const float* angles, int n) {
    uint64_t h = 1469598103934665603ull;
    TigreGeometry s = *g;
    const float* arrays[] = {g->offOrigX, g->offOrigY, g->offOrigZ, g->DSO, g->offDetecU, g->offDetecV,
                             g->DSD, g->dRoll, g->dPitch, g->dYaw, g->COR};
    s.offOrigX = s.offOrigY = s.offOrigZ = s.DSO = s.offDetecU = s.offDetecV = s.DSD = nullptr;
    s.dRoll = s.dPitch = s.dYaw = s.COR = nullptr;
    h = fnv(h, &s, sizeof(s));
    for (const float* a : arrays) {
        const unsigned char present = a != nullptr;
        h = fnv(h, &present, 1);
        if (a) h = fnv(h, a, sizeof(float) * (size_t)n);
    }
    h = fnv(h, angles, sizeof(float) * 3 * (size_t)n);
    return fnv(h, &n, sizeof(n));
}

struct DeviceState {
    std::mutex mu;
    cudaStream_t st = nullptr, st2 = nullptr;
    cudaEvent_t ev[4] = {};
    // pinned bounce buffers for large copies of pageable host memory (staged_h2d / staged_d2h)
    void* pin[2] = {};
    cudaEvent_t pin_ev[2] = {};
    void* buf[4] = {};
    size_t bytes[4] = {};
    struct Entry { uint64_t key; TigrePlan* plan; };
    std::vector<Entry> plans;

    int init(int dev) {
        if (st) return TIGRE_SUCCESS;
        TIGRE_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
        TIGRE_CUDA(cudaStreamCreateWithFlags(&st2, cudaStreamNonBlocking));
        for (auto& e : ev) TIGRE_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        for (auto& e : pin_ev) TIGRE_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        (void)dev;
        return TIGRE_SUCCESS;
    }
    int get(int slot, size_t n, void** out) {
        if (bytes[slot] < n) {
            if (buf[slot]) {
                cudaStreamSynchronize(st);
                cudaStreamSynchronize(st2);
                cudaFree(buf[slot]);
                buf[slot] = nullptr;
                bytes[slot] = 0;
            }
            TIGRE_CUDA(cudaMalloc(&buf[slot], n));
            bytes[slot] = n;
        }
        *out = buf[slot];
        return TIGRE_SUCCESS;
    }
    int plan(const TigreGeometry* g, const float* angles, int n, int dev, int flags, TigrePlan** out) {
        const uint64_t k = fnv(geometry_key(g, angles, n), &flags, sizeof(flags));
        for (auto& e : plans)
            if (e.key == k) { *out = e.plan; return TIGRE_SUCCESS; }
        TigrePlan* p = nullptr;
        if (int rc = tigre_plan_create_ex(g, angles, n, dev, flags, &p)) return rc;
        if (plans.size() >= 4) {
            cudaStreamSynchronize(st);
            tigre_plan_destroy(plans.front().plan);
            plans.erase(plans.begin());
        }
        plans.push_back({k, p});
        *out = p;
        return TIGRE_SUCCESS;
    }
    void release() {
        if (st) { cudaStreamSynchronize(st); cudaStreamSynchronize(st2); }
        for (auto& e : plans) tigre_plan_destroy(e.plan);
        plans.clear();
        for (int i = 0; i < 4; ++i) {
            if (buf[i]) cudaFree(buf[i]);
            buf[i] = nullptr;
            bytes[i] = 0;
        }
        for (auto& p : pin) {
            if (p) cudaFreeHost(p);
            p = nullptr;
        }
    }
};

std::mutex g_states_mu;
std::vector<DeviceState*> g_states;

// ---- host <-> device copies of pageable memory ----
// An upload from pageable memory goes through the driver's own small staging buffers at a
// fraction of the link's bandwidth.  Pageable uploads of at least kStageMin bytes instead go
// through two pinned bounce buffers of kStageBytes: up to kStageThreads host threads copy chunk
// k into one while the copy engine moves chunk k - 1 through the other.  Page-locked caller
// buffers keep the direct path.
constexpr size_t kStageBytes = (size_t)64 << 20;
constexpr size_t kStageMin = (size_t)32 << 20;
constexpr unsigned kStageThreads = 16;

// which (bit mask, option TIGRE_OPT_HOST_STAGING, default kStageDefault): 1 uploads of a volume, 2 downloads
// of a volume, 4 the backprojector's projection-chunk uploads, 8 the backprojector's volume
// download.  Page-locked caller buffers always take the direct path.  Measured at 512^3 on B200
// (host call): the POCS-TV call takes 175 ms direct, 146 ms with staged uploads and 62 ms with
// staged uploads and downloads; the Siddon Ax call 260 ms direct and 231 ms with its volume upload
// staged; the matched Atb call on pageable projections 229 ms through the driver's pageable path.
constexpr int kStageDefault = 1 | 2 | 4 | 8;
bool staging_on(int which) {
    const long long o = option(TIGRE_OPT_HOST_STAGING);
    const long long mask = o >= 0 ? o : kStageDefault;
    return (mask & which) != 0;
}

void par_memcpy(void* dst, const void* src, size_t n) {
    const unsigned T = std::max(1u, std::min(kStageThreads, std::thread::hardware_concurrency()));
    if (T == 1 || n < ((size_t)4 << 20)) {
        memcpy(dst, src, n);
        return;
    }
    const size_t per = ((n + T - 1) / T + 4095) & ~(size_t)4095;
    std::vector<std::thread> pool;
    for (unsigned t = 1; t < T; ++t) {
        const size_t a = (size_t)t * per;
        if (a >= n) break;
        try {
            pool.emplace_back([=] { memcpy((char*)dst + a, (const char*)src + a, std::min(per, n - a)); });
        } catch (...) {   // no thread (resource limits): the calling thread copies the rest
            memcpy((char*)dst + a, (const char*)src + a, n - a);
            break;
        }
    }
    memcpy(dst, src, std::min(per, n));
    for (auto& th : pool) th.join();
}

// true when p is page-locked host memory (cudaHostAlloc / cudaHostRegister): the copy engine
// reads and writes it directly, so a bounce buffer would only add a host copy
bool host_pinned(const void* p) {
    cudaPointerAttributes a{};
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeHost;
}

int ensure_pinned(DeviceState* S) {
    for (auto& p : S->pin)
        if (!p) TIGRE_CUDA(cudaMallocHost(&p, kStageBytes));
    return TIGRE_SUCCESS;
}

// h_src (pageable) -> d_dst on stream st; returns once h_src may be reused
int staged_h2d(DeviceState* S, void* d_dst, const void* h_src, size_t n, cudaStream_t st, int which = 1) {
    if (n < kStageMin || !staging_on(which) || host_pinned(h_src)) {
        TIGRE_CUDA(cudaMemcpyAsync(d_dst, h_src, n, cudaMemcpyHostToDevice, st));
        return TIGRE_SUCCESS;
    }
    if (int rc = ensure_pinned(S)) return rc;
    size_t c = 0;
    for (size_t off = 0; off < n; off += kStageBytes, ++c) {
        const int b = (int)(c & 1);
        const size_t m = std::min(kStageBytes, n - off);
        TIGRE_CUDA(cudaEventSynchronize(S->pin_ev[b]));   // the copy that last read pin[b] is done
        par_memcpy(S->pin[b], (const char*)h_src + off, m);
        TIGRE_CUDA(cudaMemcpyAsync((char*)d_dst + off, S->pin[b], m, cudaMemcpyHostToDevice, st));
        TIGRE_CUDA(cudaEventRecord(S->pin_ev[b], st));
    }
    return TIGRE_SUCCESS;
}

// d_src -> h_dst (pageable) after the work already queued on st; returns when h_dst is written
int staged_d2h(DeviceState* S, void* h_dst, const void* d_src, size_t n, cudaStream_t st, int which = 2) {
    if (n < kStageMin || !staging_on(which) || host_pinned(h_dst)) {
        TIGRE_CUDA(cudaMemcpyAsync(h_dst, d_src, n, cudaMemcpyDeviceToHost, st));
        TIGRE_CUDA(cudaStreamSynchronize(st));
        return TIGRE_SUCCESS;
    }
    if (int rc = ensure_pinned(S)) return rc;
    const size_t nc = (n + kStageBytes - 1) / kStageBytes;
    auto issue = [&](size_t c) -> int {
        const int b = (int)(c & 1);
        const size_t off = c * kStageBytes, m = std::min(kStageBytes, n - off);
        TIGRE_CUDA(cudaMemcpyAsync(S->pin[b], (const char*)d_src + off, m, cudaMemcpyDeviceToHost, st));
        TIGRE_CUDA(cudaEventRecord(S->pin_ev[b], st));
        return TIGRE_SUCCESS;
    };
    for (size_t c = 0; c < std::min<size_t>(2, nc); ++c)
        if (int rc = issue(c)) return rc;
    for (size_t c = 0; c < nc; ++c) {
        const int b = (int)(c & 1);
        const size_t off = c * kStageBytes, m = std::min(kStageBytes, n - off);
        TIGRE_CUDA(cudaEventSynchronize(S->pin_ev[b]));
        par_memcpy((char*)h_dst + off, S->pin[b], m);
        if (c + 2 < nc)
            if (int rc = issue(c + 2)) return rc;
    }
    return TIGRE_SUCCESS;
}

DeviceState* state(int dev) {
    std::lock_guard<std::mutex> lk(g_states_mu);
    if ((int)g_states.size() <= dev) g_states.resize(dev + 1, nullptr);
    if (!g_states[dev]) g_states[dev] = new DeviceState();
    return g_states[dev];
}

// Views per host<->device chunk: ~192 MB of projections, or option TIGRE_OPT_HOST_CHUNK_VIEWS.
size_t chunk_views(size_t per_view_bytes, int nangles) {
    size_t c = ((size_t)192 << 20) / std::max<size_t>(per_view_bytes, 1);
    if (const long long o = option(TIGRE_OPT_HOST_CHUNK_VIEWS)) c = (size_t)std::max(1LL, o);
    return std::max<size_t>(1, std::min<size_t>((size_t)nangles, c));
}

// The plan's status word after the work queued on st, cleared for the next call; stream-ordered
// (a copy into pageable memory returns once it is done), so no device-wide synchronisation.
int take_status(TigrePlan* plan, cudaStream_t st, int* out) {
    int v = 0;
    TIGRE_CUDA(cudaMemcpyAsync(&v, plan->d_status, sizeof(int), cudaMemcpyDeviceToHost, st));
    TIGRE_CUDA(cudaStreamSynchronize(st));
    TIGRE_CUDA(cudaMemsetAsync(plan->d_status, 0, sizeof(int), st));
    *out = v;
    return TIGRE_SUCCESS;
}

int host_project(const float* img, const TigreGeometry* geo, float* const* result, const float* angles, int nangles,
                 const int* ids, int n, int projector, int flags = 0) {
    TIGRE_NVTX("host projection");
    if (!img || !geo || !result || !angles) return fail(TIGRE_ERR_BAD_ASSERT, "null argument");
    int dev = 0;
    if (int rc = pick_device(ids, n, &dev)) return rc;
    DeviceGuard g(dev);
    DeviceState* S = state(dev);
    std::lock_guard<std::mutex> lk(S->mu);
    if (int rc = S->init(dev)) return rc;
    TigrePlan* plan = nullptr;
    if (int rc = S->plan(geo, angles, nangles, dev, flags, &plan)) return rc;
    const Dims& d = plan->d;
    const size_t nvox = (size_t)d.nX * d.nY * d.nZ, npix = (size_t)d.nU * d.nV;
    void* dvol = nullptr;
    if (int rc = S->get(0, nvox * sizeof(float), &dvol)) return rc;
    TIGRE_CUDA(cudaMemsetAsync(plan->d_status, 0, sizeof(int), S->st));   // this call's launches alone set it
    if (int rc = staged_h2d(S, dvol, img, nvox * sizeof(float), S->st)) return rc;
    // the volume's working copies, once for all views
    AxWork work;
    if (int rc = ax_prepare(plan, dvol, TIGRE_F32, projector, 0, nangles, S->st, &work)) return rc;
    // view chunks, double-buffered: D2H of chunk k (copy stream) overlaps the kernels of chunk k+1.
    // The last chunk's copy overlaps nothing, so the views are split to end on a short chunk.
    const int chunk = (int)chunk_views(npix * sizeof(float), nangles);
    const int tail = std::max(1, chunk / 4);
    void* buf[2];
    for (int i = 0; i < 2; ++i)
        if (int rc = S->get(1 + i, (size_t)chunk * npix * sizeof(float), &buf[i])) return rc;
    cudaEvent_t drained[2] = {S->ev[0], S->ev[1]}, computed[2] = {S->ev[2], S->ev[3]};
    int k = 0;
    for (int a = 0, cnt = 0; a < nangles; a += cnt, ++k) {
        const int rem = nangles - a;
        cnt = rem > chunk + tail ? chunk : (rem > tail && rem > chunk / 2 ? rem - tail : std::min(rem, chunk));
        const int b = k % 2;
        if (k >= 2) TIGRE_CUDA(cudaStreamWaitEvent(S->st, drained[b], 0));
        if (int rc = ax_launch(plan, work, buf[b], TIGRE_F32, a, a + cnt, S->st)) return rc;
        TIGRE_CUDA(cudaEventRecord(computed[b], S->st));
        TIGRE_CUDA(cudaStreamWaitEvent(S->st2, computed[b], 0));
        for (int i = 0; i < cnt; ++i)
            TIGRE_CUDA(cudaMemcpyAsync(result[a + i], (char*)buf[b] + (size_t)i * npix * sizeof(float),
                                       npix * sizeof(float), cudaMemcpyDeviceToHost, S->st2));
        TIGRE_CUDA(cudaEventRecord(drained[b], S->st2));
    }
    TIGRE_CUDA(cudaStreamSynchronize(S->st2));
    TIGRE_CUDA(cudaStreamSynchronize(S->st));
    // the cell-interval kernel drops (writes 0 for) a ray outside the z bound of the plan
    int status = 0;
    if (int rc = take_status(plan, S->st, &status)) return rc;
    if (status & TIGRE_STATUS_RAY_DROPPED)
        return fail(TIGRE_ERR_CUDA, "projection: a ray left the z range computed at plan time (its value is invalid)");
    return TIGRE_SUCCESS;
}

int host_backproject(const float* proj, const TigreGeometry* geo, float* result, const float* angles, int nangles,
                     const int* ids, int n, int matched, int flags = 0) {
    TIGRE_NVTX("host backprojection");
    if (!proj || !geo || !result || !angles) return fail(TIGRE_ERR_BAD_ASSERT, "null argument");
    int dev = 0;
    if (int rc = pick_device(ids, n, &dev)) return rc;
    DeviceGuard g(dev);
    DeviceState* S = state(dev);
    std::lock_guard<std::mutex> lk(S->mu);
    if (int rc = S->init(dev)) return rc;
    TigrePlan* plan = nullptr;
    if (int rc = S->plan(geo, angles, nangles, dev, flags, &plan)) return rc;
    const Dims& d = plan->d;
    const size_t nvox = (size_t)d.nX * d.nY * d.nZ, npix = (size_t)d.nU * d.nV;
    void* dvol = nullptr;
    if (int rc = S->get(0, nvox * sizeof(float), &dvol)) return rc;
    // projection chunks, double-buffered: H2D of chunk k+1 (copy stream) overlaps the
    // backprojection of chunk k, which accumulates into the volume.  The first chunk's copy
    // overlaps nothing, so views that need several chunks start with one of a quarter size
    // (views that fit one chunk keep it: a single launch sums them in one order, as the device
    // API does).
    const int chunk = (int)chunk_views(npix * sizeof(float), nangles);
    const int head = nangles > chunk ? std::max(1, chunk / 4) : chunk;
    void* buf[2];
    for (int i = 0; i < 2; ++i)
        if (int rc = S->get(1 + i, (size_t)chunk * npix * sizeof(float), &buf[i])) return rc;
    cudaEvent_t copied[2] = {S->ev[0], S->ev[1]}, consumed[2] = {S->ev[2], S->ev[3]};
    const int bp = matched ? TIGRE_BACKPROJ_MATCHED : TIGRE_BACKPROJ_FDK;
    TIGRE_CUDA(cudaMemsetAsync(plan->d_status, 0, sizeof(int), S->st));   // this call's launches alone set it
    int k = 0;
    for (int a = 0, cnt = 0; a < nangles; a += cnt, ++k) {
        cnt = std::min(k == 0 ? head : chunk, nangles - a);
        const int b = k % 2;
        if (k >= 2) TIGRE_CUDA(cudaStreamWaitEvent(S->st2, consumed[b], 0));
        if (int rc = staged_h2d(S, buf[b], proj + (size_t)a * npix, (size_t)cnt * npix * sizeof(float), S->st2, 4))
            return rc;
        TIGRE_CUDA(cudaEventRecord(copied[b], S->st2));
        TIGRE_CUDA(cudaStreamWaitEvent(S->st, copied[b], 0));
        if (int rc = tigre_atb_ex(plan, buf[b], TIGRE_F32, dvol, TIGRE_F32, bp, a, a + cnt, k > 0, S->st)) return rc;
        TIGRE_CUDA(cudaEventRecord(consumed[b], S->st));
    }
    if (int rc = staged_d2h(S, result, dvol, nvox * sizeof(float), S->st, 8)) return rc;
    TIGRE_CUDA(cudaStreamSynchronize(S->st2));
    int status = 0;
    if (int rc = take_status(plan, S->st, &status)) return rc;
    if (status & TIGRE_STATUS_WAIT_EXPIRED) return fail(TIGRE_ERR_CUDA, "backprojection: a bounded wait expired");
    return TIGRE_SUCCESS;
}

int host_pocs_tv(const float* img, float* dst, float alpha, const long* image_size, int max_iter, const int* ids,
                 int n) {
    TIGRE_NVTX("host pocs_tv");
    if (!img || !dst || !image_size) return fail(TIGRE_ERR_BAD_ASSERT, "null argument");
    const long nx = image_size[0], ny = image_size[1], nz = image_size[2];
    if (nx <= 0 || ny <= 0 || nz <= 0) return fail(TIGRE_ERR_BAD_ASSERT, "bad image size");
    int dev = 0;
    if (int rc = pick_device(ids, n, &dev)) return rc;
    DeviceGuard g(dev);
    DeviceState* S = state(dev);
    std::lock_guard<std::mutex> lk(S->mu);
    if (int rc = S->init(dev)) return rc;
    const size_t nvox = (size_t)nx * ny * nz;
    void *dimg = nullptr, *dwork = nullptr;
    if (int rc = S->get(0, nvox * sizeof(float), &dimg)) return rc;
    if (int rc = S->get(1, nvox * sizeof(float), &dwork)) return rc;
    if (int rc = staged_h2d(S, dimg, img, nvox * sizeof(float), S->st)) return rc;
    if (int rc = tigre_tv_pocs(dimg, TIGRE_F32, nx, ny, nz, alpha, max_iter, (float*)dwork, S->st)) return rc;
    return staged_d2h(S, dst, dimg, nvox * sizeof(float), S->st);
}

int host_weighted_tv(int kind, const float* img, const float* prior, float* dst, float alpha, float param,
                     const long* image_size, int max_iter, const int* ids, int n) {
    TIGRE_NVTX("host weighted tv");
    if (!img || !dst || !image_size || (kind == 1 && !prior)) return fail(TIGRE_ERR_BAD_ASSERT, "null argument");
    const long nx = image_size[0], ny = image_size[1], nz = image_size[2];
    if (nx <= 0 || ny <= 0 || nz <= 0) return fail(TIGRE_ERR_BAD_ASSERT, "bad image size");
    int dev = 0;
    if (int rc = pick_device(ids, n, &dev)) return rc;
    DeviceGuard g(dev);
    DeviceState* S = state(dev);
    std::lock_guard<std::mutex> lk(S->mu);
    if (int rc = S->init(dev)) return rc;
    const size_t nvox = (size_t)nx * ny * nz;
    void *dimg = nullptr, *dwork = nullptr, *dprior = nullptr;
    if (int rc = S->get(0, nvox * sizeof(float), &dimg)) return rc;
    if (int rc = S->get(1, nvox * sizeof(float), &dwork)) return rc;
    if (int rc = staged_h2d(S, dimg, img, nvox * sizeof(float), S->st)) return rc;
    if (kind == 1) {
        if (int rc = S->get(2, nvox * sizeof(float), &dprior)) return rc;
        if (int rc = staged_h2d(S, dprior, prior, nvox * sizeof(float), S->st)) return rc;
        if (int rc = tigre_tv_piccs(dimg, dprior, TIGRE_F32, nx, ny, nz, alpha, param, max_iter, (float*)dwork, S->st))
            return rc;
    } else if (int rc = tigre_tv_aw_pocs(dimg, TIGRE_F32, nx, ny, nz, alpha, max_iter, param, (float*)dwork, S->st)) {
        return rc;
    }
    return staged_d2h(S, dst, dimg, nvox * sizeof(float), S->st);
}

int host_tvdenoising(const float* src, float* dst, float lambda, const float* spacing, const long* image_size,
                     int max_iter, const int* ids, int n) {
    TIGRE_NVTX("host tvdenoising");
    if (!src || !dst || !image_size) return fail(TIGRE_ERR_BAD_ASSERT, "null argument");
    const long nx = image_size[0], ny = image_size[1], nz = image_size[2];
    if (nx <= 0 || ny <= 0 || nz <= 0) return fail(TIGRE_ERR_BAD_ASSERT, "bad image size");
    int dev = 0;
    if (int rc = pick_device(ids, n, &dev)) return rc;
    DeviceGuard g(dev);
    DeviceState* S = state(dev);
    std::lock_guard<std::mutex> lk(S->mu);
    if (int rc = S->init(dev)) return rc;
    const size_t nvox = (size_t)nx * ny * nz;
    void *dimg = nullptr, *dwork = nullptr;
    if (int rc = S->get(0, nvox * sizeof(float), &dimg)) return rc;
    if (int rc = S->get(1, (size_t)tigre_tv_denoise_work_floats(nx, ny, nz) * sizeof(float), &dwork)) return rc;
    if (int rc = staged_h2d(S, dimg, src, nvox * sizeof(float), S->st)) return rc;
    if (int rc = tigre_tv_denoise((const float*)dimg, (float*)dimg, nx, ny, nz, lambda, spacing, max_iter,
                                  (float*)dwork, S->st))
        return rc;
    return staged_d2h(S, dst, dimg, nvox * sizeof(float), S->st);
}

int host_noise(const float* in, long long n, int gaussian, float mu, float sigma, unsigned long long seed, float* out,
               const int* ids, int ng) {
    if (n < 0 || (n > 0 && (!in || !out))) return fail(TIGRE_ERR_BAD_ASSERT, "null argument");
    if (n == 0) return TIGRE_SUCCESS;
    int dev = 0;
    if (int rc = pick_device(ids, ng, &dev)) return rc;
    DeviceGuard g(dev);
    DeviceState* S = state(dev);
    std::lock_guard<std::mutex> lk(S->mu);
    if (int rc = S->init(dev)) return rc;
    void *din = nullptr, *dout = nullptr;
    if (int rc = S->get(0, (size_t)n * sizeof(float), &din)) return rc;
    if (int rc = S->get(1, (size_t)n * sizeof(float), &dout)) return rc;
    if (int rc = staged_h2d(S, din, in, (size_t)n * sizeof(float), S->st)) return rc;
    if (int rc = tigre_add_noise((const float*)din, (float*)dout, n, gaussian, mu, sigma, seed, S->st)) return rc;
    return staged_d2h(S, out, dout, (size_t)n * sizeof(float), S->st);
}

}  // namespace

extern "C" void tigre_release_cache(void) {
    std::lock_guard<std::mutex> lk(g_states_mu);
    for (size_t i = 0; i < g_states.size(); ++i) {
        if (!g_states[i]) continue;
        DeviceGuard g((int)i);
        std::lock_guard<std::mutex> l2(g_states[i]->mu);
        g_states[i]->release();
    }
    forget_static_addresses();
}

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
    return host_pocs_tv(img, dst, alpha, image_size, max_iter, ids, n);
}

int tigre_noise_1d(const float* in, long long n, int gaussian, float mu, float sigma, unsigned long long seed,
                   float* out, const int* ids, int ng) {
    return host_noise(in, n, gaussian, mu, sigma, seed, out, ids, ng);
}

int tigre_aw_pocs_tv(const float* img, float* dst, float alpha, const long* image_size, int max_iter, float delta,
                     const int* ids, int n) {
    return host_weighted_tv(0, img, nullptr, dst, alpha, delta, image_size, max_iter, ids, n);
}

int tigre_piccs_tv(const float* img, const float* prior, float* dst, float alpha, float ratio, const long* image_size,
                   int max_iter, const int* ids, int n) {
    return host_weighted_tv(1, img, prior, dst, alpha, ratio, image_size, max_iter, ids, n);
}

int tigre_tvdenoising(const float* src, float* dst, float lambda, const float* spacing, const long* image_size,
                      int max_iter, const int* ids, int n) {
    return host_tvdenoising(src, dst, lambda, spacing, image_size, max_iter, ids, n);
}

int tigre_siddon_ray_projection_parallel(const float* img, const TigreGeometry* geo, float* const* result,
                                         const float* angles, int nangles, const int* ids, int n) {
    return host_project(img, geo, result, angles, nangles, ids, n, TIGRE_PROJ_SIDDON, TIGRE_PLAN_PARALLEL);
}

int tigre_interpolation_projection_parallel(const float* img, const TigreGeometry* geo, float* const* result,
                                            const float* angles, int nangles, const int* ids, int n) {
    return host_project(img, geo, result, angles, nangles, ids, n, TIGRE_PROJ_INTERPOLATED, TIGRE_PLAN_PARALLEL);
}

int tigre_voxel_backprojection_parallel(const float* proj, const TigreGeometry* geo, float* result,
                                        const float* angles, int nangles, const int* ids, int n) {
    return host_backproject(proj, geo, result, angles, nangles, ids, n, 0, TIGRE_PLAN_PARALLEL);
}

}  // extern "C"
