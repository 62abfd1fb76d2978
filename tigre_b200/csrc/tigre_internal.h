// Internal declarations of libtigre_b200: plan layout, per-angle frames,
// kernel launchers.  Not part of the public ABI (see include/tigre_b200.h).
#pragma once

#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cstdint>
#include <string>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "../../include/tigre_b200.h"

namespace tigre {

// NVTX range around an entry point (visible in Nsight timelines; a few ns without a profiler)
struct NvtxRange {
    explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange&) = delete;
    NvtxRange& operator=(const NvtxRange&) = delete;
};
#define TIGRE_NVTX(name) ::tigre::NvtxRange nvtx_range__(name)

// ---------------------------------------------------------------- errors --
void set_error(const std::string& msg);
int fail(int code, const std::string& msg);
int cuda_fail(cudaError_t e, const char* what);
// process-wide count of kernels launched by this library (tigre_launch_count)
void note_launches(unsigned long long n);
// current value of a library option (TIGRE_OPT_*, tigre_set_option)
long long option(int key);
// forgets the cached device addresses of the library's fixed device arrays (tigre_release_cache)
void forget_static_addresses();

// after a kernel launch: check the launch and count it
#define TIGRE_LAUNCHED()                   \
    do {                                   \
        TIGRE_CUDA(cudaGetLastError());    \
        ::tigre::note_launches(1);         \
    } while (0)

#define TIGRE_CUDA(call)                                     \
    do {                                                     \
        cudaError_t e__ = (call);                            \
        if (e__ != cudaSuccess) return cuda_fail(e__, #call); \
    } while (0)

#define TIGRE_CHECK(cond, msg)                                    \
    do {                                                          \
        if (!(cond)) return fail(TIGRE_ERR_BAD_ASSERT, (msg));    \
    } while (0)

inline size_t dtype_size(int dt) { return dt == TIGRE_F32 ? 4 : 2; }
inline bool dtype_ok(int dt) { return dt == TIGRE_F32 || dt == TIGRE_BF16 || dt == TIGRE_F16; }

// ------------------------------------------------------- per-angle frames --
// All frames are computed on the host in FP64 from the float32 geometry, once
// per plan, with the reference's formulas (cited in geometry.cpp).

// Siddon: voxel-index units, volume corner at the origin (voxel i spans [i, i+1)).
struct FrameSiddon {
    double o[3];    // detector pixel (u=0, pixelV=0), pixelV = nV-1-v
    double du[3];   // step per u
    double dv[3];   // step per pixelV
    double s[3];    // source
    int layout;     // 0: x-fastest working layout, 1: y-fastest (transposed)
    int pad_;
};

// Interpolated: voxel-centre units (voxel i centred at i).
struct FrameInterp {
    double o[3], du[3], dv[3], s[3];
    double first_sample;   // floor(cropdist/accuracy), ray_interpolated_projection.cu:193
    double cap;            // sample-count cap (:179-189); +inf when it cannot bind
    int layout;
    int pad_;
};

// Backprojection: detector-pixel units in y/z, mm in x (computeDeltasCube).
struct FrameBP {
    double o[3], dx[3], dy[3], dz[3], s[3];
    float sina, cosa;   // of the negated alpha (voxel_backprojection.cu:510-515)
    float cor, dsd, dso;
    float offx, offy, offz;   // offOrig
    float offu, offv;         // offDetec
};

// Per-view constants of the staged backprojector (backproject_tma.cu), derived from
// FrameBP on the host so that a (column, view) needs only FMAs and one division.
struct FrameBPK {
    double b[3];             // voxel (0,0,0) minus source, y shifted by -COR/dDetecU
    double dx[3], dy[3], dz[3];
    float tnum;              // DSO - DSD - S.x
    float cu, cv;            // texture-coordinate offsets S.y + nU/2, S.z + nV/2
    float w0, wx, wy;        // FDK: U = w0 + x wx + y wy, weight (DSO/U)^2
    float dso, dsd;
    float rsx, rsy;          // matched: source position (mm)
    float daxc, daxs;        // -(DSD-DSO) cos a, -(DSD-DSO) sin a
    float sina, cosa;
    float du0, ddu, dzc, ddv;
    float rv0x, rv0y, rv0z;  // voxel (0,0,0) centre in mm (with offOrig)
    float dvx, dvy;
};

struct Plan;

// ----------------------------------------------------------------- plan ---
struct Dims {
    int nX, nY, nZ;      // volume
    int nU, nV;          // detector
    int nA;              // angles in the plan
    double sVX, sVY, sVZ, dVX, dVY, dVZ;
    double sDU, sDV, dDU, dDV;
    double accuracy;
};

}  // namespace tigre

struct TigrePlan {
    int device = 0;
    bool parallel = false;       // parallel-beam geometry (TIGRE_PLAN_PARALLEL)
    tigre::Dims d{};
    std::vector<tigre::FrameSiddon> h_siddon;
    std::vector<tigre::FrameInterp> h_interp;
    std::vector<tigre::FrameBP> h_bp;
    tigre::FrameSiddon* d_siddon = nullptr;
    tigre::FrameInterp* d_interp = nullptr;
    tigre::FrameBP* d_bp = nullptr;
    bool axial = false;          // every BP frame has dz.x == dz.y == 0 (u constant along z)
    bool columns = false;        // every Siddon frame has dv.x == dv.y == 0 (detector v parallel to z)
    double column_slope_max = 0; // max over rays of |rz| / max(|rx|, |ry|): z change per xy cell
    // cell-interval Siddon: exact maxima over all rays (FP64, the kernel's own ray setup) of the
    // z change per xy cell and of the z extent of the ray inside the xy box; cells_zpad zero
    // slices before and after each z-run of the working copy cover that extent
    double cells_slope_max = 0, cells_zspan_max = 0;
    int cells_zpad = 0;          // 0: the cell-interval kernel is not usable for this plan
    std::vector<tigre::FrameBPK> h_bpk;
    tigre::FrameBPK* d_bpk = nullptr;
    int bp_box_u = 0, bp_box_v = 0;   // TMA patch box of the staged backprojector (0: not usable)
    int bp_box_u16 = 0;               // box width for 16-bit projections
    int* d_status = nullptr;          // kernel error word (bounded waits that expired)
    // hardware-texture interpolated projector (TIGRE_OPT_INTERP_TEXTURE): FP32 3-D array + texture
    cudaArray_t tex_array = nullptr;
    unsigned long long tex_obj = 0;
    // growable stream-ordered scratch arena
    void* scratch = nullptr;
    size_t scratch_bytes = 0;
};

namespace tigre {

// staged backprojector tiling: a block is kBpTile x kBpTile voxel columns of kBpSlices slices
constexpr int kBpTile = 16;
constexpr int kBpSlices = 64;

int compute_frames(const TigreGeometry* geo, const float* angles, int nangles, TigrePlan* plan);
void* plan_scratch(TigrePlan* plan, size_t bytes, cudaStream_t st, int* rc);

// ------------------------------------------------------------ launchers ---
int launch_make_layout(const void* src, int dtype, void* dst, int nX, int nY, int nZ, int layout, int pad_lo,
                       int pad_hi, cudaStream_t st);
int launch_pad_projections(const void* src, int dtype, void* dst, int nA, int nV, int nU, cudaStream_t st);
int launch_make_quads(const void* pad, int dtype, void* dst, int nX, int nY, int nZ, int layout, cudaStream_t st);
int launch_make_zfast(const void* src, int dtype, void* dst, int nX, int nY, int nZ, int zpad, cudaStream_t st);
int launch_make_zfast_f32(const void* src, int dtype, float* dst, int nX, int nY, int nZ, int zpad, cudaStream_t st);
int launch_make_quads_f32(const void* pad, int dtype, float* dst, int nX, int nY, int nZ, int layout, cudaStream_t st);
int launch_repitch_projections_f32(const void* src, int dtype, float* dst, int nA, int nV, int nU, int pitch,
                                   cudaStream_t st);

int launch_siddon(TigrePlan* p, const void* vol_x, const void* vol_y, int vdt, void* proj, int pdt, int a0, int a1,
                  cudaStream_t st);
int launch_siddon_count(TigrePlan* p, int a0, int a1, unsigned long long* d_total, cudaStream_t st);
int launch_interp_count(TigrePlan* p, int a0, int a1, unsigned long long* d_total, cudaStream_t st);
int launch_siddon_cells(TigrePlan* p, const void* vol_z, int vdt, void* proj, int pdt, int a0, int a1,
                        cudaStream_t st);
int launch_siddon_columns(TigrePlan* p, const void* vol_z, int vdt, void* proj, int pdt, int a0, int a1,
                          cudaStream_t st);
int launch_interp(TigrePlan* p, const void* vol_x, const void* vol_y, const void* quad_x, const void* quad_y, int vdt,
                  void* proj, int pdt, int a0, int a1, cudaStream_t st);
int interp_texture(TigrePlan* p, const float* d_vol, cudaStream_t st, unsigned long long* tex_out);
int launch_interp_tex(TigrePlan* p, unsigned long long tex, void* proj, int pdt, int a0, int a1, cudaStream_t st);
bool conv_tc_halo_supported(long D, long H, long W, long Cin, long Cout);
int launch_conv_tc_halo(const __nv_bfloat16* x, const __nv_bfloat16* w, const float* bias, __nv_bfloat16* yb,
                        float* yf, long D, long H, long W, long Cin, long Cout, int relu, int flip,
                        __nv_bfloat16* wk_scratch, int* status, cudaStream_t st);
int launch_backproject(TigrePlan* p, const void* proj_pad, int pdt, void* vol, int vdt, int matched, int a0, int a1,
                       int accumulate, cudaStream_t st);

bool bp_tma_supported(const TigrePlan* p, int pdt);
int launch_backproject_tma(TigrePlan* p, const void* proj, int pitch, int pdt, void* vol, int vdt, int matched,
                           int a0, int a1, int accumulate, cudaStream_t st);
int launch_repitch_projections(const void* src, int dtype, void* dst, int nA, int nV, int nU, int pitch,
                               cudaStream_t st);

// padded projection pitch and row count used by the backprojector
__host__ __device__ inline long bp_pitch(int nU) { return (long)nU + 3; }
__host__ __device__ inline long bp_rows(int nV) { return (long)nV + 3; }

// ------------------------------------------------------ dtype helpers -----
template <typename T> __device__ __forceinline__ float to_f32(T v);
template <> __device__ __forceinline__ float to_f32<float>(float v) { return v; }
template <> __device__ __forceinline__ float to_f32<__nv_bfloat16>(__nv_bfloat16 v) { return __bfloat162float(v); }
template <> __device__ __forceinline__ float to_f32<__half>(__half v) { return __half2float(v); }

template <typename T> __device__ __forceinline__ T from_f32(float v);
template <> __device__ __forceinline__ float from_f32<float>(float v) { return v; }
template <> __device__ __forceinline__ __nv_bfloat16 from_f32<__nv_bfloat16>(float v) { return __float2bfloat16_rn(v); }
template <> __device__ __forceinline__ __half from_f32<__half>(float v) { return __float2half_rn(v); }

template <typename T> __device__ __forceinline__ float ldg_f(const T* p) { return to_f32<T>(__ldg(p)); }

// dispatch a templated functor on a storage dtype
#define TIGRE_DISPATCH_DTYPE(dt, T, ...)                       \
    switch (dt) {                                              \
        case TIGRE_F32: { using T = float; __VA_ARGS__; break; }          \
        case TIGRE_BF16: { using T = __nv_bfloat16; __VA_ARGS__; break; } \
        case TIGRE_F16: { using T = __half; __VA_ARGS__; break; }         \
        default: return fail(TIGRE_ERR_BAD_ASSERT, "unsupported dtype");  \
    }

}  // namespace tigre
