// 3x3x3 convolution on the tcgen05 tensor cores with a TMA-staged halo tile (sm_100a).
//
// y[z][y][x][co] = relu?(b[co] + sum_{t, ci} w[co][t][ci] x[z+dz][y+dy][x+dx][ci]), BF16 operands,
// FP32 accumulation in tensor memory.  One CTA computes an output tile of 8 (x) x 16 (y) x ZT (z)
// voxels for all N = Cout output channels: ZT accumulators of 128 rows (row = 8 y + x of one
// z-slice) x N FP32 columns in TMEM.
//
// The input channels are processed in chunks of 16.  For a chunk, one 5-D TMA load brings the
// halo tile -- 10 x 18 x (ZT+2) voxels x 16 channels, zero-filled outside the volume -- into
// shared memory in the layout [z'][y'][c8][x'][8 channels], and one bulk copy brings the
// chunk's weights, pre-arranged in global memory as [tap][c8][co][8 channels].  In that layout
// the A operand of tap (dz, dy, dx) for z-slice zl is the K-major canonical operand (8-row x
// 16-byte core matrices) that starts at byte ((zl+dz) 18 + dy) 2 10 16 + 16 dx of the tile, with
// 160 bytes between the two K-adjacent core matrices and 320 bytes between 8-row groups: all 27
// taps are read from the one tile by moving the descriptor, with no gather and no im2col.  The B
// operand of the tap is the weight slab at 512 N t bytes (128 bytes between 8-row groups, 16 N
// between the K halves).  One thread issues the 27 ZT MMAs of a chunk (M = 128, K = 16) and
// commits them to the chunk stage's "empty" mbarrier; the loads of the next chunks run ahead in
// STAGES buffers.  The epilogue (4 warps) reads TMEM with tcgen05.ld, adds the bias, applies
// ReLU and stores BF16 and/or FP32 channels-last rows.
//
// Every mbarrier wait is bounded: on expiry the CTA records bit 0 in the status word, waits
// (bounded) for its copies in flight and the MMAs it issued, frees its TMEM and leaves its tile
// unwritten.

#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <mutex>

#include "tigre_internal.h"

namespace tigre {
namespace {

constexpr int kTx = 8, kTy = 16;             // output tile in x and y (M = 128 rows per z-slice)
constexpr int kHx = kTx + 2, kHy = kTy + 2;  // halo tile
constexpr int kCC = 16;                      // input channels per chunk (one K = 16 MMA per tap)
constexpr unsigned kWaitPolls = 1u << 20;    // bounded waits: ~0.1 s with the back-off below

__device__ __forceinline__ uint32_t su32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ bool bar_wait(uint32_t bar, uint32_t parity) {
    for (unsigned i = 0; i < kWaitPolls; ++i) {
        uint32_t ok;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(ok)
            : "r"(bar), "r"(parity)
            : "memory");
        if (ok) return true;
        __nanosleep(64);
    }
    return false;
}

// K-major, unswizzled shared-memory operand descriptor (start, LBO = K-adjacent core
// matrices, SBO = adjacent 8-row groups; descriptor version 1)
__device__ __forceinline__ uint64_t op_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((addr & 0x3FFFFu) >> 4) | ((uint64_t)(lbo >> 4) << 16) | ((uint64_t)(sbo >> 4) << 32) |
           (1ull << 46);
}

struct ConvTcArgs {
    const __nv_bfloat16* wk;   // weights [chunk][tap][c8][co][8]
    const float* bias;
    __nv_bfloat16* yb;
    float* yf;
    int* status;
    int D, H, W, Cin, Cout, relu;
    int zt, stages, nchunks;
    uint32_t tile_bytes, w_bytes, stage_bytes, tmem_cols;
};

template <int MAXS>
__global__ void __launch_bounds__(128, 1) conv_tc_halo_kernel(const __grid_constant__ CUtensorMap xmap, ConvTcArgs p) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    __shared__ __align__(8) unsigned long long full_bar[MAXS], empty_bar[MAXS], done_bar;
    __shared__ uint32_t tmem_slot;
    __shared__ int abort_flag;
    const int tid = threadIdx.x, wid = tid >> 5, lane = tid & 31;
    const uint32_t base = (su32(smem_raw) + 1023u) & ~1023u;
    const int tiles_x = p.W / kTx, tiles_y = p.H / kTy;
    const int bx = blockIdx.x % tiles_x, by = (blockIdx.x / tiles_x) % tiles_y, bz = blockIdx.x / (tiles_x * tiles_y);
    const int x0 = bx * kTx, y0 = by * kTy, z0 = bz * p.zt;
    const int N = p.Cout;
    if (tid == 0) {
        for (int s = 0; s < p.stages; ++s) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(su32(&full_bar[s])) : "memory");
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(su32(&empty_bar[s])) : "memory");
        }
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(su32(&done_bar)) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        abort_flag = 0;
    }
    if (wid == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(su32(&tmem_slot)),
                     "r"(p.tmem_cols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_slot;

    if (tid == 0) {
        // ---- producer and MMA issuer ----
        const uint32_t idesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((128u >> 4) << 24);
        const uint32_t A_LBO = kHx * 16, A_SBO = 2 * kHx * 16;          // 160, 320
        const uint32_t B_LBO = (uint32_t)N * 16, B_SBO = 128;
        uint32_t full_ph = 0, empty_ph = 0;                             // bit s: parity to wait for
        int issued_loads = 0, issued_mma = 0;                           // chunks
        bool ok = true;
        auto load = [&](int c) {
            const int s = c % p.stages;
            const uint32_t st = base + (uint32_t)s * p.stage_bytes;
            const uint32_t fb = su32(&full_bar[s]);
            asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(fb), "r"(p.tile_bytes + p.w_bytes)
                         : "memory");
            asm volatile(
                "cp.async.bulk.tensor.5d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5, %6}], "
                "[%7];" ::"r"(st),
                "l"((unsigned long long)&xmap), "r"(0), "r"(x0 - 1), "r"(c * (kCC / 8)), "r"(y0 - 1), "r"(z0 - 1), "r"(fb)
                : "memory");
            const __nv_bfloat16* src = p.wk + (size_t)c * (p.w_bytes / 2);
            asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                             st + p.tile_bytes),
                         "l"(src), "r"(p.w_bytes), "r"(fb)
                         : "memory");
            ++issued_loads;
        };
        const int pre = min(p.stages, p.nchunks);
        for (int c = 0; c < pre; ++c) load(c);
        for (int c = 0; c < p.nchunks && ok; ++c) {
            const int s = c % p.stages;
            if (!bar_wait(su32(&full_bar[s]), (full_ph >> s) & 1u)) { ok = false; break; }
            full_ph ^= 1u << s;
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t st = base + (uint32_t)s * p.stage_bytes, wb = st + p.tile_bytes;
            for (int zl = 0; zl < p.zt; ++zl) {
                const uint32_t dtm = tmem + (uint32_t)(zl * N);
                for (int t = 0; t < 27; ++t) {
                    const int dz = t / 9, dy = (t / 3) % 3, dx = t % 3;
                    const uint32_t a = st + (uint32_t)(((zl + dz) * kHy + dy) * 2 * kHx * 16 + dx * 16);
                    const uint64_t da = op_desc(a, A_LBO, A_SBO);
                    const uint64_t db = op_desc(wb + (uint32_t)(t * 2 * N * 16), B_LBO, B_SBO);
                    const uint32_t accum = (c > 0 || t > 0) ? 1u : 0u;
                    const uint32_t no_mask = 0u;
                    asm volatile(
                        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %5, %5, %5}, p;\n\t}\n" ::"r"(dtm),
                        "l"(da), "l"(db), "r"(idesc), "r"(accum), "r"(no_mask)
                        : "memory");
                }
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                             su32(&empty_bar[s]))
                         : "memory");
            ++issued_mma;
            // keep the loads ahead: up to chunk c + stages - 1 (with one stage, chunk c + 1), each
            // into the stage of chunk L - stages once the MMAs of that chunk have read it -- with
            // two or more stages those are the MMAs of chunk c - 1, queued before the ones just
            // issued, so the copy overlaps the MMAs of chunk c
            const int target = c + max(p.stages - 1, 1);
            while (ok && issued_loads <= target && issued_loads < p.nchunks) {
                const int sp = (issued_loads - p.stages) % p.stages;
                if (!bar_wait(su32(&empty_bar[sp]), (empty_ph >> sp) & 1u)) { ok = false; break; }
                empty_ph ^= 1u << sp;
                load(issued_loads);
            }
            if (!ok) break;
        }
        if (ok) {
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                             su32(&done_bar))
                         : "memory");
        } else {
            // a wait ran out: drain what was issued -- every issued load's full barrier and the
            // MMAs (one commit covers all of them) -- each bounded, then report
            abort_flag = 1;
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                             su32(&done_bar))
                         : "memory");
            bar_wait(su32(&done_bar), 0u);
            for (int c = issued_mma; c < issued_loads; ++c) {
                const int s = c % p.stages;
                if (bar_wait(su32(&full_bar[s]), (full_ph >> s) & 1u)) full_ph ^= 1u << s;
            }
            if (p.status) atomicOr(p.status, TIGRE_STATUS_WAIT_EXPIRED);
        }
    }
    __syncwarp();
    // ---- epilogue: all 4 warps ----
    const bool done = bar_wait(su32(&done_bar), 0u);
    __syncthreads();
    if (done && !abort_flag) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const int r = 32 * wid + lane;          // accumulator row: 8 y + x
        const int x = x0 + (r & 7), y = y0 + (r >> 3);
        for (int zl = 0; zl < p.zt; ++zl) {
            const size_t vox = ((size_t)(z0 + zl) * p.H + y) * p.W + x;
            for (int c0 = 0; c0 < N; c0 += 16) {
                uint32_t v[16];
                const uint32_t taddr = tmem + ((uint32_t)(32 * wid) << 16) + (uint32_t)(zl * N + c0);
                asm volatile(
                    "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, "
                    "[%16];"
                    : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
                      "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]),
                      "=r"(v[15])
                    : "r"(taddr));
                asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
                float f[16];
#pragma unroll
                for (int j = 0; j < 16; ++j) {
                    f[j] = __uint_as_float(v[j]) + (p.bias ? __ldg(p.bias + c0 + j) : 0.f);
                    if (p.relu) f[j] = fmaxf(f[j], 0.f);
                }
                const size_t o = vox * N + c0;
                if (p.yf) {
#pragma unroll
                    for (int q = 0; q < 4; ++q)
                        reinterpret_cast<float4*>(p.yf + o)[q] = make_float4(f[4 * q], f[4 * q + 1], f[4 * q + 2], f[4 * q + 3]);
                }
                if (p.yb) {
                    uint32_t pk[8];
#pragma unroll
                    for (int q = 0; q < 8; ++q) {
                        const __nv_bfloat162 h = __floats2bfloat162_rn(f[2 * q], f[2 * q + 1]);
                        pk[q] = *reinterpret_cast<const uint32_t*>(&h);
                    }
                    reinterpret_cast<uint4*>(p.yb + o)[0] = make_uint4(pk[0], pk[1], pk[2], pk[3]);
                    reinterpret_cast<uint4*>(p.yb + o)[1] = make_uint4(pk[4], pk[5], pk[6], pk[7]);
                }
            }
        }
    } else if (!done && tid == 0 && p.status) {
        atomicOr(p.status, TIGRE_STATUS_WAIT_EXPIRED);
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (wid == 0) {
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(p.tmem_cols) : "memory");
    }
}

// wk[c][t][c8][co][e] = w[co][t][16 c + 8 c8 + e]            (forward)
// wk[c][t][c8][ci][e] = w[16 c + 8 c8 + e][26 - t][ci]       (flip: the data-gradient convolution,
//                        whose input channels are the forward's output channels)
__global__ void arrange_weights_kernel(const __nv_bfloat16* __restrict__ w, __nv_bfloat16* __restrict__ wk, int Cin,
                                       int Cout, int flip) {
    // output layout dims: nchunks x 27 x 2 x N x 8, with K = in-channels of the convolution run
    const int K = flip ? Cout : Cin, N = flip ? Cin : Cout;
    const long total = 27L * K * N;
    for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < total; e += (long)gridDim.x * blockDim.x) {
        const int ee = (int)(e % 8);
        long r = e / 8;
        const int n = (int)(r % N); r /= N;
        const int c8 = (int)(r % 2); r /= 2;
        const int t = (int)(r % 27);
        const int c = (int)(r / 27);
        const int k = c * kCC + c8 * 8 + ee;
        __nv_bfloat16 v;
        if (!flip) v = w[(size_t)n * 27 * Cin + (size_t)t * Cin + k];
        else v = w[(size_t)k * 27 * Cin + (size_t)(26 - t) * Cin + n];
        wk[e] = v;
    }
}

PFN_cuTensorMapEncodeTiled_v12000 encode_tiled() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(f);
    });
    return fn;
}

}  // namespace

// z-slices per tile and pipeline stages for an N-channel output with nchunks input chunks.
// Several CTAs per SM overlap one CTA's loads and epilogue with another's MMAs, so a
// configuration that fits two or more CTAs per SM (<= 112 KB) is preferred, with as many
// stages (<= nchunks, <= 3) as fit; else one CTA per SM within 200 KB.
static void conv_tc_shape(int N, int D, int nchunks, int* zt, int* stages, uint32_t* tile_bytes, uint32_t* w_bytes) {
    const int cand[3] = {4, 2, 1};
    *zt = 0;
    for (int budget : {112 * 1024, 200 * 1024}) {
        for (int i = 0; i < 3; ++i) {
            const int z = cand[i];
            if (D % z || (size_t)z * N > 512) continue;
            const uint32_t tb = (uint32_t)(kHx * kHy * (z + 2) * kCC * 2), wb = (uint32_t)(27 * kCC * N * 2);
            const uint32_t stb = (tb + wb + 1023u) & ~1023u;
            for (int s = std::min(3, nchunks); s >= 1; --s) {
                if (1024 + (size_t)s * stb > (size_t)budget) continue;
                // fewer than two stages only when there is a single chunk, or as the last resort
                if (s >= std::min(2, nchunks) || (budget > 112 * 1024 && i == 2)) {
                    *zt = z; *stages = s; *tile_bytes = tb; *w_bytes = wb;
                    return;
                }
                break;
            }
        }
    }
}

bool conv_tc_halo_supported(long D, long H, long W, long Cin, long Cout) {
    if (Cin % kCC || Cout % 16 || Cout < 16 || Cout > 256 || W % kTx || H % kTy) return false;
    int zt, st;
    uint32_t tb, wb;
    conv_tc_shape((int)Cout, (int)D, (int)(Cin / kCC), &zt, &st, &tb, &wb);
    return zt > 0 && encode_tiled() != nullptr && D * H * W < (1L << 31);
}

// y = conv(x, w) (+ bias, relu) with the halo-tile kernel, for a layer with Cin input and Cout
// output channels and weights w[Cout][27 Cin].  flip != 0 runs the layer's data-gradient
// convolution instead: x is then the gradient of the output (Cout channels), y the gradient of
// the input (Cin channels), with the weights flipped in the taps and transposed in the channels
// (arrange_weights_kernel).  wk_scratch: 27 Cin Cout BF16 elements, 16-byte aligned.
int launch_conv_tc_halo(const __nv_bfloat16* x, const __nv_bfloat16* w, const float* bias, __nv_bfloat16* yb,
                        float* yf, long D, long H, long W, long Cin, long Cout, int relu, int flip,
                        __nv_bfloat16* wk_scratch, int* status, cudaStream_t st) {
    // K (input channels of this convolution) and N (its output channels)
    const long K = flip ? Cout : Cin, N = flip ? Cin : Cout;
    if (!conv_tc_halo_supported(D, H, W, K, N)) return fail(TIGRE_ERR_BAD_ASSERT, "conv shape not supported by the halo kernel");
    int zt, stages;
    uint32_t tb, wb;
    conv_tc_shape((int)N, (int)D, (int)(K / kCC), &zt, &stages, &tb, &wb);
    const long total = 27L * K * N;
    arrange_weights_kernel<<<(int)std::min<long>((total + 255) / 256, 148L * 16), 256, 0, st>>>(w, wk_scratch, (int)Cin,
                                                                                                (int)Cout, flip);
    TIGRE_LAUNCHED();
    // x as a 5-D tensor, innermost first: 8 channels, x, chunks of 8 channels, y, z
    CUtensorMap tm;
    cuuint64_t dims[5] = {8, (cuuint64_t)W, (cuuint64_t)(K / 8), (cuuint64_t)H, (cuuint64_t)D};
    cuuint64_t strides[4] = {(cuuint64_t)(K * 2), 16, (cuuint64_t)(W * K * 2), (cuuint64_t)(H * W * K * 2)};
    cuuint32_t box[5] = {8, (cuuint32_t)kHx, (cuuint32_t)(kCC / 8), (cuuint32_t)kHy, (cuuint32_t)(zt + 2)};
    cuuint32_t estr[5] = {1, 1, 1, 1, 1};
    CUresult r = encode_tiled()(&tm, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 5, const_cast<__nv_bfloat16*>(x), dims, strides,
                                box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                                CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return fail(TIGRE_ERR_CUDA, "cuTensorMapEncodeTiled (conv halo tile) failed");
    ConvTcArgs a{};
    a.wk = wk_scratch;
    a.bias = bias;
    a.yb = yb;
    a.yf = yf;
    a.status = status;
    a.D = (int)D; a.H = (int)H; a.W = (int)W; a.Cin = (int)K; a.Cout = (int)N; a.relu = relu;
    a.zt = zt;
    a.stages = stages;
    a.nchunks = (int)(K / kCC);
    a.tile_bytes = tb;
    a.w_bytes = wb;
    a.stage_bytes = (tb + wb + 1023u) & ~1023u;
    uint32_t cols = 32;
    while (cols < (uint32_t)(zt * N)) cols <<= 1;
    a.tmem_cols = cols;
    // at most 512 / cols CTAs may share an SM (their TMEM must fit its 512 columns): size the
    // shared memory so that no more fit
    const int max_ctas = 512 / (int)cols;
    const size_t need = 1024 + (size_t)stages * a.stage_bytes;
    const size_t floor_smem = max_ctas >= 8 ? 0 : (size_t)(233472 / (max_ctas + 1) - 1024 + 64);
    const size_t smem = std::max(need, floor_smem);
    TIGRE_CUDA(cudaFuncSetAttribute(conv_tc_halo_kernel<3>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const long ntiles = (W / kTx) * (H / kTy) * (D / zt);
    conv_tc_halo_kernel<3><<<(unsigned)ntiles, 128, smem, st>>>(tm, a);
    TIGRE_LAUNCHED();
    return TIGRE_SUCCESS;
}

}  // namespace tigre
