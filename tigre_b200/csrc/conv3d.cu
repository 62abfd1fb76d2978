// 3x3x3 convolutions for the learned CGLS warm start: BF16 operands, FP32 accumulation on
// the tensor cores, sm_100a.
//
// Activations are channels-last volumes x[D][H][W][C] (BF16); weights w[Cout][27*Cin] with
// the tap index t = (dz*3 + dy)*3 + dx major and the input channel minor; zero padding of 1,
// stride 1.  Each convolution is an implicit GEMM done in two steps:
//   im2col:   col[v][t*Cin + c] = x at voxel v shifted by tap t      (M = D*H*W rows, K = 27*Cin)
//   forward:  y[v][co]  = relu?(sum_k col[v][k] w[co][k] + b[co])   (M x N = Cout, K)
//   data:     dcol[v][k] = sum_co dy[v][co] w[co][k];  dx = col2im(dcol) (gather over taps)
//   weight:   dw[co][k] += sum_v dy[v][co] col[v][k]                 (split over v, FP32 atomics)
// The GEMM stages 64 x 64 output tiles through shared memory in K steps of 32 and runs them on
// 16 x 16 x 16 BF16 warp MMA tiles (8 warps, each a 16 x 32 strip), zero-filling ragged edges,
// so any M, N, K work.  This is the warp-level (mma.sync) tensor-core path; moving the GEMM to
// tcgen05 with TMEM accumulators is the next step for this part.

#include <cuda_bf16.h>
#include <mma.h>

#include <algorithm>
#include <atomic>
#include <cstdint>
#include <mutex>

#include "tigre_internal.h"

namespace tigre {
namespace {

using namespace nvcuda;

constexpr int kBM = 64, kBN = 64, kBK = 32;   // block tile
constexpr int kThreads = 256;                  // 8 warps: 4 (M) x 2 (N), each 16 x 32

// Element (i, k) of op(A) (M x K) and (k, j) of op(B) (K x N).
//   A_ROW: A is row-major M x K (lda = row stride); else A is stored K x M row-major, i.e.
//          element (i, k) at A[k * lda + i].
//   B_COL: B is stored N x K row-major (element (k, j) at B[j * ldb + k]); else B is K x N
//          row-major (element (k, j) at B[k * ldb + j]).
template <bool A_ROW, bool B_COL>
__global__ void __launch_bounds__(kThreads) gemm_kernel(const __nv_bfloat16* __restrict__ A, int lda,
                                                        const __nv_bfloat16* __restrict__ B, int ldb, float* Cf,
                                                        __nv_bfloat16* Cb, int ldc, int M, int N, int K,
                                                        const float* __restrict__ bias, int relu, int k_chunk,
                                                        int atomic) {
    __shared__ __align__(32) __nv_bfloat16 sA[kBM][kBK + 8];
    __shared__ __align__(32) __nv_bfloat16 sB[kBK][kBN + 8];
    __shared__ __align__(32) float sC[kBM][kBN + 4];
    const int tid = threadIdx.x, wid = tid >> 5;
    const int m0 = blockIdx.x * kBM, n0 = blockIdx.y * kBN;
    const int kb = blockIdx.z * k_chunk, ke = min(K, kb + k_chunk);
    const int wm = (wid & 3) * 16, wn = (wid >> 2) * 32;
    wmma::fragment<wmma::accumulator, 16, 16, 16, float> acc[2];
    wmma::fill_fragment(acc[0], 0.f);
    wmma::fill_fragment(acc[1], 0.f);
    const __nv_bfloat16 zero = __float2bfloat16(0.f);
    for (int k0 = kb; k0 < ke; k0 += kBK) {
        // stage A (64 x 32) and B (32 x 64), zero outside the matrices / the K chunk
        for (int e = tid; e < kBM * kBK; e += kThreads) {
            const int i = e / kBK, k = e % kBK;
            const int gi = m0 + i, gk = k0 + k;
            __nv_bfloat16 v = zero;
            if (gi < M && gk < ke) v = A_ROW ? A[(size_t)gi * lda + gk] : A[(size_t)gk * lda + gi];
            sA[i][k] = v;
        }
        for (int e = tid; e < kBK * kBN; e += kThreads) {
            const int k = e / kBN, j = e % kBN;
            const int gk = k0 + k, gj = n0 + j;
            __nv_bfloat16 v = zero;
            if (gj < N && gk < ke) v = B_COL ? B[(size_t)gj * ldb + gk] : B[(size_t)gk * ldb + gj];
            sB[k][j] = v;
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < kBK; kk += 16) {
            wmma::fragment<wmma::matrix_a, 16, 16, 16, __nv_bfloat16, wmma::row_major> fa;
            wmma::load_matrix_sync(fa, &sA[wm][kk], kBK + 8);
#pragma unroll
            for (int t = 0; t < 2; ++t) {
                wmma::fragment<wmma::matrix_b, 16, 16, 16, __nv_bfloat16, wmma::row_major> fb;
                wmma::load_matrix_sync(fb, &sB[kk][wn + 16 * t], kBN + 8);
                wmma::mma_sync(acc[t], fa, fb, acc[t]);
            }
        }
        __syncthreads();
    }
    wmma::store_matrix_sync(&sC[wm][wn], acc[0], kBN + 4, wmma::mem_row_major);
    wmma::store_matrix_sync(&sC[wm][wn + 16], acc[1], kBN + 4, wmma::mem_row_major);
    __syncthreads();
    for (int e = tid; e < kBM * kBN; e += kThreads) {
        const int i = e / kBN, j = e % kBN;
        const int gi = m0 + i, gj = n0 + j;
        if (gi >= M || gj >= N) continue;
        float v = sC[i][j];
        if (atomic == 2) {   // split-K partial: slice blockIdx.z of M x N
            Cf[(size_t)blockIdx.z * M * ldc + (size_t)gi * ldc + gj] = v;
            continue;
        }
        if (atomic) {
            atomicAdd(Cf + (size_t)gi * ldc + gj, v);
            continue;
        }
        if (bias) v += bias[gj];
        if (relu) v = fmaxf(v, 0.f);
        if (Cf) Cf[(size_t)gi * ldc + gj] = v;
        if (Cb) Cb[(size_t)gi * ldc + gj] = __float2bfloat16(v);
    }
}

// dst[i] += sum over s < splits of ws[s * n + i], in order of s
__global__ void reduce_slices_kernel(const float* __restrict__ ws, float* __restrict__ dst, long n, long splits) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        float acc = dst[i];
        for (long s = 0; s < splits; ++s) acc += ws[s * n + i];
        dst[i] = acc;
    }
}

// col[v][t*C + c] = x[z+dz-1][y+dy-1][x+dx-1][c] (0 outside)
__global__ void im2col_kernel(const __nv_bfloat16* __restrict__ x, __nv_bfloat16* __restrict__ col, int D, int H,
                              int W, int C) {
    const long K = 27L * C, total = (long)D * H * W * K;
    for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < total; e += (long)gridDim.x * blockDim.x) {
        const long v = e / K;
        const int k = (int)(e - v * K), t = k / C, c = k - t * C;
        const int xx = (int)(v % W), yy = (int)((v / W) % H), zz = (int)(v / ((long)W * H));
        const int sx = xx + t % 3 - 1, sy = yy + (t / 3) % 3 - 1, sz = zz + t / 9 - 1;
        __nv_bfloat16 val = __float2bfloat16(0.f);
        if (sx >= 0 && sx < W && sy >= 0 && sy < H && sz >= 0 && sz < D)
            val = x[(((long)sz * H + sy) * W + sx) * C + c];
        col[e] = val;
    }
}

// dx[z][y][x][c] = sum over taps t of dcol[v(t)][t*C + c], v(t) = the voxel whose tap t reads (z,y,x)
__global__ void col2im_kernel(const float* __restrict__ dcol, float* __restrict__ dx, int D, int H, int W, int C) {
    const long total = (long)D * H * W * C, K = 27L * C;
    for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < total; e += (long)gridDim.x * blockDim.x) {
        const int c = (int)(e % C);
        const long v = e / C;
        const int xx = (int)(v % W), yy = (int)((v / W) % H), zz = (int)(v / ((long)W * H));
        float s = 0.f;
#pragma unroll
        for (int t = 0; t < 27; ++t) {
            // tap t of output voxel o reads o + off(t); so o = (z,y,x) - off(t)
            const int ox = xx - (t % 3 - 1), oy = yy - ((t / 3) % 3 - 1), oz = zz - (t / 9 - 1);
            if (ox >= 0 && ox < W && oy >= 0 && oy < H && oz >= 0 && oz < D)
                s += dcol[(((long)oz * H + oy) * W + ox) * K + (long)t * C + c];
        }
        dx[e] = s;
    }
}

// Implicit-GEMM forward convolution (Cin a multiple of 8): the A tile (128 voxels x 32
// channels of one tap) is gathered straight from the channels-last input with 16-byte
// cp.async copies (zero-filled outside the volume and past Cin), the B tile (BN output
// channels x the same 32 k) from the weight rows, both double-buffered; no im2col buffer.
// The accumulators start from the bias; ReLU and the BF16 / FP32 store go through a small
// per-warp staging tile so that ragged edges are masked.
__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src, bool valid) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(dst), "l"(src), "r"(valid ? 16 : 0));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

template <int BN>
__global__ void __launch_bounds__(256) conv_fwd_implicit_kernel(const __nv_bfloat16* __restrict__ x,
                                                                const __nv_bfloat16* __restrict__ w,
                                                                const float* __restrict__ bias,
                                                                __nv_bfloat16* yb, float* yf, int D, int H, int W,
                                                                int Cin, int Cout, int relu) {
    constexpr int BM = 128, BK = 32, LDA = BK + 8, LDB = BK + 8, NF = BN / 16;
    __shared__ __align__(128) __nv_bfloat16 sA[2][BM][LDA];
    __shared__ __align__(128) __nv_bfloat16 sB[2][BN][LDB];   // [n][k]: matrix_b col-major
    __shared__ __align__(128) float sBias[16][BN + 4];
    __shared__ __align__(128) float sStage[8][16][20];
    const int tid = threadIdx.x, wid = tid >> 5, lane = tid & 31;
    const long M = (long)D * H * W;
    const long m0 = (long)blockIdx.x * BM;
    const int n0 = blockIdx.y * BN;
    const int K27 = 27 * Cin;
    for (int e = tid; e < 16 * BN; e += 256) {
        const int j = e % BN, gj = n0 + j;
        sBias[e / BN][j] = (bias && gj < Cout) ? bias[gj] : 0.f;
    }
    // A: 128 rows x 4 chunks of 8 channels -> 2 chunks per thread; B: BN rows x 4 chunks
    const int a_row0 = tid >> 2, a_chunk = tid & 3;   // rows a_row0 and a_row0 + 64
    long av[2];
    int az[2], ay[2], ax[2];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
        av[h] = m0 + a_row0 + 64 * h;
        const long v = av[h] < M ? av[h] : 0;
        ax[h] = (int)(v % W);
        ay[h] = (int)((v / W) % H);
        az[h] = (int)(v / ((long)W * H));
    }
    const int csteps = (Cin + BK - 1) / BK, nsteps = 27 * csteps;
    auto load_stage = [&](int step, int buf) {
        const int tap = step / csteps, c0 = (step - tap * csteps) * BK;
        const int dx = tap % 3 - 1, dy = (tap / 3) % 3 - 1, dz = tap / 9 - 1;
        const int c = c0 + a_chunk * 8;
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int sx = ax[h] + dx, sy = ay[h] + dy, sz = az[h] + dz;
            const bool ok = av[h] < M && c < Cin && sx >= 0 && sx < W && sy >= 0 && sy < H && sz >= 0 && sz < D;
            const __nv_bfloat16* src = ok ? x + ((((long)sz * H + sy) * W + sx) * Cin + c) : x;
            cp_async16((uint32_t)__cvta_generic_to_shared(&sA[buf][a_row0 + 64 * h][a_chunk * 8]), src, ok);
        }
        for (int e = tid; e < BN * 4; e += 256) {
            const int j = e >> 2, ch = e & 3, gj = n0 + j, cc = c0 + ch * 8;
            const bool ok = gj < Cout && cc < Cin;
            const __nv_bfloat16* src = ok ? w + ((long)gj * K27 + (long)tap * Cin + cc) : w;
            cp_async16((uint32_t)__cvta_generic_to_shared(&sB[buf][j][ch * 8]), src, ok);
        }
        cp_async_commit();
    };
    __syncthreads();   // sBias
    wmma::fragment<wmma::accumulator, 16, 16, 16, float> acc[NF];
    const int wm = wid * 16;
#pragma unroll
    for (int t = 0; t < NF; ++t) wmma::load_matrix_sync(acc[t], &sBias[0][16 * t], BN + 4, wmma::mem_row_major);
    load_stage(0, 0);
    for (int step = 0; step < nsteps; ++step) {
        const int buf = step & 1;
        if (step + 1 < nsteps) {
            load_stage(step + 1, buf ^ 1);
            cp_async_wait<1>();
        } else {
            cp_async_wait<0>();
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < BK; kk += 16) {
            wmma::fragment<wmma::matrix_a, 16, 16, 16, __nv_bfloat16, wmma::row_major> fa;
            wmma::load_matrix_sync(fa, &sA[buf][wm][kk], LDA);
#pragma unroll
            for (int t = 0; t < NF; ++t) {
                wmma::fragment<wmma::matrix_b, 16, 16, 16, __nv_bfloat16, wmma::col_major> fb;
                wmma::load_matrix_sync(fb, &sB[buf][16 * t][kk], LDB);
                wmma::mma_sync(acc[t], fa, fb, acc[t]);
            }
        }
        __syncthreads();   // buffer buf is refilled by the next iteration's load
    }
#pragma unroll
    for (int t = 0; t < NF; ++t) {
        if (relu) {
#pragma unroll
            for (int i = 0; i < acc[t].num_elements; ++i) acc[t].x[i] = fmaxf(acc[t].x[i], 0.f);
        }
        wmma::store_matrix_sync(&sStage[wid][0][0], acc[t], 20, wmma::mem_row_major);
        __syncwarp();
        for (int e = lane; e < 256; e += 32) {
            const int i = e >> 4, j = e & 15;
            const long gi = m0 + wm + i;
            const int gj = n0 + 16 * t + j;
            if (gi < M && gj < Cout) {
                const float v = sStage[wid][i][j];
                if (yf) yf[gi * Cout + gj] = v;
                if (yb) yb[gi * Cout + gj] = __float2bfloat16(v);
            }
        }
        __syncwarp();
    }
}

// ---- tcgen05 implicit-GEMM forward convolution (Cin % 8 == 0, Cout % 16 == 0) ----
//
// One CTA of 4 warps computes a 128-voxel x BN-channel tile.  Per K step (one tap x 32 input
// channels) all threads gather the A tile (128 x 32 BF16) and the B tile (BN x 32) with 16-byte
// cp.async copies into the K-major, unswizzled canonical layout of the tensor-core operands
// (8-row x 16-byte core matrices; LBO = 128 B between the four core matrices along K, SBO =
// 512 B between 8-row groups), then one thread issues two tcgen05.mma (K = 16 each) that
// accumulate in TMEM (128 lanes x BN FP32 columns) and commits them to the stage's mbarrier.
// Two smem stages: a stage is refilled only after the MMAs that read it have completed (their
// mbarrier phase).  The epilogue reads TMEM with tcgen05.ld (warp w: lanes 32w..32w+31 = its
// 32 voxels), adds the bias, applies ReLU and stores.  Every mbarrier wait is bounded; on
// expiry the tile is left unwritten and the status word gets bit 0.
constexpr unsigned kTcWaitLimit = 1u << 20;   // polls of ~100 ns: about 0.1 s

__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((addr & 0x3FFFFu) >> 4) | ((uint64_t)(lbo >> 4) << 16) | ((uint64_t)(sbo >> 4) << 32) |
           (1ull << 46);   // descriptor version 1; base offset 0; no swizzle
}

__device__ __forceinline__ bool tc_wait(uint32_t bar, uint32_t phase) {
    for (unsigned i = 0; i < kTcWaitLimit; ++i) {
        uint32_t ok;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(ok)
            : "r"(bar), "r"(phase)
            : "memory");
        if (ok) return true;
        __nanosleep(64);
    }
    return false;
}

template <int BN>
__global__ void __launch_bounds__(128) conv_fwd_tc_kernel(const __nv_bfloat16* __restrict__ x,
                                                          const __nv_bfloat16* __restrict__ w,
                                                          const float* __restrict__ bias, __nv_bfloat16* yb,
                                                          float* yf, int D, int H, int W, int Cin, int Cout, int relu,
                                                          int* status) {
    static_assert(BN % 16 == 0 && BN >= 16 && BN <= 128, "N tile");
    constexpr int BM = 128, BK = 64, STAGES = 3;
    constexpr int A_BYTES = BM * BK * 2, B_BYTES = BN * BK * 2, STAGE_BYTES = A_BYTES + B_BYTES;
    constexpr uint32_t TCOLS = BN <= 32 ? 32 : (BN <= 64 ? 64 : 128);
    constexpr uint32_t LBO = 128, SBO = 1024;   // K-adjacent core matrices / 8-row groups
    extern __shared__ __align__(1024) unsigned char tc_smem[];
    __shared__ __align__(8) unsigned long long mma_bar[STAGES];
    __shared__ uint32_t tmem_slot;
    const int tid = threadIdx.x, wid = tid >> 5, lane = tid & 31;
    const uint32_t base = ((uint32_t)__cvta_generic_to_shared(tc_smem) + 1023u) & ~1023u;
    const long M = (long)D * H * W;
    const long m0 = (long)blockIdx.x * BM;
    const int n0 = blockIdx.y * BN;
    const int K27 = 27 * Cin;
    if (tid == 0) {
        for (int s = 0; s < STAGES; ++s)
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"((uint32_t)__cvta_generic_to_shared(&mma_bar[s]))
                         : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (wid == 0) {
        const uint32_t slot = (uint32_t)__cvta_generic_to_shared(&tmem_slot);
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(slot), "r"(TCOLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_slot;
    // A loads: eight lanes take one voxel's eight consecutive 16-byte chunks (128 contiguous bytes
    // when the chunks stay in one tap), so a warp reads 4 voxels per copy; this thread serves rows
    // (tid >> 3) + 16 i, i = 0..7, always chunk tid & 7
    const int jA = tid & 7;
    int rx[8], ry[8], rz[8];
    bool rin[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const long av = m0 + (tid >> 3) + 16 * i;
        rin[i] = av < M;
        const long vv = rin[i] ? av : 0;
        rx[i] = (int)(vv % W);
        ry[i] = (int)((vv / W) % H);
        rz[i] = (int)(vv / ((long)W * H));
    }
    const int nsteps = (K27 + BK - 1) / BK;
    auto tile_off = [](int r, int j) -> uint32_t { return (uint32_t)((r >> 3) * SBO + j * LBO + (r & 7) * 16); };
    // a step covers K range [64 step, 64 step + 64) of the flattened (tap, channel) index, eight
    // 16-byte chunks per row; a chunk never straddles two taps (Cin % 8 == 0)
    auto load_stage = [&](int step, int s) {
        const uint32_t sa = base + (uint32_t)s * STAGE_BYTES, sb = sa + A_BYTES;
        const int k = step * BK + 8 * jA;
        const int tap = k / Cin, c = k - tap * Cin;
        const int dx = tap % 3 - 1, dy = (tap / 3) % 3 - 1, dz = tap / 9 - 1;
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            const int sx = rx[i] + dx, sy = ry[i] + dy, sz = rz[i] + dz;
            const bool ok = k < K27 && rin[i] && sx >= 0 && sx < W && sy >= 0 && sy < H && sz >= 0 && sz < D;
            const long off = (((long)sz * H + sy) * W + sx) * Cin + c;
            cp_async16(sa + tile_off((tid >> 3) + 16 * i, jA), ok ? (const void*)(x + off) : (const void*)x, ok);
        }
        for (int e = tid; e < BN * 8; e += 128) {
            const int r = e >> 3, j = e & 7, gj = n0 + r, k = step * BK + 8 * j;
            const bool ok = gj < Cout && k < K27;
            cp_async16(sb + tile_off(r, j), ok ? (const void*)(w + (long)gj * K27 + k) : (const void*)w, ok);
        }
    };
    constexpr uint32_t idesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(BN >> 3) << 17) |
                               ((uint32_t)(BM >> 4) << 24);
    bool ok_all = true;
    uint32_t phase_bits = 0u;   // bit s: parity to wait for on stage s
    unsigned issued_bits = 0u;
    auto wait_stage = [&](int s) {
        if ((issued_bits >> s) & 1u) {
            const uint32_t bar = (uint32_t)__cvta_generic_to_shared(&mma_bar[s]);
            if (ok_all && !tc_wait(bar, (phase_bits >> s) & 1u)) ok_all = false;
            phase_bits ^= 1u << s;
            issued_bits &= ~(1u << s);
        }
    };
    // prologue: the first STAGES-1 steps in flight (one cp.async group each, empty ones too)
    for (int p = 0; p < STAGES - 1; ++p) {
        if (p < nsteps) load_stage(p, p);
        cp_async_commit();
    }
    for (int step = 0; step < nsteps; ++step) {
        const int s = step % STAGES;
        cp_async_wait<STAGES - 2>();
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (tid == 0 && ok_all) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t sa = base + (uint32_t)s * STAGE_BYTES, sb = sa + A_BYTES;
#pragma unroll
            for (int kk = 0; kk < BK / 16; ++kk) {
                const uint64_t da = smem_desc(sa + 2u * LBO * kk, LBO, SBO);
                const uint64_t db = smem_desc(sb + 2u * LBO * kk, LBO, SBO);
                const uint32_t acc = (step > 0 || kk > 0) ? 1u : 0u;
                const uint32_t no_mask = 0u;
                asm volatile(
                    "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                    "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %5, %5, %5}, p;\n\t}\n" ::"r"(tmem),
                    "l"(da), "l"(db), "r"(idesc), "r"(acc), "r"(no_mask)
                    : "memory");
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                             (uint32_t)__cvta_generic_to_shared(&mma_bar[s]))
                         : "memory");
        }
        issued_bits |= 1u << s;
        // refill the stage of step-1 with step+STAGES-1 once the MMAs of step-1 have read it
        const int next = step + STAGES - 1;
        const int ns = next % STAGES;
        if (next < nsteps) {
            wait_stage(ns);
            load_stage(next, ns);
        }
        cp_async_commit();
    }
    for (int s = 0; s < STAGES; ++s) wait_stage(s);
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const long row = m0 + 32 * wid + lane;
    if (ok_all) {
#pragma unroll
        for (int t = 0; t < BN / 16; ++t) {
            uint32_t r[16];
            const uint32_t taddr = tmem + ((uint32_t)(32 * wid) << 16) + (uint32_t)(16 * t);
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, "
                "[%16];"
                : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                  "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
                  "=r"(r[15])
                : "r"(taddr));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if (row < M) {
                // this thread's 16 consecutive channels: 16-byte vector stores (Cout % BN == 0, so
                // every column exists and the row segment is 32-byte aligned)
                float v[16];
#pragma unroll
                for (int j = 0; j < 16; ++j) {
                    v[j] = __uint_as_float(r[j]) + (bias ? bias[n0 + 16 * t + j] : 0.f);
                    if (relu) v[j] = fmaxf(v[j], 0.f);
                }
                const long o = row * Cout + n0 + 16 * t;
                if (yf) {
#pragma unroll
                    for (int q = 0; q < 4; ++q)
                        reinterpret_cast<float4*>(yf + o)[q] = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
                }
                if (yb) {
                    uint32_t pk[8];
#pragma unroll
                    for (int q = 0; q < 8; ++q) {
                        const __nv_bfloat162 h = __floats2bfloat162_rn(v[2 * q], v[2 * q + 1]);
                        pk[q] = *reinterpret_cast<const uint32_t*>(&h);
                    }
                    reinterpret_cast<uint4*>(yb + o)[0] = make_uint4(pk[0], pk[1], pk[2], pk[3]);
                    reinterpret_cast<uint4*>(yb + o)[1] = make_uint4(pk[4], pk[5], pk[6], pk[7]);
                }
            }
        }
    } else if (tid == 0 && status) {
        atomicOr(status, 1);
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (wid == 0) {
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TCOLS) : "memory");
    }
}

// Launch of the tcgen05 kernel with dynamic shared memory sized so that at most 512 / TCOLS CTAs
// share an SM: their TMEM allocations then always fit the SM's 512 columns.
template <int BN>
int launch_conv_tc(const __nv_bfloat16* x, const __nv_bfloat16* w, const float* bias, __nv_bfloat16* yb, float* yf,
                   int D, int H, int W, int Cin, int Cout, int relu, int* status, cudaStream_t st) {
    constexpr int TCOLS = BN <= 32 ? 32 : (BN <= 64 ? 64 : 128);
    constexpr int max_ctas = 512 / TCOLS;
    const long M = (long)D * H * W;
    const int need = 1024 + 3 * (128 * 64 * 2 + BN * 64 * 2);
    const int floor_smem = max_ctas >= 16 ? 0 : 233472 / (max_ctas + 1) - 1024 + 64;
    const int smem = std::max(need, floor_smem);
    TIGRE_CUDA(cudaFuncSetAttribute(conv_fwd_tc_kernel<BN>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    dim3 grid((unsigned)((M + 127) / 128), (unsigned)(Cout / BN), 1);
    conv_fwd_tc_kernel<BN><<<grid, 128, smem, st>>>(x, w, bias, yb, yf, D, H, W, Cin, Cout, relu, status);
    TIGRE_LAUNCHED();
    return TIGRE_SUCCESS;
}

int grid_for_conv(long n) { return (int)std::min<long>((n + 255) / 256, 148L * 32); }

}  // namespace
}  // namespace tigre

using namespace tigre;

// Forward path selection: 3 (default) = the tcgen05 halo-tile kernel (conv3d_tc.cu) wherever its
// shape rules hold (Cin % 16 == 0, Cout % 16 == 0, W % 8 == 0, H % 16 == 0), else mode 2;
// 0 = warp-level implicit GEMM, 1 = tcgen05 implicit GEMM with per-step gathers, 2 = that
// tcgen05 kernel for narrow layers (Cin <= 16 or Cout == 16) and the warp-level one for wider ones.
static std::atomic<int> g_conv_tcgen05{3};

// Per-device status word of the tensor-core convolution kernels (bit 0: a bounded wait expired
// and that tile was left unwritten), allocated on first use; read by tigre_conv3d_status.
namespace {
constexpr int kMaxConvDevices = 64;
std::mutex g_conv_status_mu;
int* g_conv_status[kMaxConvDevices] = {};

int* conv_status_word() {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxConvDevices) return nullptr;
    std::lock_guard<std::mutex> lk(g_conv_status_mu);
    if (!g_conv_status[dev]) {
        int* p = nullptr;
        if (cudaMalloc(&p, sizeof(int)) != cudaSuccess) return nullptr;
        if (cudaMemset(p, 0, sizeof(int)) != cudaSuccess) { cudaFree(p); return nullptr; }
        g_conv_status[dev] = p;
    }
    return g_conv_status[dev];
}
}  // namespace

extern "C" {

int tigre_conv3d_set_tcgen05(int mode) { return g_conv_tcgen05.exchange(mode < 0 || mode > 3 ? 3 : mode); }

int tigre_conv3d_status(int reset) {
    int* w = conv_status_word();
    if (!w) return -1;
    int v = 0;
    if (cudaDeviceSynchronize() != cudaSuccess) return -1;
    if (cudaMemcpy(&v, w, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) return -1;
    if (reset && cudaMemset(w, 0, sizeof(int)) != cudaSuccess) return -1;
    return v;
}

long long tigre_conv3d_col_elems(long D, long H, long W, long C) { return 27LL * D * H * W * C; }

int tigre_conv3d_fwd(const void* d_x, const void* d_w, const float* d_bias, void* d_y_bf16, float* d_y_f32, long D,
                     long H, long W, long Cin, long Cout, int relu, void* d_col, void* stream) {
    TIGRE_NVTX("tigre_conv3d_fwd");
    if (!d_x || !d_w || !d_col || (!d_y_bf16 && !d_y_f32) || D <= 0 || H <= 0 || W <= 0 || Cin <= 0 || Cout <= 0)
        return fail(TIGRE_ERR_BAD_ASSERT, "bad conv3d arguments");
    const long M = D * H * W, K = 27 * Cin;
    cudaStream_t st = (cudaStream_t)stream;
    int tc_mode = g_conv_tcgen05.load();
    int* status = conv_status_word();
    if (tc_mode == 3 && ((uintptr_t)d_x & 15) == 0 && ((uintptr_t)d_col & 15) == 0 &&
        27L * Cin * Cout <= tigre_conv3d_col_elems(D, H, W, Cin) && conv_tc_halo_supported(D, H, W, Cin, Cout))
        return launch_conv_tc_halo((const __nv_bfloat16*)d_x, (const __nv_bfloat16*)d_w, d_bias,
                                   (__nv_bfloat16*)d_y_bf16, d_y_f32, D, H, W, Cin, Cout, relu, 0,
                                   (__nv_bfloat16*)d_col, status, st);
    if (tc_mode == 3) tc_mode = 2;
    // the other paths index the im2col matrix (M x 27 Cin) with 32-bit row counts
    if (M * K >= (1L << 31) * 4L || M >= (1L << 31) / 64 * 64) return fail(TIGRE_ERR_BAD_ASSERT, "conv3d too large");
    const bool tc_wanted = tc_mode == 1 || (tc_mode == 2 && (Cin <= 16 || Cout == 16));
    if (tc_wanted && Cin % 8 == 0 && Cout % 16 == 0 && ((uintptr_t)d_x & 15) == 0 && ((uintptr_t)d_w & 15) == 0) {
        // tensor-core (tcgen05) implicit GEMM: N tile = the largest of 128 / 64 / 48 / 32 / 16 dividing Cout
        const __nv_bfloat16* xb = (const __nv_bfloat16*)d_x;
        const __nv_bfloat16* wb = (const __nv_bfloat16*)d_w;
        __nv_bfloat16* yb = (__nv_bfloat16*)d_y_bf16;
        const int iD = (int)D, iH = (int)H, iW = (int)W, ci = (int)Cin, co = (int)Cout;
        if (Cout % 128 == 0) return launch_conv_tc<128>(xb, wb, d_bias, yb, d_y_f32, iD, iH, iW, ci, co, relu, status, st);
        if (Cout % 64 == 0) return launch_conv_tc<64>(xb, wb, d_bias, yb, d_y_f32, iD, iH, iW, ci, co, relu, status, st);
        if (Cout % 48 == 0) return launch_conv_tc<48>(xb, wb, d_bias, yb, d_y_f32, iD, iH, iW, ci, co, relu, status, st);
        if (Cout % 32 == 0) return launch_conv_tc<32>(xb, wb, d_bias, yb, d_y_f32, iD, iH, iW, ci, co, relu, status, st);
        return launch_conv_tc<16>(xb, wb, d_bias, yb, d_y_f32, iD, iH, iW, ci, co, relu, status, st);
    }
    if (Cin % 8 == 0 && ((uintptr_t)d_x & 15) == 0 && ((uintptr_t)d_w & 15) == 0) {
        // implicit GEMM: 16-byte channel chunks need Cin % 8 == 0 and 16-byte aligned bases
        const int bn = Cout <= 16 ? 16 : (Cout <= 32 ? 32 : 64);
        dim3 grid((unsigned)((M + 127) / 128), (unsigned)((Cout + bn - 1) / bn), 1);
        const __nv_bfloat16* xb = (const __nv_bfloat16*)d_x;
        const __nv_bfloat16* wb = (const __nv_bfloat16*)d_w;
        if (bn == 16)
            conv_fwd_implicit_kernel<16><<<grid, 256, 0, st>>>(xb, wb, d_bias, (__nv_bfloat16*)d_y_bf16, d_y_f32,
                                                              (int)D, (int)H, (int)W, (int)Cin, (int)Cout, relu);
        else if (bn == 32)
            conv_fwd_implicit_kernel<32><<<grid, 256, 0, st>>>(xb, wb, d_bias, (__nv_bfloat16*)d_y_bf16, d_y_f32,
                                                              (int)D, (int)H, (int)W, (int)Cin, (int)Cout, relu);
        else
            conv_fwd_implicit_kernel<64><<<grid, 256, 0, st>>>(xb, wb, d_bias, (__nv_bfloat16*)d_y_bf16, d_y_f32,
                                                              (int)D, (int)H, (int)W, (int)Cin, (int)Cout, relu);
        TIGRE_LAUNCHED();
        return TIGRE_SUCCESS;
    }
    im2col_kernel<<<grid_for_conv(M * K), 256, 0, st>>>((const __nv_bfloat16*)d_x, (__nv_bfloat16*)d_col, (int)D,
                                                        (int)H, (int)W, (int)Cin);
    TIGRE_LAUNCHED();
    dim3 grid((unsigned)((M + kBM - 1) / kBM), (unsigned)((Cout + kBN - 1) / kBN), 1);
    gemm_kernel<true, true><<<grid, kThreads, 0, st>>>((const __nv_bfloat16*)d_col, (int)K,
                                                      (const __nv_bfloat16*)d_w, (int)K, d_y_f32,
                                                      (__nv_bfloat16*)d_y_bf16, (int)Cout, (int)M, (int)Cout, (int)K,
                                                      d_bias, relu, (int)K, 0);
    TIGRE_LAUNCHED();
    return TIGRE_SUCCESS;
}

// dx (FP32, channels-last) from dy (BF16, M x Cout) and w; d_dcol: M * 27*Cin floats of scratch.
int tigre_conv3d_bwd_data(const void* d_dy, const void* d_w, float* d_dx, long D, long H, long W, long Cin, long Cout,
                          float* d_dcol, void* stream) {
    TIGRE_NVTX("tigre_conv3d_bwd_data");
    if (!d_dy || !d_w || !d_dx || !d_dcol || D <= 0 || H <= 0 || W <= 0 || Cin <= 0 || Cout <= 0)
        return fail(TIGRE_ERR_BAD_ASSERT, "bad conv3d arguments");
    const long M = D * H * W, K = 27 * Cin;
    cudaStream_t st = (cudaStream_t)stream;
    if (g_conv_tcgen05.load() == 3 && ((uintptr_t)d_dy & 15) == 0 && ((uintptr_t)d_dcol & 15) == 0 &&
        conv_tc_halo_supported(D, H, W, Cout, Cin)) {
        // the data gradient is the convolution of dy with the tap-flipped, channel-transposed
        // weights: the halo kernel, FP32 output, no im2col (d_dcol holds the arranged weights)
        return launch_conv_tc_halo((const __nv_bfloat16*)d_dy, (const __nv_bfloat16*)d_w, nullptr, nullptr, d_dx, D,
                                   H, W, Cin, Cout, 0, 1, (__nv_bfloat16*)d_dcol, conv_status_word(), st);
    }
    dim3 grid((unsigned)((M + kBM - 1) / kBM), (unsigned)((K + kBN - 1) / kBN), 1);
    // dcol (M x K) = dy (M x Cout, row-major) . w (Cout x K, row-major)
    gemm_kernel<true, false><<<grid, kThreads, 0, st>>>((const __nv_bfloat16*)d_dy, (int)Cout,
                                                       (const __nv_bfloat16*)d_w, (int)K, d_dcol, nullptr, (int)K,
                                                       (int)M, (int)K, (int)Cout, nullptr, 0, (int)Cout, 0);
    TIGRE_LAUNCHED();
    col2im_kernel<<<grid_for_conv(M * Cin), 256, 0, st>>>(d_dcol, d_dx, (int)D, (int)H, (int)W, (int)Cin);
    TIGRE_LAUNCHED();
    return TIGRE_SUCCESS;
}

// dw (FP32, Cout x 27*Cin) += dy^T . col, with col = im2col(x) recomputed into d_col.
int tigre_conv3d_bwd_weight(const void* d_x, const void* d_dy, float* d_dw, long D, long H, long W, long Cin,
                            long Cout, void* d_col, void* stream) {
    TIGRE_NVTX("tigre_conv3d_bwd_weight");
    if (!d_x || !d_dy || !d_dw || !d_col || D <= 0 || H <= 0 || W <= 0 || Cin <= 0 || Cout <= 0)
        return fail(TIGRE_ERR_BAD_ASSERT, "bad conv3d arguments");
    const long M = D * H * W, K = 27 * Cin;
    cudaStream_t st = (cudaStream_t)stream;
    im2col_kernel<<<grid_for_conv(M * K), 256, 0, st>>>((const __nv_bfloat16*)d_x, (__nv_bfloat16*)d_col, (int)D,
                                                        (int)H, (int)W, (int)Cin);
    TIGRE_LAUNCHED();
    // The reduction runs over the M voxels.  It is split over blocks, each writing its partial
    // dw to its own slice of a stream-ordered workspace, and the slices are then summed in a
    // fixed order: the result does not depend on the blocks' timing (no atomics).
    const long per = (long)Cout * K;
    long splits = std::max(1L, std::min<long>((M + 4095) / 4096, 256));
    while (splits > 1 && splits * per > (1L << 26)) splits = (splits + 1) / 2;   // <= 256 MB of workspace
    const long chunk = (M + splits - 1) / splits;
    splits = (M + chunk - 1) / chunk;
    float* ws = nullptr;
    TIGRE_CUDA(cudaMallocAsync(&ws, sizeof(float) * (size_t)(splits * per), st));
    dim3 grid((unsigned)((Cout + kBM - 1) / kBM), (unsigned)((K + kBN - 1) / kBN), (unsigned)splits);
    // op(A) = dy^T (Cout x M): stored M x Cout row-major -> element (i=co, k=v) at dy[v * Cout + co];
    // block z writes rows [0, Cout) x [0, K) of slice z (gemm_kernel's split index offsets K only,
    // so each slice is addressed through its own C pointer below)
    gemm_kernel<false, false><<<grid, kThreads, 0, st>>>((const __nv_bfloat16*)d_dy, (int)Cout,
                                                        (const __nv_bfloat16*)d_col, (int)K, ws, nullptr, (int)K,
                                                        (int)Cout, (int)K, (int)M, nullptr, 0, (int)chunk, 2);
    TIGRE_LAUNCHED();
    reduce_slices_kernel<<<grid_for_conv(per), 256, 0, st>>>(ws, d_dw, per, splits);
    TIGRE_LAUNCHED();
    TIGRE_CUDA(cudaFreeAsync(ws, st));
    return TIGRE_SUCCESS;
}

}  // extern "C"
