// kpcnn.cu -- the learned denoiser: a kernel-predicting CNN (3 x conv3x3
// with 32 channels and ReLU, a 3x3 head of 25 logits, a per-pixel softmax
// 5x5 filter applied to the noisy radiance), with BF16 operands and FP32
// accumulation on the tcgen05 tensor cores, for inference and training.
// The reference has no learned denoiser; this is new work beside its
// à-trous filter (post/atrous_denoise.frag), which stays the fallback.
//
// Data layout (HBM):
//   activations   NHWC bf16, C = 16 (network input: log1p radiance, albedo,
//                 normal, depth, 6 zero channels) or 32 (hidden layers)
//   logits        NHWC fp32, 32 channels (25 used)
//   radiance      float4 per pixel (rgb, unused w)
//   parameters    one fp32 vector (RC_KPCNN_PARAMS floats): per layer
//                 W[tap][co][ci] (tap = 3*dy + dx) then bias[co]
//   packed        bf16 copies of each W in the tensor cores' K-major
//                 operand layout [tap][ci/8][co][8], plus for layers 2, 3
//                 and the head the flipped/transposed copy used by the
//                 backward-data convolution
//
// Kernels:
//   conv3x3_kernel<CIN>  implicit GEMM, one CTA per 128 pixels of an image
//                        row: D[128 px][32 co] = sum over 9 taps and CIN/16
//                        k-steps of A[px][16 ci] x B[16 ci][32 co].  The
//                        three input rows (130 px with the halo) sit in
//                        shared memory channel-group-major, pixel-contiguous
//                        ([row][ci/8][px][8 ci], 16 B per pixel and group), so
//                        the A operand of horizontal tap dx is the same
//                        K-major matrix shifted by dx * 16 bytes.  Epilogue:
//                        bias, ReLU or ReLU-mask (backward), bf16 or fp32.
//   wgrad_kernel<CIN>    dW[tap][co][ci] = sum_px dY[px][co] X[px+tap][ci]:
//                        M = (tap, ci) in tiles of 128, N = 32 co, K = pixels,
//                        both operands MN-major tiles of 128 pixels, FP32
//                        partial sums atomically added per CTA; bias grads
//                        from the same staged dY.
//   head_kernel          softmax over 25 logits, the 5x5 filter (edge
//                        clamped), and for training the relative-MSE loss
//                        (x-r)^2/(r^2+0.01) with its gradient w.r.t. logits.
//   features / crop / pack / adam   small SIMT kernels.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "retrocam.h"
#include "host_checks.h"
#include "tc_sm100.cuh"

namespace rc {
namespace kp {

constexpr int kTile = 128;          // pixels per CTA (one row segment)
constexpr int kHalo = kTile + 2;    // staged pixels per row
constexpr int kPStride = 136;       // staged row pitch in 16-byte units
constexpr int kCo = 32;             // output channels of every convolution
constexpr uint32_t kWaitTries = 1u << 20;   // bounded mbarrier polls

constexpr int kParamW1 = 0, kParamB1 = kParamW1 + 9 * 32 * 16;
constexpr int kParamW2 = kParamB1 + 32, kParamB2 = kParamW2 + 9 * 32 * 32;
constexpr int kParamW3 = kParamB2 + 32, kParamB3 = kParamW3 + 9 * 32 * 32;
constexpr int kParamWH = kParamB3 + 32, kParamBH = kParamWH + 9 * 32 * 32;
constexpr int kParams = kParamBH + 32;
static_assert(kParams == RC_KPCNN_PARAMS, "parameter layout");

struct ConvArgs {
    const __nv_bfloat16* in;    // NHWC, CIN channels
    const __nv_bfloat16* wpk;   // packed [9][CIN/8][32][8]
    const float* bias;          // 32 or null
    void* out;                  // NHWC 32 channels, bf16 or fp32
    const __nv_bfloat16* mask;  // NHWC 32 channels: out *= (mask > 0), or null
    int n, h, w;
    int relu;
    int out_f32;
    unsigned int* err;
    // inference head fused into the epilogue (head_kernel without a
    // target): the 32 outputs are the logits, head_out gets the filtered
    // head_color and `out` is not written; null: plain convolution
    const float4* head_color;
    float4* head_out;
};

// The network's head: softmax of 25 logits (in place: the normalised
// weights) and the 5x5 filter of the noisy colour of image `img` with them,
// edges clamped.
// The 5x5 neighbourhood of (y, x) in img (rgb), edges clamped.
__device__ __forceinline__ void head_taps(const float4* __restrict__ img, int y, int x, int h, int w,
                                          float3 (&c)[25]) {
#pragma unroll
    for (int t = 0; t < 25; ++t) {
        const int yy = min(max(y + t / 5 - 2, 0), h - 1), xx = min(max(x + t % 5 - 2, 0), w - 1);
        const float4 v = __ldg(img + (size_t)yy * w + xx);
        c[t] = make_float3(v.x, v.y, v.z);
    }
}

__device__ __forceinline__ float3 head_filter(float (&l)[25], const float3 (&c)[25]) {
    float m = l[0];
#pragma unroll
    for (int t = 1; t < 25; ++t) m = fmaxf(m, l[t]);
    float s = 0.0f;
#pragma unroll
    for (int t = 0; t < 25; ++t) {
        l[t] = __expf(l[t] - m);
        s += l[t];
    }
    const float inv = 1.0f / s;
    float3 o = make_float3(0.0f, 0.0f, 0.0f);
#pragma unroll
    for (int t = 0; t < 25; ++t) {
        l[t] *= inv;
        o.x += l[t] * c[t].x;
        o.y += l[t] * c[t].y;
        o.z += l[t] * c[t].z;
    }
    return o;
}

__device__ __forceinline__ float3 apply_head(float (&l)[25], const float4* __restrict__ img, int y, int x, int h,
                                             int w) {
    float3 c[25];
    head_taps(img, y, x, h, w, c);
    return head_filter(l, c);
}

// Shared memory of the convolution: a ring of five staged image rows (the
// three of the tile being multiplied and the new rows of the next two tiles,
// in flight; the previous tile's first row gives its slot up once that
// tile's MMAs are done), the weights, and the mbarriers: one per ring slot
// (its row has landed), one per TMEM accumulator for "MMAs done" and one per
// accumulator for "epilogue read it".  A slot is one row of kHalo pixels,
// channel-group-major: [CIN/8][kPStride][16 B].
constexpr int kAhead = 2;             // row copies in flight ahead of the tile
constexpr int kSlots = 3 + kAhead;

template <int CIN>
struct ConvSmem {
    alignas(128) uint4 rows[kSlots][(CIN / 8) * kPStride];
    alignas(128) uint4 wts[9 * (CIN / 8) * kCo];
    uint64_t full[kSlots];
    uint64_t mbar[2];
    uint64_t empty[2];
    uint32_t tmem;
};

// Image row y (pixels x0-1 .. x0+128) of image n into a slot, as CIN/8 TMA
// boxes of 8 channels x kHalo pixels (channel group g lands at [g][0..129]);
// pixels and rows outside the image read as zero.  One thread.
template <int CIN>
__device__ __forceinline__ void produce_row(const void* tmap, uint4* slot, uint64_t* full, int n, int y, int x0) {
    constexpr int G = CIN / 8;
    tc::mbar_arrive_expect_tx(full, G * kHalo * 16);
#pragma unroll
    for (int g = 0; g < G; ++g) tc::tma_load_4d(tc::smem_u32(slot + g * kPStride), tmap, 8 * g, x0 - 1, y, n, full);
}

// The 9 taps x CIN/16 k-steps of one tile: rows[dy] is the slot of image row
// y - 1 + dy; the A operand of tap (dy, dx) is that slot shifted by dx pixels.
// A descriptor's start address is its low 14 bits (address / 16; shared
// memory is below 256 KB), so the descriptor of base + offset is the base
// descriptor plus offset / 16: each MMA adds a compile-time constant.
template <int CIN>
__device__ __forceinline__ void issue_tile(const uint32_t (&rows)[3], uint32_t wts, uint32_t tmem_d, uint64_t* mbar) {
    constexpr int G = CIN / 8;   // 16-byte channel groups per pixel (two per k-step)
    constexpr uint32_t idesc = tc::idesc_bf16(128, kCo, false, false);
    const uint64_t da[3] = {tc::smem_desc(rows[0], kPStride * 16, 128), tc::smem_desc(rows[1], kPStride * 16, 128),
                            tc::smem_desc(rows[2], kPStride * 16, 128)};
    const uint64_t db = tc::smem_desc(wts, kCo * 16, 128);
#pragma unroll
    for (int tap = 0; tap < 9; ++tap) {
        const int dy = tap / 3, dx = tap - 3 * dy;
#pragma unroll
        for (int ks = 0; ks < CIN / 16; ++ks) {
            const uint64_t a = da[dy] + (uint64_t)((2 * ks) * kPStride + dx);
            const uint64_t b = db + (uint64_t)((tap * G + 2 * ks) * kCo);
            tc::mma_bf16(tmem_d, a, b, idesc, (tap | ks) != 0);
        }
    }
    tc::mma_commit(mbar);
}

// The head's radiance taps of this thread's pixel of tile t (HEAD only),
// loaded before the tile's MMAs are waited for so their latency overlaps.
template <bool HEAD>
__device__ __forceinline__ void epilogue_taps(const ConvArgs& A, int t, int tiles_x, float3 (&c)[25]) {
    if (!HEAD) return;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int xt = t % tiles_x, rest = t / tiles_x;
    const int y = rest % A.h, n = rest / A.h;
    const int x = xt * kTile + warp * 32 + lane;
    if (x >= A.w) return;
    head_taps(A.head_color + (size_t)n * A.h * A.w, y, x, A.h, A.w, c);
}

template <bool HEAD>
__device__ __forceinline__ void conv_epilogue(const ConvArgs& A, const float (&vin)[32], int t, int tiles_x,
                                              const float3 (&taps)[25]) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int xt = t % tiles_x, rest = t / tiles_x;
    const int y = rest % A.h, n = rest / A.h;
    const int x = xt * kTile + warp * 32 + lane;
    if (x >= A.w) return;
    float v[32];
#pragma unroll
    for (int c = 0; c < 32; ++c) v[c] = vin[c];
    const size_t pix = ((size_t)n * A.h + y) * A.w + x;
    if (A.bias) {
#pragma unroll
        for (int c = 0; c < 32; ++c) v[c] += __ldg(A.bias + c);
    }
    if (A.relu) {
#pragma unroll
        for (int c = 0; c < 32; ++c) v[c] = fmaxf(v[c], 0.0f);
    }
    if (A.mask) {
        const uint4* m = reinterpret_cast<const uint4*>(A.mask + pix * 32);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const uint4 mv = __ldg(m + q);
            const uint32_t w4[4] = {mv.x, mv.y, mv.z, mv.w};
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const __nv_bfloat162 h2 = *reinterpret_cast<const __nv_bfloat162*>(&w4[j]);
                if (!(__bfloat162float(h2.x) > 0.0f)) v[q * 8 + 2 * j] = 0.0f;
                if (!(__bfloat162float(h2.y) > 0.0f)) v[q * 8 + 2 * j + 1] = 0.0f;
            }
        }
    }
    if (HEAD) {
        float l[25];
#pragma unroll
        for (int t = 0; t < 25; ++t) l[t] = v[t];
        const float3 o = head_filter(l, taps);
        A.head_out[pix] = make_float4(o.x, o.y, o.z, 1.0f);
        return;
    }
    if (A.out_f32) {
        float4* o = reinterpret_cast<float4*>(static_cast<float*>(A.out) + pix * 32);
#pragma unroll
        for (int q = 0; q < 8; ++q) o[q] = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
    } else {
        uint4* o = reinterpret_cast<uint4*>(static_cast<__nv_bfloat16*>(A.out) + pix * 32);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            uint32_t w4[4];
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const __nv_bfloat162 h2 = __floats2bfloat162_rn(v[q * 8 + 2 * j], v[q * 8 + 2 * j + 1]);
                w4[j] = *reinterpret_cast<const uint32_t*>(&h2);
            }
            o[q] = make_uint4(w4[0], w4[1], w4[2], w4[3]);
        }
    }
}

// Implicit-GEMM convolution over column strips: CTA s takes a segment of
// `seg_rows` consecutive image rows of one 128-pixel-wide strip, so the
// tiles it walks share rows -- tile y needs rows y-1..y+1 and only row y+1 is
// new.  Thread 0 is the producer and the MMA issuer: at step k it waits for
// the rows of tile k (TMA, per-slot mbarrier) and for the epilogues of tile
// k-2 to have read accumulator k&1, issues the MMAs of tile k, and once tile
// k-1's MMAs are done loads the new row of tile k+2 into the slot tile k-1
// read first.  Every warp drains its quarter of tile k-1's accumulator in
// the meantime, so no step passes a CTA-wide barrier.  All waits are
// bounded; a timeout sets RC_GUARD_MMA_WAIT and the CTA winds down after
// waiting (bounded) for the copies and MMAs it started.
template <int CIN, bool HEAD>
__global__ void __launch_bounds__(128)
    conv3x3_kernel(ConvArgs A, int seg_rows, const __grid_constant__ CUtensorMap tmap) {
    extern __shared__ __align__(128) unsigned char conv_smem_raw[];
    // TMA destinations start on 128-byte boundaries (the launch adds 128
    // bytes of slack for this)
    unsigned char* smem_base = conv_smem_raw + ((128u - (tc::smem_u32(conv_smem_raw) & 127u)) & 127u);
    ConvSmem<CIN>& S = *reinterpret_cast<ConvSmem<CIN>*>(smem_base);
    constexpr int G = CIN / 8;
    constexpr uint32_t FULL = 0xffffffffu;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int tiles_x = (A.w + kTile - 1) / kTile;
    const int segs = (A.h + seg_rows - 1) / seg_rows;       // segments per strip
    const int strip = blockIdx.x / segs;                    // (image, column) strip
    const int n = strip / tiles_x, xt = strip - n * tiles_x;
    const int y0 = (blockIdx.x - strip * segs) * seg_rows;
    const int rows_here = min(seg_rows, A.h - y0);
    if (n >= A.n || rows_here <= 0) return;
    const int x0 = xt * kTile;
    const void* tm = &tmap;
    if (warp == 0) tc::tmem_alloc(&S.tmem, 64);
    if (tid == 0) {
        for (int i = 0; i < kSlots; ++i) tc::mbar_init(&S.full[i], 1);
        for (int a = 0; a < 2; ++a) {
            tc::mbar_init(&S.mbar[a], 1);
            tc::mbar_init(&S.empty[a], 4);    // one arrival per warp
        }
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = S.tmem;
    const uint32_t wts = tc::smem_u32(S.wts);
    // image row y0 - 1 + j lives in slot j % kSlots, its fill number j / kSlots
    int produced = -1, consumed = -1;   // thread 0: rows loaded / waited for
    if (tid == 0) {
        // the weights ride on the first row's barrier (whose one arrival is
        // produce_row's)
        tc::mbar_expect_tx(&S.full[0], 9 * G * kCo * 16);
        tc::bulk_load(wts, A.wpk, 9 * G * kCo * 16, &S.full[0]);
        for (int j = 0; j < 3 + kAhead - 1 && j < rows_here + 2; ++j) {
            produce_row<CIN>(tm, S.rows[j], &S.full[j], n, y0 - 1 + j, x0);
            produced = j;
        }
    }
    bool ok = true;       // warp-uniform
    bool ok0 = true;      // thread 0's own waits
    int k = 0;
    for (; k < rows_here; ++k) {
        const int acc = k & 1;
        const int y = y0 + k;
        if (tid == 0) {
            // rows k..k+2 of tile k (only row k+2 is new after tile 0)
            for (int j = k == 0 ? 0 : k + 2; j <= k + 2 && ok0; ++j) {
                ok0 = tc::mbar_wait(&S.full[j % kSlots], (uint32_t)(j / kSlots) & 1u, kWaitTries);
                if (ok0) consumed = j;
            }
            // accumulator acc was last read by the epilogues of tile k-2
            if (ok0 && k >= 2) ok0 = tc::mbar_wait(&S.empty[acc], (uint32_t)((k - 2) >> 1) & 1u, kWaitTries);
            if (ok0) {
                tc::fence_after_sync();
                const uint32_t rows[3] = {tc::smem_u32(S.rows[k % kSlots]), tc::smem_u32(S.rows[(k + 1) % kSlots]),
                                          tc::smem_u32(S.rows[(k + 2) % kSlots])};
                issue_tile<CIN>(rows, wts, tmem + acc * 32, &S.mbar[acc]);
            }
        }
        if (k == 0) {
            if (tid == 0 && ok0 && kAhead < rows_here) {
                produce_row<CIN>(tm, S.rows[2 + kAhead], &S.full[2 + kAhead], n, y + 1 + kAhead, x0);
                produced = 2 + kAhead;
            }
            ok = __all_sync(FULL, ok0);
            if (!ok) break;
            continue;
        }
        // epilogue of tile k-1 while the tensor cores work on tile k
        const int pa = acc ^ 1;
        float3 taps[25];
        epilogue_taps<HEAD>(A, ((n * A.h) + y - 1) * tiles_x + xt, tiles_x, taps);
        ok = __all_sync(FULL, ok0 && tc::mbar_wait(&S.mbar[pa], (uint32_t)((k - 1) >> 1) & 1u, kWaitTries));
        if (!ok) break;
        tc::fence_after_sync();
        // tile k-1's MMAs are done with its first row: that slot takes the
        // new row of tile k + kAhead
        if (tid == 0 && k + kAhead < rows_here) {
            const int j = k + 2 + kAhead;
            produce_row<CIN>(tm, S.rows[j % kSlots], &S.full[j % kSlots], n, y + 1 + kAhead, x0);
            produced = j;
        }
        float v[32];
        tc::tmem_ld32(tmem + pa * 32 + (static_cast<uint32_t>(warp * 32) << 16), v);
        tc::fence_before_sync();
        __syncwarp();
        if (lane == 0) tc::mbar_arrive(&S.empty[pa]);
        conv_epilogue<HEAD>(A, v, ((n * A.h) + y - 1) * tiles_x + xt, tiles_x, taps);
    }
    // epilogue of the last tile
    if (ok && k > 0) {
        const int pa = (k - 1) & 1;
        float3 taps[25];
        epilogue_taps<HEAD>(A, ((n * A.h) + y0 + k - 1) * tiles_x + xt, tiles_x, taps);
        ok = __all_sync(FULL, tc::mbar_wait(&S.mbar[pa], (uint32_t)((k - 1) >> 1) & 1u, kWaitTries));
        if (ok) {
            tc::fence_after_sync();
            float v[32];
            tc::tmem_ld32(tmem + pa * 32 + (static_cast<uint32_t>(warp * 32) << 16), v);
            conv_epilogue<HEAD>(A, v, ((n * A.h) + y0 + k - 1) * tiles_x + xt, tiles_x, taps);
        }
    }
    ok = __syncthreads_and(ok);
    if (!ok) {
        if (tid == 0) {
            atomicOr(A.err, RC_GUARD_MMA_WAIT);
            // rows still in flight land before the shared memory is released
            for (int j = consumed + 1; j <= produced; ++j)
                (void)tc::mbar_wait(&S.full[j % kSlots], (uint32_t)(j / kSlots) & 1u, kWaitTries);
        }
        // MMAs still in flight get a bounded time before the columns go
        for (int a = 0; a < 2; ++a) (void)tc::mbar_wait(&S.mbar[a], (uint32_t)(k >> 1) & 1u, kWaitTries);
    }
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) tc::tmem_dealloc(tmem, 64);
}

// ---------------------------------------------------------------------------
// weight gradients
// ---------------------------------------------------------------------------
struct WgradArgs {
    const __nv_bfloat16* x;    // NHWC CIN: the layer's input
    const __nv_bfloat16* dy;   // NHWC 32: gradient at the layer's pre-activation
    float* dw;                 // [9][32][CIN] (+=)
    float* db;                 // [32] (+=)
    int n, h, w;
    unsigned int* err;
};

struct WgradSmem {
    alignas(128) uint4 a[16 * kTile];   // [m/8][px][8]: im2col of X for one M tile
    alignas(128) uint4 b[4 * kTile];    // [co/8][px][8]: dY
    uint64_t mbar;
    uint32_t tmem;
};

template <int CIN>
__global__ void __launch_bounds__(128) wgrad_kernel(WgradArgs A) {
    constexpr int G = CIN / 8;
    constexpr int T = 128 / CIN;             // taps per M tile
    constexpr int MT = (9 + T - 1) / T;      // M tiles
    constexpr int NCOL = MT * 32 <= 32 ? 32 : (MT * 32 <= 64 ? 64 : 128);
    __shared__ WgradSmem S;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    if (warp == 0) tc::tmem_alloc(&S.tmem, NCOL);
    if (tid == 0) tc::mbar_init(&S.mbar, 1);
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = S.tmem;
    const int tiles_x = (A.w + kTile - 1) / kTile;
    const int ntiles = tiles_x * A.h * A.n;
    const uint4 zero = make_uint4(0u, 0u, 0u, 0u);
    constexpr uint32_t idesc = tc::idesc_bf16(128, kCo, true, true);
    float bsum[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    uint32_t phase = 0;
    bool ok = true;
    int issued = 0;
    for (int t = blockIdx.x; t < ntiles && ok; t += gridDim.x) {
        const int xt = t % tiles_x, rest = t / tiles_x;
        const int y = rest % A.h, n = rest / A.h;
        const int x0 = xt * kTile;
        // dY tile, channel-group-major; bias sums per thread (fixed group)
        for (int i = tid; i < 4 * kTile; i += 128) {
            const int p = i >> 2, g = i & 3;
            const int xx = x0 + p;
            uint4 v = zero;
            if (xx < A.w) v = __ldg(reinterpret_cast<const uint4*>(A.dy + (((size_t)n * A.h + y) * A.w + xx) * 32) + g);
            S.b[g * kTile + p] = v;
            const uint32_t w4[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const __nv_bfloat162 h2 = *reinterpret_cast<const __nv_bfloat162*>(&w4[j]);
                bsum[2 * j] += __bfloat162float(h2.x);
                bsum[2 * j + 1] += __bfloat162float(h2.y);
            }
        }
        for (int mt = 0; mt < MT && ok; ++mt) {
            if (issued > 0) {   // the previous MMAs still read S.a / S.b
                ok = __syncthreads_and(tc::mbar_wait(&S.mbar, phase, kWaitTries));
                phase ^= 1u;
                tc::fence_after_sync();
                if (!ok) break;
            }
            for (int i = tid; i < 16 * kTile; i += 128) {
                const int p = i / 16, mg = i - 16 * p;   // group fastest: 16 B pieces of one pixel
                const int tl = mg / G, g = mg - tl * G;
                const int tap = mt * T + tl;
                uint4 v = zero;
                if (tap < 9) {
                    const int dy = tap / 3, dx = tap - 3 * dy;
                    const int yy = y + dy - 1, xx = x0 + p + dx - 1;
                    if (yy >= 0 && yy < A.h && xx >= 0 && xx < A.w && x0 + p < A.w)
                        v = __ldg(reinterpret_cast<const uint4*>(A.x + (((size_t)n * A.h + yy) * A.w + xx) * CIN) + g);
                }
                S.a[mg * kTile + p] = v;
            }
            tc::fence_async_smem();
            tc::fence_before_sync();
            __syncthreads();
            tc::fence_after_sync();
            if (tid == 0) {
                const uint32_t sa = tc::smem_u32(S.a), sb = tc::smem_u32(S.b);
#pragma unroll
                for (int ks = 0; ks < kTile / 16; ++ks) {
                    const uint64_t a = tc::smem_desc(sa + ks * 256, 128, kTile * 16);
                    const uint64_t b = tc::smem_desc(sb + ks * 256, 128, kTile * 16);
                    tc::mma_bf16(tmem + mt * 32, a, b, idesc, (t != (int)blockIdx.x || ks > 0) ? 1u : 0u);
                }
                tc::mma_commit(&S.mbar);
            }
            ++issued;
        }
        if (!ok) break;
        // the next tile overwrites S.b: wait for this tile's last MMAs
        ok = __syncthreads_and(tc::mbar_wait(&S.mbar, phase, kWaitTries));
        phase ^= 1u;
        issued = 0;
        tc::fence_after_sync();
        __syncthreads();
    }
    if (!ok) {
        if (tid == 0) atomicOr(A.err, RC_GUARD_MMA_WAIT);
    } else if ((int)blockIdx.x < ntiles) {
        // bias: reduce the 8 sums of threads sharing a channel group (lane % 4)
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            float s = bsum[j];
            s += __shfl_xor_sync(0xffffffffu, s, 4);
            s += __shfl_xor_sync(0xffffffffu, s, 8);
            s += __shfl_xor_sync(0xffffffffu, s, 16);
            if (lane < 4) atomicAdd(A.db + lane * 8 + j, s);
        }
        for (int mt = 0; mt < MT; ++mt) {
            float v[32];
            tc::tmem_ld32(tmem + (static_cast<uint32_t>(warp * 32) << 16) + mt * 32, v);
            const int m = warp * 32 + lane;
            const int tl = m / CIN, ci = m - tl * CIN;
            const int tap = mt * T + tl;
            if (tap < 9) {
#pragma unroll
                for (int co = 0; co < 32; ++co) atomicAdd(A.dw + (tap * 32 + co) * CIN + ci, v[co]);
            }
        }
    }
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) tc::tmem_dealloc(tmem, NCOL);
}

// ---------------------------------------------------------------------------
// head: softmax 5x5 filter, loss and its gradient
// ---------------------------------------------------------------------------
struct HeadArgs {
    const float* logits;        // NHWC 32 (25 used)
    const float4* color;        // noisy radiance
    const float4* target;       // reference radiance, or null (inference)
    float4* out;                // filtered radiance (w = 1)
    __nv_bfloat16* dlogits;     // NHWC 32, or null
    double* loss;               // sum of per-channel relative squared errors, or null
    float grad_scale;           // d(total loss)/d(per-channel term)
    int n, h, w;
};

__global__ void __launch_bounds__(128) head_kernel(HeadArgs A) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y, n = blockIdx.z;
    float lsum = 0.0f;
    if (x < A.w) {
        const size_t pix = ((size_t)n * A.h + y) * A.w + x;
        float l[25];
        const float4* lg = reinterpret_cast<const float4*>(A.logits + pix * 32);
#pragma unroll
        for (int q = 0; q < 6; ++q) {
            const float4 v = lg[q];
            l[4 * q] = v.x;
            l[4 * q + 1] = v.y;
            l[4 * q + 2] = v.z;
            l[4 * q + 3] = v.w;
        }
        l[24] = lg[6].x;
        const size_t img = (size_t)n * A.h * A.w;
        const float3 o = apply_head(l, A.color + img, y, x, A.h, A.w);
        A.out[pix] = make_float4(o.x, o.y, o.z, 1.0f);
        if (A.target) {
            const float4 r = __ldg(A.target + pix);
            const float dr = o.x - r.x, dg = o.y - r.y, db = o.z - r.z;
            const float qr = 1.0f / (r.x * r.x + 0.01f), qg = 1.0f / (r.y * r.y + 0.01f),
                        qb = 1.0f / (r.z * r.z + 0.01f);
            lsum = dr * dr * qr + dg * dg * qg + db * db * qb;
            if (A.dlogits) {
                const float gx = 2.0f * dr * qr * A.grad_scale, gy = 2.0f * dg * qg * A.grad_scale,
                            gz = 2.0f * db * qb * A.grad_scale;
                float dw[25], wsum = 0.0f;
#pragma unroll
                for (int t = 0; t < 25; ++t) {
                    const int yy = min(max(y + t / 5 - 2, 0), A.h - 1), xx = min(max(x + t % 5 - 2, 0), A.w - 1);
                    const float4 c = __ldg(A.color + img + (size_t)yy * A.w + xx);
                    dw[t] = gx * c.x + gy * c.y + gz * c.z;
                    wsum += l[t] * dw[t];
                }
                uint32_t packed[16];
#pragma unroll
                for (int j = 0; j < 16; ++j) {
                    const float a = 2 * j < 25 ? l[2 * j] * (dw[2 * j] - wsum) : 0.0f;
                    const float b = 2 * j + 1 < 25 ? l[2 * j + 1] * (dw[2 * j + 1] - wsum) : 0.0f;
                    const __nv_bfloat162 h2 = __floats2bfloat162_rn(a, b);
                    packed[j] = *reinterpret_cast<const uint32_t*>(&h2);
                }
                uint4* d = reinterpret_cast<uint4*>(A.dlogits + pix * 32);
#pragma unroll
                for (int q = 0; q < 4; ++q)
                    d[q] = make_uint4(packed[4 * q], packed[4 * q + 1], packed[4 * q + 2], packed[4 * q + 3]);
            }
        }
    }
    if (A.loss) {
        __shared__ float red[4];
        float v = lsum;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
        __syncthreads();
        if (threadIdx.x == 0) atomicAdd(A.loss, (double)(red[0] + red[1] + red[2] + red[3]));
    }
}

// ---------------------------------------------------------------------------
// features, crops, packing, optimizer
// ---------------------------------------------------------------------------
__device__ __forceinline__ float h2f(unsigned short u) { return __half2float(__ushort_as_half(u)); }

// Network input from a context's images: log1p radiance, albedo, normal,
// depth mapped to t/(1+t); plus the radiance itself for the filter.
__global__ void features_kernel(const float4* __restrict__ accum, const ushort4* __restrict__ gbuf,
                                const ushort4* __restrict__ galb, __nv_bfloat16* __restrict__ feat,
                                float4* __restrict__ color, int count) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const float4 a = accum[i];
    const float inv = 1.0f / fmaxf(a.w, 1.0f);
    const float r = a.x * inv, g = a.y * inv, b = a.z * inv;
    color[i] = make_float4(r, g, b, 1.0f);
    const ushort4 gb = gbuf[i], ga = galb[i];
    const float t = h2f(gb.w);
    float f[16] = {log1pf(fmaxf(r, 0.0f)), log1pf(fmaxf(g, 0.0f)), log1pf(fmaxf(b, 0.0f)), h2f(ga.x), h2f(ga.y),
                   h2f(ga.z), h2f(gb.x), h2f(gb.y), h2f(gb.z), t / (1.0f + fabsf(t)), 0, 0, 0, 0, 0, 0};
    uint32_t p[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        const __nv_bfloat162 h2 = __floats2bfloat162_rn(f[2 * j], f[2 * j + 1]);
        p[j] = *reinterpret_cast<const uint32_t*>(&h2);
    }
    uint4* o = reinterpret_cast<uint4*>(feat + (size_t)i * 16);
    o[0] = make_uint4(p[0], p[1], p[2], p[3]);
    o[1] = make_uint4(p[4], p[5], p[6], p[7]);
}

// Training crops: crop b copies the size x size window at (oy, ox) of input
// image src[b] (features + radiance) and of target image tgt[b].
__global__ void crop_kernel(const __nv_bfloat16* __restrict__ feat_all, const float4* __restrict__ color_all,
                            const float4* __restrict__ target_all, const int* __restrict__ src,
                            const int* __restrict__ tgt, const int* __restrict__ oy, const int* __restrict__ ox,
                            int H, int W, int size, __nv_bfloat16* __restrict__ feat, float4* __restrict__ color,
                            float4* __restrict__ target) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y, b = blockIdx.z;
    if (x >= size) return;
    const size_t s = ((size_t)src[b] * H + oy[b] + y) * W + ox[b] + x;
    const size_t r = ((size_t)tgt[b] * H + oy[b] + y) * W + ox[b] + x;
    const size_t d = ((size_t)b * size + y) * size + x;
    const uint4* fi = reinterpret_cast<const uint4*>(feat_all + s * 16);
    uint4* fo = reinterpret_cast<uint4*>(feat + d * 16);
    fo[0] = fi[0];
    fo[1] = fi[1];
    color[d] = color_all[s];
    target[d] = target_all[r];
}

// fp32 parameters -> bf16 operand copies.  Forward layout [tap][ci/8][co][8];
// backward-data layout [tap][co/8][ci][8] with tap flipped (8 - tap).
__global__ void pack_kernel(const float* __restrict__ params, __nv_bfloat16* __restrict__ w1,
                            __nv_bfloat16* __restrict__ w2, __nv_bfloat16* __restrict__ w3,
                            __nv_bfloat16* __restrict__ wh, __nv_bfloat16* __restrict__ w2b,
                            __nv_bfloat16* __restrict__ w3b, __nv_bfloat16* __restrict__ whb) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e < 9 * 32 * 16) {
        const int tap = e / 512, rem = e % 512, g = rem / 256, co = (rem % 256) / 8, j = rem % 8;
        w1[e] = __float2bfloat16_rn(params[kParamW1 + (tap * 32 + co) * 16 + g * 8 + j]);
    }
    if (e < 9 * 32 * 32) {
        const int tap = e / 1024, rem = e % 1024, g = rem / 256, r = (rem % 256) / 8, j = rem % 8;
        // forward: r = co, channel g*8+j = ci
        w2[e] = __float2bfloat16_rn(params[kParamW2 + (tap * 32 + r) * 32 + g * 8 + j]);
        w3[e] = __float2bfloat16_rn(params[kParamW3 + (tap * 32 + r) * 32 + g * 8 + j]);
        wh[e] = __float2bfloat16_rn(params[kParamWH + (tap * 32 + r) * 32 + g * 8 + j]);
        // backward: r = ci (output of the transposed conv), g*8+j = co
        const int src = ((8 - tap) * 32 + g * 8 + j) * 32 + r;
        w2b[e] = __float2bfloat16_rn(params[kParamW2 + src]);
        w3b[e] = __float2bfloat16_rn(params[kParamW3 + src]);
        whb[e] = __float2bfloat16_rn(params[kParamWH + src]);
    }
}

__global__ void adam_kernel(float* __restrict__ p, float* __restrict__ g, float* __restrict__ m,
                            float* __restrict__ v, int count, float lr, float b1, float b2, float eps, float c1,
                            float c2) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.0f - b1) * gi;
    const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi * c1) / (sqrtf(vi * c2) + eps);
    g[i] = 0.0f;
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
// cuTensorMapEncodeTiled from the driver (the library links only the
// runtime), looked up once.
static PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
    static const PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            p = nullptr;
        return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }();
    return fn;
}

// A convolution's input as a 4-D tensor map (channels, pixels, rows, images;
// NHWC bf16) read in boxes of 8 channels x kHalo pixels of one row, no
// swizzle, zeros outside.  The ABI checks that the input is 16-byte
// aligned; every row pitch is a multiple of 16 bytes (CIN * 2 per pixel).
template <int CIN>
static cudaError_t conv_tensor_map(const ConvArgs& A, CUtensorMap* m) {
    const PFN_cuTensorMapEncodeTiled_v12000 enc = tensor_map_encoder();
    if (!enc) return cudaErrorNotSupported;
    const cuuint64_t dims[4] = {(cuuint64_t)CIN, (cuuint64_t)A.w, (cuuint64_t)A.h, (cuuint64_t)A.n};
    const cuuint64_t strides[3] = {(cuuint64_t)CIN * 2, (cuuint64_t)A.w * CIN * 2, (cuuint64_t)A.h * A.w * CIN * 2};
    const cuuint32_t box[4] = {8, (cuuint32_t)kHalo, 1, 1};
    const cuuint32_t elem[4] = {1, 1, 1, 1};
    const CUresult r = enc(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<__nv_bfloat16*>(A.in), dims, strides, box,
                           elem, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                           CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}

template <int CIN, bool HEAD>
static cudaError_t launch_conv_t(const ConvArgs& A, cudaStream_t s) {
    // resident CTAs per SM, found (and the shared-memory limit raised) once
    // per device and instantiation
    static int per_device[64] = {};
    const size_t smem = sizeof(ConvSmem<CIN>) + 128;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    int scratch = 0;
    int& per = dev >= 0 && dev < 64 ? per_device[dev] : scratch;
    if (per == 0) {
        cudaError_t e = cudaFuncSetAttribute(conv3x3_kernel<CIN, HEAD>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(conv3x3_kernel<CIN, HEAD>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                     (int)cudaSharedmemCarveoutMaxShared);
        if (e != cudaSuccess) return e;
        // shared memory bounds the CTAs per SM (3 with 32 input channels);
        // registers allow 7 of 128 threads and TMEM 8 of 64 columns
        int smem_sm = 0;
        cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
        per = (int)(smem_sm / (smem + 1024));   // 1 KB reserved per CTA
        if (per < 1) per = 1;
        if (per > 7) per = 7;
    }
    // one segment per resident CTA: rows per segment so that the strips'
    // segments fill the GPU once
    const int strips = ((A.w + kTile - 1) / kTile) * A.n;
    const int cap = sms * per;
    if (strips <= 0 || A.h <= 0) return cudaSuccess;
    int seg_rows = (int)(((long)strips * A.h + cap - 1) / cap);
    if (seg_rows < 1) seg_rows = 1;
    const int grid = strips * ((A.h + seg_rows - 1) / seg_rows);
    CUtensorMap tmap;
    const cudaError_t te = conv_tensor_map<CIN>(A, &tmap);
    if (te != cudaSuccess) return te;
    conv3x3_kernel<CIN, HEAD><<<grid, 128, smem, s>>>(A, seg_rows, tmap);
    return cudaGetLastError();
}

// The fused head (A.head_color) is a 32-channel instantiation of its own,
// so its 25 prefetched taps do not raise the other layers' registers.
cudaError_t launch_conv(const ConvArgs& A, int cin, cudaStream_t s) {
    if (A.head_color) return cin == 32 ? launch_conv_t<32, true>(A, s) : cudaErrorInvalidValue;
    return cin == 16 ? launch_conv_t<16, false>(A, s) : launch_conv_t<32, false>(A, s);
}

cudaError_t launch_wgrad(const WgradArgs& A, int cin, cudaStream_t s) {
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int tiles = ((A.w + kTile - 1) / kTile) * A.h * A.n;
    const int grid = tiles < sms * 4 ? tiles : sms * 4;
    if (grid <= 0) return cudaSuccess;
    if (cin == 16)
        wgrad_kernel<16><<<grid, 128, 0, s>>>(A);
    else
        wgrad_kernel<32><<<grid, 128, 0, s>>>(A);
    return cudaGetLastError();
}

cudaError_t launch_head(const HeadArgs& A, cudaStream_t s) {
    const dim3 grid((A.w + 127) / 128, A.h, A.n);
    head_kernel<<<grid, 128, 0, s>>>(A);
    return cudaGetLastError();
}

cudaError_t launch_features(const float4* accum, const ushort4* gbuf, const ushort4* galb, __nv_bfloat16* feat,
                            float4* color, int count, cudaStream_t s) {
    features_kernel<<<(count + 255) / 256, 256, 0, s>>>(accum, gbuf, galb, feat, color, count);
    return cudaGetLastError();
}

cudaError_t launch_pack(const float* params, __nv_bfloat16* const* w, cudaStream_t s) {
    pack_kernel<<<(9 * 32 * 32 + 255) / 256, 256, 0, s>>>(params, w[0], w[1], w[2], w[3], w[4], w[5], w[6]);
    return cudaGetLastError();
}

// bf16 elements of the seven packed weight copies, in rc_kp_pack order
constexpr size_t kPackedElems[7] = {9 * 32 * 16, 9 * 32 * 32, 9 * 32 * 32, 9 * 32 * 32,
                                    9 * 32 * 32, 9 * 32 * 32, 9 * 32 * 32};

size_t packed_bytes() {
    size_t b = 0;
    for (size_t e : kPackedElems) b += e * 2;
    return b;
}

// Inference over one W x H frame: the weight packing (only with `repack`:
// the packed copy is kept between calls with the same parameters),
// features, three hidden convolutions and the head convolution with the
// filter in its epilogue (5 launches, 6 with the packing).
cudaError_t run_inference(const float* params, void* packed, bool repack, const float4* accum, const ushort4* gbuf,
                          const ushort4* galb, void* feat, void* act0, void* act1, float* logits, float4* color,
                          float4* out, int W, int H, unsigned int* err, cudaStream_t s) {
    __nv_bfloat16* w[7];
    __nv_bfloat16* p = static_cast<__nv_bfloat16*>(packed);
    for (int i = 0; i < 7; ++i) {
        w[i] = p;
        p += kPackedElems[i];
    }
    cudaError_t e = repack ? launch_pack(params, w, s) : cudaSuccess;
    if (e == cudaSuccess) e = launch_features(accum, gbuf, galb, static_cast<__nv_bfloat16*>(feat), color, W * H, s);
    const __nv_bfloat16* f = static_cast<const __nv_bfloat16*>(feat);
    __nv_bfloat16* a0 = static_cast<__nv_bfloat16*>(act0);
    __nv_bfloat16* a1 = static_cast<__nv_bfloat16*>(act1);
    if (e == cudaSuccess) e = launch_conv({f, w[0], params + kParamB1, a0, nullptr, 1, H, W, 1, 0, err}, 16, s);
    if (e == cudaSuccess) e = launch_conv({a0, w[1], params + kParamB2, a1, nullptr, 1, H, W, 1, 0, err}, 32, s);
    if (e == cudaSuccess) e = launch_conv({a1, w[2], params + kParamB3, a0, nullptr, 1, H, W, 1, 0, err}, 32, s);
    // the last convolution applies the head in its epilogue (no logits in HBM)
    if (e == cudaSuccess)
        e = launch_conv({a0, w[3], params + kParamBH, logits, nullptr, 1, H, W, 0, 1, err, color, out}, 32, s);
    return e;
}

}  // namespace kp
}  // namespace rc

// ---------------------------------------------------------------------------
// C ABI of the building blocks (device pointers; the training driver and the
// tests call these on their own buffers and stream)
// ---------------------------------------------------------------------------
using namespace rc::kp;

extern "C" {

int rc_kp_conv3x3(const void* in, int cin, const void* wpk, const float* bias, void* out, int out_f32, int relu,
                  const void* mask, int n, int h, int w, unsigned int* err, void* stream) {
    if (!in || !wpk || !out || !err || (cin != 16 && cin != 32) || n <= 0 || h <= 0 || w <= 0)
        return RC_ERR_INVALID_ARG;
    if (!rc::aligned_to(in, 16) || !rc::aligned_to(wpk, 16) || !rc::aligned_to(out, 16) ||
        !rc::aligned_to(mask, 16) || !rc::aligned_to(bias, 4) || !rc::aligned_to(err, 4))
        return RC_ERR_INVALID_ARG;
    ConvArgs A{static_cast<const __nv_bfloat16*>(in), static_cast<const __nv_bfloat16*>(wpk), bias, out,
               static_cast<const __nv_bfloat16*>(mask), n, h, w, relu, out_f32, err, nullptr, nullptr};
    return launch_conv(A, cin, static_cast<cudaStream_t>(stream)) == cudaSuccess ? RC_OK : RC_ERR_CUDA;
}

int rc_kp_wgrad(const void* x, int cin, const void* dy, float* dw, float* db, int n, int h, int w,
                unsigned int* err, void* stream) {
    if (!x || !dy || !dw || !db || !err || (cin != 16 && cin != 32) || n <= 0 || h <= 0 || w <= 0)
        return RC_ERR_INVALID_ARG;
    if (!rc::aligned_to(x, 16) || !rc::aligned_to(dy, 16) || !rc::aligned_to(dw, 4) || !rc::aligned_to(db, 4) ||
        !rc::aligned_to(err, 4))
        return RC_ERR_INVALID_ARG;
    WgradArgs A{static_cast<const __nv_bfloat16*>(x), static_cast<const __nv_bfloat16*>(dy), dw, db, n, h, w, err};
    return launch_wgrad(A, cin, static_cast<cudaStream_t>(stream)) == cudaSuccess ? RC_OK : RC_ERR_CUDA;
}

int rc_kp_head(const float* logits, const void* color, const void* target, void* out, void* dlogits,
               double* loss, float grad_scale, int n, int h, int w, void* stream) {
    if (!logits || !color || !out || n <= 0 || h <= 0 || w <= 0 || (dlogits && !target)) return RC_ERR_INVALID_ARG;
    if (!rc::aligned_to(logits, 16) || !rc::aligned_to(color, 16) || !rc::aligned_to(target, 16) ||
        !rc::aligned_to(out, 16) || !rc::aligned_to(dlogits, 16) || !rc::aligned_to(loss, 8))
        return RC_ERR_INVALID_ARG;
    HeadArgs A{logits,
               static_cast<const float4*>(color),
               static_cast<const float4*>(target),
               static_cast<float4*>(out),
               static_cast<__nv_bfloat16*>(dlogits),
               loss,
               grad_scale,
               n,
               h,
               w};
    return launch_head(A, static_cast<cudaStream_t>(stream)) == cudaSuccess ? RC_OK : RC_ERR_CUDA;
}

int rc_kp_pack(const float* params, void* const* packed7, void* stream) {
    if (!params || !packed7 || !rc::aligned_to(params, 4)) return RC_ERR_INVALID_ARG;
    __nv_bfloat16* w[7];
    for (int i = 0; i < 7; ++i) {
        if (!packed7[i] || !rc::aligned_to(packed7[i], 16)) return RC_ERR_INVALID_ARG;
        w[i] = static_cast<__nv_bfloat16*>(packed7[i]);
    }
    return launch_pack(params, w, static_cast<cudaStream_t>(stream)) == cudaSuccess ? RC_OK : RC_ERR_CUDA;
}

int rc_kp_adam(float* params, float* grads, float* m, float* v, int count, float lr, float beta1, float beta2,
               float eps, int step, void* stream) {
    if (!params || !grads || !m || !v || count <= 0 || step < 1) return RC_ERR_INVALID_ARG;
    if (!rc::aligned_to(params, 4) || !rc::aligned_to(grads, 4) || !rc::aligned_to(m, 4) || !rc::aligned_to(v, 4))
        return RC_ERR_INVALID_ARG;
    const float c1 = 1.0f / (1.0f - powf(beta1, (float)step)), c2 = 1.0f / (1.0f - powf(beta2, (float)step));
    adam_kernel<<<(count + 255) / 256, 256, 0, static_cast<cudaStream_t>(stream)>>>(params, grads, m, v, count, lr,
                                                                                     beta1, beta2, eps, c1, c2);
    return cudaGetLastError() == cudaSuccess ? RC_OK : RC_ERR_CUDA;
}

int rc_kp_crop(const void* feat_all, const void* color_all, const void* target_all, const int* src, const int* tgt,
               const int* oy, const int* ox, int batch, int H, int W, int size, void* feat, void* color,
               void* target, void* stream) {
    if (!feat_all || !color_all || !target_all || !src || !tgt || !oy || !ox || !feat || !color || !target ||
        batch <= 0 || size <= 0 || size > H || size > W)
        return RC_ERR_INVALID_ARG;
    for (const void* q : {feat_all, color_all, target_all, (const void*)feat, (const void*)color, (const void*)target})
        if (!rc::aligned_to(q, 16)) return RC_ERR_INVALID_ARG;
    for (const void* q : {(const void*)src, (const void*)tgt, (const void*)oy, (const void*)ox})
        if (!rc::aligned_to(q, 4)) return RC_ERR_INVALID_ARG;
    const dim3 grid((size + 127) / 128, size, batch);
    crop_kernel<<<grid, 128, 0, static_cast<cudaStream_t>(stream)>>>(
        static_cast<const __nv_bfloat16*>(feat_all), static_cast<const float4*>(color_all),
        static_cast<const float4*>(target_all), src, tgt, oy, ox, H, W, size, static_cast<__nv_bfloat16*>(feat),
        static_cast<float4*>(color), static_cast<float4*>(target));
    return cudaGetLastError() == cudaSuccess ? RC_OK : RC_ERR_CUDA;
}

}  // extern "C"
