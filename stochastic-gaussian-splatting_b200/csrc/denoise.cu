// Learned resolve: a 6-layer 3x3 convolutional denoiser on BF16 tensor cores (tcgen05, FP32 in TMEM).
//
// The reference has no learned resolve; plain progressive averaging (resolve.cu, Static mode) is the
// fallback and the yardstick of its error. This file holds every kernel of the denoiser:
//   conv3x3_kernel        implicit-GEMM 3x3 convolution, zero padding 1, stride 1. Forward layers
//                         (bias + ReLU, or bias + residual for the last layer) and data gradients
//                         (flipped, transposed weights; the ReLU mask of the layer below fused).
//   conv3x3_wgrad_kernel  weight and bias gradients of one layer, summed over all pixels.
//   features_*            the 8-channel FP16 input built from the per-sample renders.
//
// Activations are NHWC BF16 [batch][height][width][channels], channels 16 or 32. One CTA of 128
// threads computes an 8 x 16 pixel tile (M = 128) at a time: it stages the 10 x 18 input halo in
// shared memory as [8-channel chunk][halo pixel][8 channels], so that for every tap (dy, dx) the A
// operand is a K-major no-swizzle view of the halo starting (dy * 10 + dx) * 16 bytes in: the 8
// pixels of a tile row are 16 bytes apart (one core matrix), tile rows 160 bytes apart (SBO), the
// next 8 channels one chunk (2880 bytes) away (LBO). The weights of all 9 taps stay resident in
// shared memory as [tap][chunk][output channel][8] (K-major B). One elected thread issues the
// 9 * CIN / 16 MMAs (M 128, N COUT, K 16) into a 32-column TMEM accumulator and commits them to an
// mbarrier; all four warps then read their 32 TMEM lanes (= 32 pixels) back with tcgen05.ld and
// run the epilogue. Several CTAs share an SM (about 30 KB of shared memory each), so one CTA's
// halo loads overlap another's MMAs and epilogue.
//
// The weight gradient is a GEMM over pixels: dW[tap][co][ci] = sum_p dZ[p][co] * X[p + tap][ci].
// Per tile the kernel builds an im2col block in shared memory, [group][pixel][8], group =
// (tap, 8-channel chunk) plus one group whose first channel is 1 (its row of the product is the
// bias gradient), and multiplies it as an MN-major A (M = 128 rows of (tap, channel)) with the
// tile's output gradient as an MN-major B (N = COUT). Accumulators stay in TMEM across all the
// tiles a CTA handles and are added to the global gradient once at the end.
//
// Every wait on an mbarrier is bounded: when it runs out the kernel sets an error word (read by
// sgs_denoise_status), stops, waits once more with a bound, releases its TMEM and returns.
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>

#include "sgs_b200.h"
#include "sgs_internal.h"
#include "sgs_tcgen05.cuh"

namespace sgs {
namespace dn {

constexpr int kTileW = 8;
constexpr int kTileH = 16;
constexpr int kHaloW = kTileW + 2;
constexpr int kHaloH = kTileH + 2;
constexpr int kHaloPx = kHaloW * kHaloH;  // 180
constexpr int kTilePx = kTileW * kTileH;  // 128 = MMA M
constexpr int kThreads = 128;
constexpr uint32_t kWaitLimit = 1u << 20;

enum InKind { kInBf16 = 0, kInFeatures = 1 };
enum Epilogue { kEpiRelu = SGS_CONV_RELU, kEpiFinal = SGS_CONV_FINAL, kEpiMask = SGS_CONV_MASK };

__device__ unsigned int g_error;

struct ConvArgs {
    const void* in;
    void* out;
    const uint4* weights;
    const float* bias;
    const uint4* mask;
    const uint4* residual;
    int batch, height, width, tiles_x, tiles_y, n_tiles;
};

struct WgradArgs {
    const void* in;
    const uint4* grad_out;
    float* grad_w;
    float* grad_b;
    int batch, height, width, tiles_x, tiles_y, n_tiles;
};

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
    const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<const uint32_t*>(&v);
}

__device__ __forceinline__ float bf16_lo(uint32_t w) { return __uint_as_float(w << 16); }
__device__ __forceinline__ float bf16_hi(uint32_t w) { return __uint_as_float(w & 0xFFFF0000u); }

__device__ __forceinline__ uint32_t half2_to_bf162(uint32_t h) {
    const float2 f = __half22float2(*reinterpret_cast<const __half2*>(&h));
    return pack_bf16(f.x, f.y);
}

__device__ __forceinline__ uint4 half8_to_bf16x8(uint4 v) {
    return make_uint4(half2_to_bf162(v.x), half2_to_bf162(v.y), half2_to_bf162(v.z), half2_to_bf162(v.w));
}

struct TileXY {
    int b, x0, y0;
};

__device__ __forceinline__ TileXY tile_xy(int t, int tiles_x, int tiles_y) {
    const int tx = t % tiles_x;
    const int rest = t / tiles_x;
    return {rest / tiles_y, tx * kTileW, (rest % tiles_y) * kTileH};
}

// Stages the 10 x 18 halo of the tile at (x0, y0) as [chunk][halo pixel][8] BF16, zero outside the
// image. kInFeatures: 8 FP16 channels per pixel, converted to BF16, channels 8..15 zero.
template <int CIN, int IN>
__device__ __forceinline__ void load_halo(const void* in, uint4* halo, const TileXY& t, int height, int width) {
    const uint4* src = static_cast<const uint4*>(in);
    if constexpr (IN == kInFeatures) {
        static_assert(CIN == 16, "features stage as 16 channels");
        for (int p = threadIdx.x; p < kHaloPx; p += kThreads) {
            const int gx = t.x0 - 1 + p % kHaloW, gy = t.y0 - 1 + p / kHaloW;
            uint4 v = make_uint4(0u, 0u, 0u, 0u);
            if (gx >= 0 && gx < width && gy >= 0 && gy < height)
                v = half8_to_bf16x8(__ldg(src + (static_cast<size_t>(t.b) * height + gy) * width + gx));
            halo[p] = v;
            halo[kHaloPx + p] = make_uint4(0u, 0u, 0u, 0u);
        }
    } else {
        constexpr int KC = CIN / 8;
        for (int i = threadIdx.x; i < kHaloPx * KC; i += kThreads) {
            const int p = i / KC, c = i % KC;
            const int gx = t.x0 - 1 + p % kHaloW, gy = t.y0 - 1 + p / kHaloW;
            uint4 v = make_uint4(0u, 0u, 0u, 0u);
            if (gx >= 0 && gx < width && gy >= 0 && gy < height)
                v = __ldg(src + ((static_cast<size_t>(t.b) * height + gy) * width + gx) * KC + c);
            halo[c * kHaloPx + p] = v;
        }
    }
}

template <int N>
__device__ __forceinline__ void load_accumulator(uint32_t taddr, float (&acc)[N]) {
    static_assert(N % 16 == 0, "16-column loads");
#pragma unroll
    for (int h = 0; h < N / 16; ++h) {
        float v[16];
        tc::tmem_ld16(taddr + 16 * h, v);
#pragma unroll
        for (int i = 0; i < 16; ++i) acc[16 * h + i] = v[i];
    }
    tc::tmem_wait_ld();
}

// Epilogue of one output pixel (thread m of the tile owns pixel m = 8 * row + column): bias and
// ReLU, bias and residual (final layer), or the ReLU mask of the layer below (data gradient).
// kPlanar: the BF16 output is stored as 8-channel planes [batch][channel / 8][y][x][8] (the layout of
// the denoiser's internal activations: a warp's store covers 128 contiguous bytes per tile row, and a
// halo box of one plane is a 160-byte run per row) instead of NHWC.
template <int COUT, int EPI, bool kPlanar = false>
__device__ __forceinline__ void store_pixel(const ConvArgs& a, const TileXY& tile, int m, const float (&acc)[COUT],
                                            const float (&bias)[COUT]) {
    const int x = tile.x0 + (m & 7), y = tile.y0 + (m >> 3);
    if (x >= a.width || y >= a.height) return;
    const size_t pixel = (static_cast<size_t>(tile.b) * a.height + y) * a.width + x;
    if constexpr (EPI == kEpiFinal) {
        const uint4 r = __ldg(a.residual + pixel);
        const float2 rg = __half22float2(*reinterpret_cast<const __half2*>(&r.x));
        const float2 bx = __half22float2(*reinterpret_cast<const __half2*>(&r.y));
        float* out = static_cast<float*>(a.out) + pixel * 3;
        out[0] = acc[0] + bias[0] + rg.x;
        out[1] = acc[1] + bias[1] + rg.y;
        out[2] = acc[2] + bias[2] + bx.x;
    } else {
        const size_t plane = static_cast<size_t>(a.height) * a.width;
        const size_t first = kPlanar ? (static_cast<size_t>(tile.b) * (COUT / 8) * plane + static_cast<size_t>(y) * a.width + x)
                                     : pixel * (COUT / 8);
        const size_t step = kPlanar ? plane : 1;
        uint4* out = static_cast<uint4*>(a.out) + first;
#pragma unroll
        for (int q = 0; q < COUT / 8; ++q) {
            float v[8];
#pragma unroll
            for (int i = 0; i < 8; ++i) v[i] = acc[8 * q + i] + bias[8 * q + i];
            if constexpr (EPI == kEpiRelu) {
#pragma unroll
                for (int i = 0; i < 8; ++i) v[i] = fmaxf(v[i], 0.0f);
            } else {
                const uint4 mk = __ldg(a.mask + pixel * (COUT / 8) + q);
                const uint32_t mw[4] = {mk.x, mk.y, mk.z, mk.w};
#pragma unroll
                for (int i = 0; i < 4; ++i) {
                    if (!(bf16_lo(mw[i]) > 0.0f)) v[2 * i] = 0.0f;
                    if (!(bf16_hi(mw[i]) > 0.0f)) v[2 * i + 1] = 0.0f;
                }
            }
            out[q * step] = make_uint4(pack_bf16(v[0], v[1]), pack_bf16(v[2], v[3]), pack_bf16(v[4], v[5]),
                                       pack_bf16(v[6], v[7]));
        }
    }
}

template <int CIN, int COUT, int IN, int EPI, bool kPlanar = false>
__global__ void __launch_bounds__(kThreads, 1) conv3x3_kernel(const ConvArgs a) {
    constexpr int KC = CIN / 8;
    constexpr int kWeightVecs = 9 * KC * COUT;
    constexpr int kHaloVecs = KC * kHaloPx;
    constexpr uint32_t kIdesc = tc::instr_desc_bf16(kTilePx, COUT, false, false);
    static_assert(CIN % 16 == 0 && (COUT == 16 || COUT == 32), "tile shapes");

    extern __shared__ __align__(128) unsigned char smem_raw[];
    uint4* w_s = reinterpret_cast<uint4*>(smem_raw);
    uint4* halo = w_s + kWeightVecs;
    uint64_t* bar_s = reinterpret_cast<uint64_t*>(halo + kHaloVecs);
    uint32_t* slot = reinterpret_cast<uint32_t*>(bar_s + 1);
    const int tid = threadIdx.x, warp = tid >> 5;

    for (int i = tid; i < kWeightVecs; i += kThreads) w_s[i] = __ldg(a.weights + i);
    if (warp == 0) tc::tmem_alloc(tc::smem_u32(slot), 32);
    if (tid == 0) tc::mbar_init(tc::smem_u32(bar_s), 1);
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = *slot;
    const uint32_t bar = tc::smem_u32(bar_s);
    const uint32_t halo_a = tc::smem_u32(halo);
    const uint32_t w_a = tc::smem_u32(w_s);

    float bias[COUT];
#pragma unroll
    for (int n = 0; n < COUT; ++n) bias[n] = (EPI == kEpiMask) ? 0.0f : __ldg(a.bias + n);

    uint32_t phase = 0;
    bool failed = false;
    for (int t = blockIdx.x; t < a.n_tiles; t += gridDim.x) {
        const TileXY tile = tile_xy(t, a.tiles_x, a.tiles_y);
        load_halo<CIN, IN>(a.in, halo, tile, a.height, a.width);
        tc::fence_async_smem();
        tc::fence_before_sync();
        __syncthreads();
        if (tid == 0) {
            tc::fence_after_sync();
#pragma unroll
            for (int tap = 0; tap < 9; ++tap) {
#pragma unroll
                for (int j = 0; j < KC / 2; ++j) {
                    const uint32_t a_addr = halo_a + ((2 * j) * kHaloPx + (tap / 3) * kHaloW + tap % 3) * 16;
                    const uint32_t b_addr = w_a + ((tap * KC + 2 * j) * COUT) * 16;
                    tc::mma_bf16(tmem, tc::smem_desc(a_addr, kHaloPx * 16, kHaloW * 16),
                                 tc::smem_desc(b_addr, COUT * 16, 128), kIdesc, (tap | j) != 0 ? 1u : 0u);
                }
            }
            tc::commit(bar);
        }
        __syncwarp();
        const bool ok = tc::mbar_wait(bar, phase, kWaitLimit);
        phase ^= 1u;
        __syncwarp();
        tc::fence_after_sync();
        float acc[COUT];
        load_accumulator<COUT>(tmem + (static_cast<uint32_t>(warp * 32) << 16), acc);

        if (ok) store_pixel<COUT, EPI, kPlanar>(a, tile, tid, acc, bias);
        tc::fence_before_sync();
        if (__syncthreads_or(!ok)) {
            failed = true;
            break;
        }
    }
    if (failed) {
        if (tid == 0) atomicExch(&g_error, 1u);
        tc::mbar_wait(bar, phase ^ 1u, kWaitLimit);
    }
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) {
        tc::fence_after_sync();
        tc::tmem_dealloc(tmem, 32);
    }
}

// Warp-specialised variant for BF16 inputs, persistent over tiles. Warp 4 (one lane) loads each
// tile's halo with TMA, one 8 x 10 x 18 box per 8-channel chunk of a 4-D tensor map over the NHWC
// input (zero fill outside the image), into a ring of kStages halo slots; warp 5 (one lane) issues
// the tile's MMAs into one of two TMEM accumulators and commits them to the slot's "empty" and the
// accumulator's "full" barrier; warps 0-3 drain the accumulator (tcgen05.ld), release it and run
// the epilogue while the next tile's loads and MMAs are in flight.
constexpr int kStages = 3;
constexpr int kTmaThreads = 192;
constexpr int kTmaCols = 64;  // two 32-column accumulators

template <int CIN, int COUT>
struct TmaConv {
    static constexpr int KC = CIN / 8;
    static constexpr int kWeightVecs = 9 * KC * COUT;
    // TMA destinations start on 128-byte boundaries: chunks 184 pixels (2944 bytes) apart
    static constexpr int kChunkPx = 184;
    static constexpr int kHaloVecs = KC * kChunkPx;
    static constexpr uint32_t kHaloBytes = kHaloVecs * 16;
    static constexpr uint32_t kTxBytes = KC * kHaloPx * 16;  // bytes the KC boxes deliver
    static constexpr int kBars = 2 * kStages + 4;
    static constexpr size_t kSmem =
        static_cast<size_t>(kWeightVecs + kStages * kHaloVecs) * 16 + kBars * 8 + 16 + 128;
    static_assert((kChunkPx * 16) % 128 == 0 && (kWeightVecs * 16) % 128 == 0, "128-byte TMA destinations");
};

// kPlanar: input and BF16 output in the 8-channel-plane layout of store_pixel (the tensor map is then
// over [batch][plane][y][x * 8 + channel] and a chunk's halo is one box of 10 x 18 pixels).
// Held to 4 CTAs per SM (80 registers, no spills): 0.357 against 0.365 ms per 1080p denoiser call at
// the 3 that 90 registers allow.
template <int CIN, int COUT, int EPI, bool kPlanar = false>
__global__ void __launch_bounds__(kTmaThreads, 4) conv3x3_tma_kernel(const __grid_constant__ CUtensorMap in_map,
                                                                  const ConvArgs a) {
    using S = TmaConv<CIN, COUT>;
    constexpr uint32_t kIdesc = tc::instr_desc_bf16(kTilePx, COUT, false, false);
    static_assert(COUT <= kTmaCols / 2, "two accumulators");
    extern __shared__ __align__(128) unsigned char smem_raw[];
    uint4* w_s = reinterpret_cast<uint4*>(smem_raw + ((128u - (tc::smem_u32(smem_raw) & 127u)) & 127u));
    uint4* halo = w_s + S::kWeightVecs;
    uint64_t* bars = reinterpret_cast<uint64_t*>(halo + kStages * S::kHaloVecs);
    uint32_t* slot = reinterpret_cast<uint32_t*>(bars + S::kBars);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    // barriers: full[s], empty[s] (halo slots), acc_full[k], acc_empty[k] (accumulators)
    const uint32_t bar0 = tc::smem_u32(bars);
#define SGS_FULL(st) (bar0 + 8u * (st))
#define SGS_EMPTY(st) (bar0 + 8u * (kStages + (st)))
#define SGS_ACC_FULL(k) (bar0 + 8u * (2 * kStages + (k)))
#define SGS_ACC_EMPTY(k) (bar0 + 8u * (2 * kStages + 2 + (k)))

    for (int i = tid; i < S::kWeightVecs; i += kTmaThreads) w_s[i] = __ldg(a.weights + i);
    tc::fence_async_smem();
    if (warp == 0) tc::tmem_alloc(tc::smem_u32(slot), kTmaCols);
    if (tid == 0) {
        for (int st = 0; st < kStages; ++st) {
            tc::mbar_init(SGS_FULL(st), 1);
            tc::mbar_init(SGS_EMPTY(st), 1);
        }
        for (int k = 0; k < 2; ++k) {
            tc::mbar_init(SGS_ACC_FULL(k), 1);
            tc::mbar_init(SGS_ACC_EMPTY(k), 4);
        }
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = *slot;
    const uint32_t halo_a = tc::smem_u32(halo);
    const uint32_t w_a = tc::smem_u32(w_s);
    bool failed = false;
    int issued = 0;  // producer: tiles whose loads were issued; MMA: tiles whose MMAs were committed

    if (warp == 4) {
        if (lane == 0) {
            for (int t = blockIdx.x; t < a.n_tiles; t += gridDim.x, ++issued) {
                const int st = issued % kStages;
                const uint32_t ph = (issued / kStages) & 1u;
                if (issued >= kStages && !tc::mbar_wait(SGS_EMPTY(st), ph ^ 1u, kWaitLimit)) {
                    failed = true;
                    break;
                }
                const TileXY tile = tile_xy(t, a.tiles_x, a.tiles_y);
                tc::mbar_arrive_expect_tx(SGS_FULL(st), S::kTxBytes);
#pragma unroll
                for (int c = 0; c < S::KC; ++c) {
                    const uint32_t dst = halo_a + (st * S::kHaloVecs + c * S::kChunkPx) * 16;
                    if constexpr (kPlanar)  // x in elements: 8 per pixel, so always a 16-byte multiple
                        tc::tma_load_4d(dst, &in_map, SGS_FULL(st), (tile.x0 - 1) * 8, tile.y0 - 1, c, tile.b);
                    else
                        tc::tma_load_4d(dst, &in_map, SGS_FULL(st), c * 8, tile.x0 - 1, tile.y0 - 1, tile.b);
                }
            }
        }
    } else if (warp == 5) {
        if (lane == 0) {
            for (int t = blockIdx.x; t < a.n_tiles; t += gridDim.x, ++issued) {
                const int st = issued % kStages, k = issued & 1;
                const uint32_t ph = (issued / kStages) & 1u, aph = (issued >> 1) & 1u;
                if (!tc::mbar_wait(SGS_FULL(st), ph, kWaitLimit) ||
                    (issued >= 2 && !tc::mbar_wait(SGS_ACC_EMPTY(k), aph ^ 1u, kWaitLimit))) {
                    failed = true;
                    break;
                }
                tc::fence_after_sync();
                const uint32_t h = halo_a + st * S::kHaloBytes;
#pragma unroll
                for (int tap = 0; tap < 9; ++tap) {
#pragma unroll
                    for (int j = 0; j < S::KC / 2; ++j) {
                        const uint32_t a_addr = h + ((2 * j) * S::kChunkPx + (tap / 3) * kHaloW + tap % 3) * 16;
                        const uint32_t b_addr = w_a + ((tap * S::KC + 2 * j) * COUT) * 16;
                        tc::mma_bf16(tmem + k * (kTmaCols / 2), tc::smem_desc(a_addr, S::kChunkPx * 16, kHaloW * 16),
                                     tc::smem_desc(b_addr, COUT * 16, 128), kIdesc, (tap | j) != 0 ? 1u : 0u);
                    }
                }
                tc::commit(SGS_EMPTY(st));
                tc::commit(SGS_ACC_FULL(k));
            }
        }
    } else {
        float bias[COUT];
#pragma unroll
        for (int n = 0; n < COUT; ++n) bias[n] = (EPI == kEpiMask) ? 0.0f : __ldg(a.bias + n);
        int i = 0;
        for (int t = blockIdx.x; t < a.n_tiles; t += gridDim.x, ++i) {
            const int k = i & 1;
            const bool ok = __all_sync(0xFFFFFFFFu, tc::mbar_wait(SGS_ACC_FULL(k), (i >> 1) & 1u, kWaitLimit));
            if (!ok) {
                failed = true;
                break;
            }
            tc::fence_after_sync();
            float acc[COUT];
            load_accumulator<COUT>(tmem + (static_cast<uint32_t>(warp * 32) << 16) + k * (kTmaCols / 2), acc);
            tc::fence_before_sync();
            __syncwarp();
            if (lane == 0) tc::mbar_arrive(SGS_ACC_EMPTY(k));
            store_pixel<COUT, EPI, kPlanar>(a, tile_xy(t, a.tiles_x, a.tiles_y), tid, acc, bias);
        }
    }

    if (__syncthreads_or(failed)) {
        if (tid == 0) atomicExch(&g_error, 1u);
        // let this CTA's own copies and MMAs in flight finish (bounded) before its memory goes away
        if (warp == 4 && lane == 0)
            for (int q = issued - 1; q >= 0 && q >= issued - kStages; --q)
                tc::mbar_wait(SGS_FULL(q % kStages), (q / kStages) & 1u, kWaitLimit);
        if (warp == 5 && lane == 0 && issued > 0)
            tc::mbar_wait(SGS_ACC_FULL((issued - 1) & 1), ((issued - 1) >> 1) & 1u, kWaitLimit);
    }
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) {
        tc::fence_after_sync();
        tc::tmem_dealloc(tmem, kTmaCols);
    }
#undef SGS_FULL
#undef SGS_EMPTY
#undef SGS_ACC_FULL
#undef SGS_ACC_EMPTY
}

// Weight-gradient geometry: im2col groups of 8 rows, (tap, chunk) for tap-major order, then the
// bias group, then zero groups up to the allocation. M-tile m reads groups start(m) .. start(m)+15
// and owns (adds to the gradient) groups [own(m), own(m+1)).
template <int CIN, int COUT>
struct Wgrad {
    static constexpr int KC = CIN / 8;
    static constexpr int KCO = COUT / 8;
    static constexpr int kConvGroups = 9 * KC;
    static constexpr int kBiasGroup = kConvGroups;
    static constexpr int kMTiles = CIN == 32 ? 3 : 2;
    static constexpr int kGroups = CIN == 32 ? 40 : 20;
    static constexpr int kCols = kMTiles * COUT <= 32 ? 32 : kMTiles * COUT <= 64 ? 64 : 128;
    static constexpr int kHaloVecs = KC * kHaloPx;
    static constexpr int kGradVecs = KCO * kTilePx;
    static constexpr int kColVecs = kGroups * kTilePx;
    static constexpr size_t kSmem = static_cast<size_t>(kHaloVecs + kGradVecs + kColVecs) * 16 + 16;
    __host__ __device__ static constexpr int start(int m) { return CIN == 32 ? (m == 0 ? 0 : m == 1 ? 16 : 24) : (m == 0 ? 0 : 4); }
    __host__ __device__ static constexpr int own(int m) { return m == 0 ? 0 : m == kMTiles ? kGroups : 16 * m; }
    static_assert(start(kMTiles - 1) + 16 == kGroups, "last M tile ends at the allocation");
    static_assert(kBiasGroup < kGroups, "bias group allocated");
};

template <int CIN, int COUT, int IN>
__global__ void __launch_bounds__(kThreads) conv3x3_wgrad_kernel(const WgradArgs a) {
    using G = Wgrad<CIN, COUT>;
    constexpr uint32_t kIdesc = tc::instr_desc_bf16(kTilePx, COUT, true, true);
    constexpr uint32_t kGroupBytes = kTilePx * 16;  // 2048

    extern __shared__ __align__(128) unsigned char smem_raw[];
    uint4* halo = reinterpret_cast<uint4*>(smem_raw);
    uint4* grad_s = halo + G::kHaloVecs;
    uint4* col = grad_s + G::kGradVecs;
    uint64_t* bar_s = reinterpret_cast<uint64_t*>(col + G::kColVecs);
    uint32_t* slot = reinterpret_cast<uint32_t*>(bar_s + 1);
    const int tid = threadIdx.x, warp = tid >> 5;

    // constant groups: the bias group (first channel 1.0 for every pixel) and the zero padding
    for (int i = G::kBiasGroup * kTilePx + tid; i < G::kColVecs; i += kThreads)
        col[i] = make_uint4(i < (G::kBiasGroup + 1) * kTilePx ? 0x3F80u : 0u, 0u, 0u, 0u);
    if (warp == 0) tc::tmem_alloc(tc::smem_u32(slot), G::kCols);
    if (tid == 0) tc::mbar_init(tc::smem_u32(bar_s), 1);
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = *slot;
    const uint32_t bar = tc::smem_u32(bar_s);
    const uint32_t col_a = tc::smem_u32(col);
    const uint32_t grad_a = tc::smem_u32(grad_s);

    uint32_t phase = 0;
    bool failed = false;
    bool first = true;
    for (int t = blockIdx.x; t < a.n_tiles; t += gridDim.x) {
        const TileXY tile = tile_xy(t, a.tiles_x, a.tiles_y);
        load_halo<CIN, IN>(a.in, halo, tile, a.height, a.width);
        for (int i = tid; i < G::kGradVecs; i += kThreads) {
            const int k = i / G::KCO, c = i % G::KCO;
            const int x = tile.x0 + (k & 7), y = tile.y0 + (k >> 3);
            uint4 v = make_uint4(0u, 0u, 0u, 0u);
            if (x < a.width && y < a.height)
                v = __ldg(a.grad_out + ((static_cast<size_t>(tile.b) * a.height + y) * a.width + x) * G::KCO + c);
            grad_s[c * kTilePx + k] = v;
        }
        __syncthreads();
        for (int i = tid; i < G::kConvGroups * kTilePx; i += kThreads) {
            const int g = i >> 7, k = i & 127;
            const int tap = g / G::KC, c = g % G::KC;
            col[i] = halo[c * kHaloPx + ((k >> 3) + tap / 3) * kHaloW + (k & 7) + tap % 3];
        }
        tc::fence_async_smem();
        tc::fence_before_sync();
        __syncthreads();
        if (tid == 0) {
            tc::fence_after_sync();
#pragma unroll
            for (int m = 0; m < G::kMTiles; ++m) {
#pragma unroll
                for (int kk = 0; kk < kTilePx / 16; ++kk) {
                    const uint64_t ad = tc::smem_desc(col_a + G::start(m) * kGroupBytes + kk * 256, 128, kGroupBytes);
                    const uint64_t bd = tc::smem_desc(grad_a + kk * 256, 128, kGroupBytes);
                    tc::mma_bf16(tmem + m * COUT, ad, bd, kIdesc, (first && kk == 0) ? 0u : 1u);
                }
            }
            tc::commit(bar);
        }
        first = false;
        __syncwarp();
        const bool ok = tc::mbar_wait(bar, phase, kWaitLimit);
        phase ^= 1u;
        if (__syncthreads_or(!ok)) {
            failed = true;
            break;
        }
    }
    if (failed) {
        if (tid == 0) atomicExch(&g_error, 1u);
        tc::mbar_wait(bar, phase ^ 1u, kWaitLimit);
    } else if (!first) {
        __syncwarp();
        tc::fence_after_sync();
#pragma unroll
        for (int m = 0; m < G::kMTiles; ++m) {
            float acc[COUT];
            load_accumulator<COUT>(tmem + (static_cast<uint32_t>(warp * 32) << 16) + m * COUT, acc);
            const int g = G::start(m) + (tid >> 3), ch = tid & 7;
            if (g >= G::own(m) && g < G::own(m + 1)) {
                if (g < G::kConvGroups) {
                    const int tap = g / G::KC, ci = (g % G::KC) * 8 + ch;
#pragma unroll
                    for (int n = 0; n < COUT; ++n) atomicAdd(a.grad_w + (tap * COUT + n) * CIN + ci, acc[n]);
                } else if (g == G::kBiasGroup && ch == 0) {
#pragma unroll
                    for (int n = 0; n < COUT; ++n) atomicAdd(a.grad_b + n, acc[n]);
                }
            }
        }
    }
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) {
        tc::fence_after_sync();
        tc::tmem_dealloc(tmem, G::kCols);
    }
}

// ---- input features -----------------------------------------------------------------------

// accum per pixel: float4 (sum r, sum g, sum b, sum alpha), float4 (sum depth, sum lum^2,
// winner changes, last winner index bits).
__global__ void features_accumulate_kernel(const float* __restrict__ image, const float* __restrict__ alpha,
                                           const float* __restrict__ depth,
                                           const unsigned long long* __restrict__ framebuffer,
                                           float4* __restrict__ accum, uint32_t n_px, int first) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_px) return;
    const float r = image[3 * i], g = image[3 * i + 1], b = image[3 * i + 2];
    const float al = alpha[i], d = depth[i];
    const float lum = 0.2126f * r + 0.7152f * g + 0.0722f * b;
    const uint32_t idx = framebuffer != nullptr ? static_cast<uint32_t>(framebuffer[i]) : 0xFFFFFFFFu;
    float4 s0 = make_float4(r, g, b, al);
    float4 s1 = make_float4(d, lum * lum, 0.0f, __uint_as_float(idx));
    if (!first) {
        const float4 p0 = accum[2 * i], p1 = accum[2 * i + 1];
        s0 = make_float4(p0.x + r, p0.y + g, p0.z + b, p0.w + al);
        s1 = make_float4(p1.x + d, p1.y + lum * lum, p1.z + (__float_as_uint(p1.w) != idx ? 1.0f : 0.0f), s1.w);
    }
    accum[2 * i] = s0;
    accum[2 * i + 1] = s1;
}

// features per pixel, FP16: mean r, g, b, mean alpha, mean depth * depth_scale, standard error of
// the mean luminance, fraction of consecutive samples whose winner changed, 0.
__global__ void features_finalize_kernel(const float4* __restrict__ accum, uint4* __restrict__ features,
                                         uint32_t n_px, uint32_t n_samples, float depth_scale) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_px) return;
    const float inv = 1.0f / static_cast<float>(n_samples);
    const float4 s0 = accum[2 * i], s1 = accum[2 * i + 1];
    const float r = s0.x * inv, g = s0.y * inv, b = s0.z * inv;
    const float lum = 0.2126f * r + 0.7152f * g + 0.0722f * b;
    const float var = fmaxf(s1.y * inv - lum * lum, 0.0f);
    const float se = sqrtf(var * inv);
    const float change = s1.z / static_cast<float>(n_samples > 1 ? n_samples - 1 : 1);
    const __half2 h0 = __floats2half2_rn(r, g), h1 = __floats2half2_rn(b, s0.w * inv);
    const __half2 h2 = __floats2half2_rn(s1.x * inv * depth_scale, se), h3 = __floats2half2_rn(change, 0.0f);
    features[i] = make_uint4(*reinterpret_cast<const uint32_t*>(&h0), *reinterpret_cast<const uint32_t*>(&h1),
                             *reinterpret_cast<const uint32_t*>(&h2), *reinterpret_cast<const uint32_t*>(&h3));
}

// ---- host side --------------------------------------------------------------------------------

int sm_count() {
    static int count = 0;
    static std::once_flag once;
    std::call_once(once, [] {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&count, cudaDevAttrMultiProcessorCount, dev);
        if (count <= 0) count = 148;
    });
    return count;
}

// CTAs of `kernel` that fit on one SM, from its shared memory (with the maximum carveout), registers
// and threads; at most `cap`. (The occupancy query answers for the default carveout, which keeps
// these small-footprint kernels at one CTA per SM.)
template <typename Kernel>
int resident_ctas(Kernel kernel, size_t smem, int cap, int threads = kThreads) {
    int dev = 0, smem_sm = 0, regs_sm = 0;
    cudaFuncAttributes attr{};
    if (cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)) !=
            cudaSuccess ||
        cudaFuncSetAttribute(kernel, cudaFuncAttributePreferredSharedMemoryCarveout, cudaSharedmemCarveoutMaxShared) !=
            cudaSuccess ||
        cudaFuncGetAttributes(&attr, kernel) != cudaSuccess || cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&regs_sm, cudaDevAttrMaxRegistersPerMultiprocessor, dev) != cudaSuccess)
        return 0;
    const size_t per_cta = smem + attr.sharedSizeBytes + 1024;  // 1 KB reserved per CTA
    int blocks = static_cast<int>(static_cast<size_t>(smem_sm) / per_cta);
    const int regs = attr.numRegs > 0 ? attr.numRegs * threads : 1;
    if (regs_sm / regs < blocks) blocks = regs_sm / regs;
    if (2048 / threads < blocks) blocks = 2048 / threads;
    return blocks < cap ? blocks : cap;
}

template <int CIN, int COUT, int IN, int EPI, bool kPlanar = false>
cudaError_t launch_conv(const ConvArgs& a, cudaStream_t stream) {
    constexpr size_t smem = static_cast<size_t>(9 * (CIN / 8) * COUT + (CIN / 8) * kHaloPx) * 16 + 16;
    auto kernel = conv3x3_kernel<CIN, COUT, IN, EPI, kPlanar>;
    static const int per_sm = resident_ctas(kernel, smem, 8);
    if (per_sm <= 0) return cudaErrorInvalidConfiguration;
    const int grid = a.n_tiles < sm_count() * per_sm ? a.n_tiles : sm_count() * per_sm;
    kernel<<<grid, kThreads, smem, stream>>>(a);
    return cudaGetLastError();
}

// cuTensorMapEncodeTiled from the driver, looked up through the runtime (no libcuda link).
PFN_cuTensorMapEncodeTiled_v12000 encode_tiled() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    });
    return fn;
}

// 4-D map over a BF16 NHWC tensor [batch][height][width][channels] with a box of 8 channels x the
// 10 x 18 halo x 1 image.
bool nhwc_halo_map(CUtensorMap* map, const void* base, int batch, int height, int width, int channels) {
    const auto fn = encode_tiled();
    if (fn == nullptr) return false;
    const cuuint64_t dims[4] = {static_cast<cuuint64_t>(channels), static_cast<cuuint64_t>(width),
                                static_cast<cuuint64_t>(height), static_cast<cuuint64_t>(batch)};
    const cuuint64_t strides[3] = {static_cast<cuuint64_t>(channels) * 2,
                                   static_cast<cuuint64_t>(width) * channels * 2,
                                   static_cast<cuuint64_t>(height) * width * channels * 2};
    const cuuint32_t box[4] = {8, kHaloW, kHaloH, 1};
    const cuuint32_t elem[4] = {1, 1, 1, 1};
    return fn(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<void*>(base), dims, strides, box, elem,
              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// The same halo boxes over activations in 8-channel planes, [batch][channels / 8][y][x][8]: dimension 0
// runs over x * 8 + channel, so a plane's box is 10 pixels (160 bytes) wide and 18 rows high.
bool planar_halo_map(CUtensorMap* map, const void* base, int batch, int height, int width, int channels) {
    const auto fn = encode_tiled();
    if (fn == nullptr) return false;
    const cuuint64_t dims[4] = {static_cast<cuuint64_t>(width) * 8, static_cast<cuuint64_t>(height),
                                static_cast<cuuint64_t>(channels / 8), static_cast<cuuint64_t>(batch)};
    const cuuint64_t strides[3] = {static_cast<cuuint64_t>(width) * 16,
                                   static_cast<cuuint64_t>(height) * width * 16,
                                   static_cast<cuuint64_t>(channels / 8) * height * width * 16};
    const cuuint32_t box[4] = {kHaloW * 8, kHaloH, 1, 1};
    const cuuint32_t elem[4] = {1, 1, 1, 1};
    return fn(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<void*>(base), dims, strides, box, elem,
              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

template <int CIN, int COUT, int EPI, bool kPlanar = false>
cudaError_t launch_conv_tma(const ConvArgs& a, cudaStream_t stream) {
    using S = TmaConv<CIN, COUT>;
    auto kernel = conv3x3_tma_kernel<CIN, COUT, EPI, kPlanar>;
    static const int per_sm = resident_ctas(kernel, S::kSmem, 512 / kTmaCols, kTmaThreads);
    if (per_sm <= 0) return cudaErrorInvalidConfiguration;
    CUtensorMap map;
    const bool mapped = kPlanar ? planar_halo_map(&map, a.in, a.batch, a.height, a.width, CIN)
                                : nhwc_halo_map(&map, a.in, a.batch, a.height, a.width, CIN);
    if (!mapped) return cudaErrorInvalidValue;
    const int grid = a.n_tiles < sm_count() * per_sm ? a.n_tiles : sm_count() * per_sm;
    kernel<<<grid, kTmaThreads, S::kSmem, stream>>>(map, a);
    return cudaGetLastError();
}

template <int CIN, int COUT, int IN>
cudaError_t launch_wgrad(const WgradArgs& a, cudaStream_t stream) {
    using G = Wgrad<CIN, COUT>;
    auto kernel = conv3x3_wgrad_kernel<CIN, COUT, IN>;
    // TMEM columns bound the CTAs per SM: 512 / kCols
    static const int per_sm = resident_ctas(kernel, G::kSmem, 512 / G::kCols);
    if (per_sm <= 0) return cudaErrorInvalidConfiguration;
    const int grid = a.n_tiles < sm_count() * per_sm ? a.n_tiles : sm_count() * per_sm;
    kernel<<<grid, kThreads, G::kSmem, stream>>>(a);
    return cudaGetLastError();
}

bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

size_t weights_bytes(int in_channels, int out_channels) {
    const int cin = in_channels == 8 ? 16 : in_channels;
    return static_cast<size_t>(9) * cin * out_channels * 2;
}

int check_shape(int batch, int height, int width) {
    if (batch <= 0 || height <= 0 || width <= 0)
        return record_error(SGS_ERROR_INVALID_ARGUMENT, "conv3x3: batch, height and width must be positive");
    const long long tiles =
        static_cast<long long>(batch) * ((height + kTileH - 1) / kTileH) * ((width + kTileW - 1) / kTileW);
    if (tiles > 0x7FFFFFFFll)
        return record_error(SGS_ERROR_INVALID_ARGUMENT, "conv3x3: too many pixels for one call");
    return SGS_OK;
}

// Layer shapes of the denoiser: (input channels as the ABI counts them, output channels, epilogue).
constexpr int kLayers = SGS_DENOISE_LAYERS;
constexpr int kLayerIn[kLayers] = {8, 32, 32, 32, 32, 32};
constexpr int kLayerOut[kLayers] = {32, 32, 32, 32, 32, 16};

}  // namespace dn
}  // namespace sgs

using namespace sgs;
using namespace sgs::dn;

extern "C" {

size_t sgs_conv3x3_weights_size(int32_t in_channels, int32_t out_channels) {
    return weights_bytes(in_channels, out_channels);
}

int sgs_conv3x3(const sgs_conv3x3_args* p, void* stream_ptr) {
    if (p == nullptr) return record_error(SGS_ERROR_INVALID_ARGUMENT, "conv3x3: null descriptor");
    if (int st = check_shape(p->batch, p->height, p->width)) return st;
    if (p->input == nullptr || p->output == nullptr || p->weights == nullptr)
        return record_error(SGS_ERROR_INVALID_ARGUMENT, "conv3x3: input, output and weights are required");
    if (!aligned16(p->input) || !aligned16(p->weights) || !aligned16(p->mask) || !aligned16(p->residual) ||
        (p->epilogue != SGS_CONV_FINAL && !aligned16(p->output)))
        return record_error(SGS_ERROR_INVALID_ARGUMENT, "conv3x3: arrays must be 16-byte aligned");
    if (p->epilogue != SGS_CONV_MASK && p->bias == nullptr)
        return record_error(SGS_ERROR_INVALID_ARGUMENT, "conv3x3: bias is required");
    if (p->epilogue == SGS_CONV_MASK && p->mask == nullptr)
        return record_error(SGS_ERROR_INVALID_ARGUMENT, "conv3x3: the mask epilogue needs a mask");
    if (p->epilogue == SGS_CONV_FINAL && p->residual == nullptr)
        return record_error(SGS_ERROR_INVALID_ARGUMENT, "conv3x3: the final epilogue needs the features");
    ConvArgs a{p->input, p->output, static_cast<const uint4*>(p->weights), p->bias,
               static_cast<const uint4*>(p->mask), static_cast<const uint4*>(p->residual),
               p->batch, p->height, p->width, (p->width + kTileW - 1) / kTileW, (p->height + kTileH - 1) / kTileH, 0};
    a.n_tiles = a.batch * a.tiles_x * a.tiles_y;
    cudaStream_t stream = static_cast<cudaStream_t>(stream_ptr);
    const int ci = p->in_channels, co = p->out_channels, epi = p->epilogue;
    cudaError_t err;
    if (ci == 8 && co == 32 && epi == SGS_CONV_RELU)
        err = launch_conv<16, 32, kInFeatures, kEpiRelu>(a, stream);
    else if (ci == 32 && co == 32 && epi == SGS_CONV_RELU)
        err = launch_conv_tma<32, 32, kEpiRelu>(a, stream);
    else if (ci == 32 && co == 16 && epi == SGS_CONV_FINAL)
        err = launch_conv_tma<32, 16, kEpiFinal>(a, stream);
    else if (ci == 32 && co == 32 && epi == SGS_CONV_MASK)
        err = launch_conv_tma<32, 32, kEpiMask>(a, stream);
    else if (ci == 16 && co == 32 && epi == SGS_CONV_MASK)
        err = launch_conv_tma<16, 32, kEpiMask>(a, stream);
    else
        return record_error(SGS_ERROR_INVALID_ARGUMENT, "conv3x3: unsupported shape %d -> %d, epilogue %d", ci, co,
                            epi);
    if (err != cudaSuccess) return record_error(SGS_ERROR_CUDA, "conv3x3: %s", cudaGetErrorString(err));
    return SGS_OK;
}

int sgs_conv3x3_wgrad(const void* input, int32_t in_channels, const void* grad_output, int32_t out_channels,
                      int32_t batch, int32_t height, int32_t width, float* grad_weights, float* grad_bias,
                      void* stream_ptr) {
    if (int st = check_shape(batch, height, width)) return st;
    if (input == nullptr || grad_output == nullptr || grad_weights == nullptr || grad_bias == nullptr)
        return record_error(SGS_ERROR_INVALID_ARGUMENT, "conv3x3_wgrad: all arrays are required");
    if (!aligned16(input) || !aligned16(grad_output))
        return record_error(SGS_ERROR_INVALID_ARGUMENT, "conv3x3_wgrad: arrays must be 16-byte aligned");
    WgradArgs a{input, static_cast<const uint4*>(grad_output), grad_weights, grad_bias, batch, height, width,
                (width + kTileW - 1) / kTileW, (height + kTileH - 1) / kTileH, 0};
    a.n_tiles = a.batch * a.tiles_x * a.tiles_y;
    cudaStream_t stream = static_cast<cudaStream_t>(stream_ptr);
    cudaError_t err;
    if (in_channels == 8 && out_channels == 32)
        err = launch_wgrad<16, 32, kInFeatures>(a, stream);
    else if (in_channels == 32 && out_channels == 32)
        err = launch_wgrad<32, 32, kInBf16>(a, stream);
    else if (in_channels == 32 && out_channels == 16)
        err = launch_wgrad<32, 16, kInBf16>(a, stream);
    else
        return record_error(SGS_ERROR_INVALID_ARGUMENT, "conv3x3_wgrad: unsupported shape %d -> %d", in_channels,
                            out_channels);
    if (err != cudaSuccess) return record_error(SGS_ERROR_CUDA, "conv3x3_wgrad: %s", cudaGetErrorString(err));
    return SGS_OK;
}

int sgs_denoise_features_accumulate(const float* image, const float* alpha, const float* depth,
                                    const uint64_t* framebuffer, float* accum, uint32_t n_pixels, int32_t first,
                                    void* stream_ptr) {
    if (image == nullptr || alpha == nullptr || depth == nullptr || accum == nullptr)
        return record_error(SGS_ERROR_INVALID_ARGUMENT, "denoise features: image, alpha, depth and accum are required");
    if (!aligned16(accum)) return record_error(SGS_ERROR_INVALID_ARGUMENT, "denoise features: accum not aligned");
    if (n_pixels == 0) return SGS_OK;
    features_accumulate_kernel<<<(n_pixels + 255) / 256, 256, 0, static_cast<cudaStream_t>(stream_ptr)>>>(
        image, alpha, depth, reinterpret_cast<const unsigned long long*>(framebuffer), reinterpret_cast<float4*>(accum),
        n_pixels, first);
    const cudaError_t err = cudaGetLastError();
    if (err != cudaSuccess) return record_error(SGS_ERROR_CUDA, "denoise features: %s", cudaGetErrorString(err));
    return SGS_OK;
}

int sgs_denoise_features_finalize(const float* accum, uint32_t n_pixels, uint32_t n_samples, float depth_scale,
                                  void* features, void* stream_ptr) {
    if (accum == nullptr || features == nullptr || n_samples == 0)
        return record_error(SGS_ERROR_INVALID_ARGUMENT, "denoise features: accum, features and n_samples > 0 required");
    if (!aligned16(accum) || !aligned16(features))
        return record_error(SGS_ERROR_INVALID_ARGUMENT, "denoise features: arrays must be 16-byte aligned");
    if (n_pixels == 0) return SGS_OK;
    features_finalize_kernel<<<(n_pixels + 255) / 256, 256, 0, static_cast<cudaStream_t>(stream_ptr)>>>(
        reinterpret_cast<const float4*>(accum), static_cast<uint4*>(features), n_pixels, n_samples, depth_scale);
    const cudaError_t err = cudaGetLastError();
    if (err != cudaSuccess) return record_error(SGS_ERROR_CUDA, "denoise features: %s", cudaGetErrorString(err));
    return SGS_OK;
}

size_t sgs_denoise_weights_size(void) {
    size_t total = 0;
    for (int l = 0; l < kLayers; ++l) total += weights_bytes(kLayerIn[l], kLayerOut[l]);
    return total;
}

size_t sgs_denoise_scratch_size(int32_t batch, int32_t height, int32_t width) {
    if (batch <= 0 || height <= 0 || width <= 0) return 0;
    return static_cast<size_t>(2) * batch * height * width * SGS_DENOISE_WIDTH * 2;
}

int sgs_denoise(const void* features, int32_t batch, int32_t height, int32_t width, const void* weights,
                const float* biases, void* scratch, size_t scratch_bytes, float* output, void* stream_ptr) {
    if (int st = check_shape(batch, height, width)) return st;
    if (features == nullptr || weights == nullptr || biases == nullptr || scratch == nullptr || output == nullptr)
        return record_error(SGS_ERROR_INVALID_ARGUMENT, "denoise: all arrays are required");
    if (scratch_bytes < sgs_denoise_scratch_size(batch, height, width) || !aligned16(scratch))
        return record_error(SGS_ERROR_WORKSPACE, "denoise: scratch needs %zu bytes, 16-byte aligned",
                            sgs_denoise_scratch_size(batch, height, width));
    if (!aligned16(features) || !aligned16(weights))
        return record_error(SGS_ERROR_INVALID_ARGUMENT, "denoise: features and weights must be 16-byte aligned");
    // the hidden activations live only in the scratch, so they use the 8-channel-plane layout (wider
    // halo boxes, coalesced stores); the same arithmetic as the NHWC layers of sgs_conv3x3
    unsigned char* act[2] = {static_cast<unsigned char*>(scratch),
                             static_cast<unsigned char*>(scratch) + sgs_denoise_scratch_size(batch, height, width) / 2};
    const unsigned char* w = static_cast<const unsigned char*>(weights);
    const float* b = biases;
    cudaStream_t stream = static_cast<cudaStream_t>(stream_ptr);
    const int tiles_x = (width + kTileW - 1) / kTileW, tiles_y = (height + kTileH - 1) / kTileH;
    for (int l = 0; l < kLayers; ++l) {
        const bool last = l == kLayers - 1;
        ConvArgs a{l == 0 ? features : act[(l + 1) & 1], last ? static_cast<void*>(output) : act[l & 1],
                   reinterpret_cast<const uint4*>(w), b, nullptr,
                   last ? static_cast<const uint4*>(features) : nullptr, batch, height, width, tiles_x, tiles_y, 0};
        a.n_tiles = batch * tiles_x * tiles_y;
        cudaError_t err;
        if (l == 0)
            err = launch_conv<16, 32, kInFeatures, kEpiRelu, true>(a, stream);
        else if (!last)
            err = launch_conv_tma<32, 32, kEpiRelu, true>(a, stream);
        else
            err = launch_conv_tma<32, 16, kEpiFinal, true>(a, stream);
        if (err != cudaSuccess) return record_error(SGS_ERROR_CUDA, "denoise layer %d: %s", l + 1, cudaGetErrorString(err));
        w += weights_bytes(kLayerIn[l], kLayerOut[l]);
        b += kLayerOut[l];
    }
    return SGS_OK;
}

int sgs_denoise_status(void* stream_ptr) {
    const cudaError_t sync = cudaStreamSynchronize(static_cast<cudaStream_t>(stream_ptr));
    if (sync != cudaSuccess) return record_error(SGS_ERROR_CUDA, "denoise: %s", cudaGetErrorString(sync));
    unsigned int flag = 0, zero = 0;
    if (cudaMemcpyFromSymbol(&flag, g_error, sizeof(flag)) != cudaSuccess ||
        cudaMemcpyToSymbol(g_error, &zero, sizeof(zero)) != cudaSuccess)
        return record_error(SGS_ERROR_CUDA, "denoise: cannot read the error word");
    if (flag != 0) return record_error(SGS_ERROR_CUDA, "denoise: a tensor-core wait ran out of its bound");
    return SGS_OK;
}

}  // extern "C"
