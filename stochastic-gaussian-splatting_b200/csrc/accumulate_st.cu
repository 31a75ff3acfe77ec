// Stochastic-transparency accumulation: the closest accepted fragment per (sub)pixel.
//
// Semantics follow accumulate_scatter.cu:19-77 and scatter_utils.cuh:14-95 of the reference:
// every pixel of a Gaussian's clipped AABB with alpha >= 1/255 accepts the Gaussian when a
// threshold u(frame, Gaussian, pixel) < alpha, and the framebuffer keeps the minimum packed
// (depth_bits << 32 | index) key. The threshold is a stateless function of (frame, Gaussian,
// pixel) and the merge is a minimum, so the result does not depend on which thread evaluates
// which fragment. This file uses that freedom for a B200-oriented schedule:
//
//  * rows, then spans: a warp expands its 32 Gaussians into AABB rows, 32 rows at a time, and
//    each lane computes the conservative x-span of the alpha >= 1/255 ellipse on its row (the AABB
//    corners, ~45% of its pixels, are never evaluated);
//  * a pixel-pair stream per warp: every non-empty span is published to a small shared-memory ring
//    (the row's alpha and threshold constants, its first pair in the warp's stream) and its first
//    pair sets one bit of a row-start bitmap; the warp then consumes the stream 32 pairs at a time,
//    one pair of adjacent pixels per lane, the owning row found with one popc of that bitmap word.
//    Rows of 1 to 128 pixels (almost all of them) so keep every lane busy, where walking one row
//    per lane made a warp step as often as its longest row needed (under half of the lane-steps
//    did work on the 6M-Gaussian 1080p scene). Both pixels' alpha exponents are evaluated with
//    packed FP32x2 instructions (fma/mul/sub .f32x2 of sm_100a, each element rounded like the scalar
//    instruction); each accepted pixel issues one predicated RED. Longer rows are walked one row per
//    lane;
//  * a device-side work queue for Gaussians covering more than kBigFragments pixels: their rows are
//    cut into chunks of about kChunkPixels pixels that a persistent kernel steals across all SMs (no
//    cross-warp tail, no host synchronisation). A chunk has R rows (a power of two <= 32) and each
//    row is split into 32 / R segments, one lane per segment, so wide footprints keep every lane
//    walking;
//  * u64 atomicMin (fire-and-forget RED) on the L2-resident framebuffer.
//
// Bit-exactness. The reference's alpha exponent `dx * (cx * dx + cy * dy) + cz * dy * dy` is
// contracted into fused multiply-adds differently by its scatter loops and by its hybrid gather
// kernel (measured on a B200 against the reference's own kernels over ~3.6e10 fragments):
//   scatter (accumulate_st_cu and hybrid::bin_cu):  fma(cz*dy, dy, dx * fma(cx, dx, cy*dy))
//   hybrid gather (hybrid::gather_cu):              fma(dx, fma(cx, dx, cy*dy), (cz*dy)*dy)
// Both forms are written out here with explicitly rounded intrinsics. With hybrid scheduling
// the reference gathers the Gaussians whose AABB exceeds 512 pixels (the first
// min(N, 2^20) of them, accumulate_hybrid.cu:26-27,98-111); those use the gather form.
#include <cstdint>
#include <cuda_runtime.h>
#include "sgs_internal.h"
#include "sgs_rows.cuh"

namespace sgs {
namespace {

constexpr uint32_t kBlock = 256;              // queue kernel
constexpr uint32_t kScatterBlock = 128;       // scatter kernel: 4 warps, each with its own pair stream
constexpr uint32_t kScatterWarps = kScatterBlock / 32;
constexpr uint32_t kScatterBlocksPerSM = 8;
// Pair stream of a scatter warp: ring of published rows and ring of row-start bitmap words (powers of
// two). At most 31 rows hold pairs left over from a window when a batch of 32 rows is published, so
// 64 ring entries hold every live row; a batch adds at most 32 x kStreamMaxPairs pairs, so 128
// bitmap words (4096 pairs) cover every pair not yet consumed.
constexpr uint32_t kStreamRows = 64;
constexpr uint32_t kStreamWords = 128;
// Rows with more pixels than 2 x kStreamMaxPairs are walked one row per lane instead.
constexpr uint32_t kStreamMaxPairs = 64;
constexpr uint32_t kFullMask = 0xffffffffu;
// Gaussians whose AABB exceeds this many pixels go to the work queue.
constexpr uint32_t kBigFragments = 2048;
// Pixels per stolen chunk of a queued Gaussian (whole rows, at most 32 of them).
constexpr uint32_t kChunkPixels = 2048;
constexpr uint32_t kQueueBlocksPerSM = 8;
// Hybrid scheduling: AABBs above this many pixels are gathered by the reference (accumulate_hybrid.cu:26).
constexpr uint32_t kBinningPixelThreshold = 512;
// Flag in RowGaussian::flags: evaluate with the hybrid gather's contraction.
constexpr uint32_t kGatherFormFlag = 0x80000000u;

// Per-Gaussian constants of the row/span expansion (64 bytes, four 16-byte words).
struct RowGaussian {
    float mx, my;       // mean2d - 0.5: pixel (x, y) has delta (x - mx, y - my)
    float cx, cy;       // exp2-scaled conic (x, y)
    float cz;           // exp2-scaled conic z
    float opacity;
    SpanConstants span; // conservative row spans (sgs_rows.cuh)
    uint32_t key_lo, key_hi;
    uint32_t x_min;
    uint32_t y_min, w;
    uint32_t row_first; // first row position in the warp's row list (level 1)
    uint32_t flags;     // kGatherFormFlag
};

// A published row of the pair stream (64 bytes, four 16-byte words): the packed alpha constants,
// then depth key and threshold seed, then where its pixels and pairs are.
struct __align__(16) StreamRow {
    float mx[2], cx[2];      // shifted mean x and exp2-scaled conic x, each twice (packed FP32x2 operands)
    float cydy[2], czdy[2];  // cy * dy and cz * dy, each twice
    float dy, opacity;
    uint32_t key_lo, key_hi;
    uint32_t seed;           // white noise: the row seed; blue noise: slice row texel | x offset << 16
    uint32_t x0;             // first pixel's x | kGatherFormFlag
    uint32_t start_len;      // first pair in the warp's stream | pixels << 24
    uint32_t index;          // framebuffer index of the first pixel
};
static_assert(sizeof(StreamRow) == 64, "four 16-byte words");

// Packed FP32x2 arithmetic (sm_100a): two independent round-to-nearest operations per instruction,
// bit-identical to the scalar __fsub_rn / __fmul_rn / __fmaf_rn of each element.
__device__ __forceinline__ unsigned long long f2_pack(const float lo, const float hi) {
    unsigned long long r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
    return r;
}
__device__ __forceinline__ float2 f2_unpack(const unsigned long long r) {
    float2 v;
    asm("mov.b64 {%0, %1}, %2;" : "=f"(v.x), "=f"(v.y) : "l"(r));
    return v;
}
__device__ __forceinline__ unsigned long long f2_fma(const unsigned long long a, const unsigned long long b,
                                                     const unsigned long long c) {
    unsigned long long d;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
    return d;
}
__device__ __forceinline__ unsigned long long f2_mul(const unsigned long long a, const unsigned long long b) {
    unsigned long long d;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ unsigned long long f2_add(const unsigned long long a, const unsigned long long b) {
    unsigned long long d;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ unsigned long long f2_sub(const unsigned long long a, const unsigned long long b) {
    unsigned long long d;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}

// Bits of 1 + u for the white-noise threshold u of pixel x on a row with seed
// gaussian ^ frame * 1973 ^ y * 2699 (pcg_hash of math_utils.h:113-122; ((w >> 22) ^ w) >> 9 is
// written as (w >> 9) ^ (w >> 31)).
__device__ __forceinline__ uint32_t st_threshold_bits(const uint32_t row_seed, const uint32_t x) {
    const uint32_t state = (row_seed ^ (x * 9277u)) * 747796405u + 2891336453u;
    const uint32_t word = ((state >> ((state >> 28u) + 4u)) ^ state) * 277803737u;
    return 0x3f800000u | ((word >> 9u) ^ (word >> 31u));
}

// Blue-noise threshold of pixel x on a row whose slice row starts at texel `row_texel`, with the
// Gaussian's x offset bx (math_utils.h:125-136).
__device__ __forceinline__ float st_blue_threshold(const FrameRng& rng, const uint32_t row_texel, const uint32_t x,
                                                   const uint32_t bx) {
    const uint32_t texel = row_texel + ((x + bx) % kBlueNoiseWidth);
    const uint32_t value = (static_cast<uint32_t>(rng.slice[texel]) << 24u) + (1u << 23u) + rng.rotation;
    return static_cast<float>(value >> 8u) * 5.9604644775390625e-8f;
}

// Per-row random-number seed: the white-noise seed of row y, or the blue-noise slice row with the
// Gaussian's x offset in `bx` (math_utils.h:119-136).
template <bool kBlue>
__device__ __forceinline__ uint32_t row_seed(const FrameRng& rng, const uint32_t key_lo, const uint32_t y,
                                             uint32_t& bx) {
    if (kBlue) {
        const uint32_t oy = (key_lo * 0x91E10DA5u) >> 25u;
        bx = (key_lo * 0xC13FA9A9u) >> 25u;
        return ((y + oy) % kBlueNoiseHeight) * kBlueNoiseWidth;
    }
    bx = 0;
    return key_lo ^ (rng.frame * 1973u) ^ (y * 2699u);
}

// One predicated 64-bit RED.MIN (no branch around it).
__device__ __forceinline__ void red_min_if(unsigned long long* address, const unsigned long long key, const bool pred) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.u32 p, %2, 0;\n\t@p red.relaxed.gpu.global.min.u64 [%0], %1;\n\t}" ::"l"(address),
        "l"(key), "r"(static_cast<uint32_t>(pred))
        : "memory");
}

// Alpha tests and thresholds of pixels x0 and x0 + 1 of one row (scatter_utils.cuh:35-46 per pixel):
// `px` points at pixel x0 of the framebuffer (of the first sample), fx holds (x0, x0 + 1) as floats,
// the other operands are the row's constants, each held twice for the packed FP32x2 instructions.
// in0 / in1: the pixel lies in the row's span. Every lane of the warp calls it (the callers keep the
// warp converged).
template <bool kBlue, bool kHybrid, bool kMulti>
__device__ __forceinline__ void eval_pair(const AccumulateParams& a, const FrameRng& rng, unsigned long long* px,
                                          const uint32_t x0, const unsigned long long fx,
                                          const unsigned long long mx2, const unsigned long long cx2,
                                          const unsigned long long cydy2, const unsigned long long czdy2,
                                          const unsigned long long dy2, const unsigned long long opacity2,
                                          const unsigned long long key, const uint32_t seed, const uint32_t bx,
                                          const bool gather_form, const bool in0, const bool in1) {
    // alpha of both pixels with the reference's contraction of the exponent
    const unsigned long long dx = f2_sub(fx, mx2);
    const unsigned long long inner = f2_fma(cx2, dx, cydy2);
    const unsigned long long e2 =
        kHybrid && gather_form ? f2_fma(dx, inner, f2_mul(czdy2, dy2)) : f2_fma(czdy2, dy2, f2_mul(dx, inner));
    const float2 e = f2_unpack(e2);
    const float2 alpha = f2_unpack(f2_mul(opacity2, f2_pack(exp2f(fminf(e.x, 0.0f)), exp2f(fminf(e.y, 0.0f)))));
    if (!kMulti) {
        float2 u;
        if (kBlue) {
            u = make_float2(st_blue_threshold(rng, seed, x0, bx), st_blue_threshold(rng, seed, x0 + 1u, bx));
        } else {
            u = f2_unpack(f2_sub(f2_pack(__uint_as_float(st_threshold_bits(seed, x0)),
                                         __uint_as_float(st_threshold_bits(seed, x0 + 1u))),
                                 f2_pack(1.0f, 1.0f)));
        }
        red_min_if(px, key, in0 && alpha.x >= kMinAlpha && u.x < alpha.x);
        red_min_if(px + 1, key, in1 && alpha.y >= kMinAlpha && u.y < alpha.y);
    } else {
        // the same two pixels in every sample of the call: alpha once, one threshold per frame
        const bool ok0 = in0 && alpha.x >= kMinAlpha;
        const bool ok1 = in1 && alpha.y >= kMinAlpha;
        unsigned long long* px_s = px;
        for (uint32_t sm = 0; sm < a.n_samples; ++sm, px_s += a.fb_stride) {
            const uint32_t frame = rng.frame + sm;
            float2 u;
            if (kBlue) {
                const FrameRng rs = frame_rng_at(a, frame);
                u = make_float2(st_blue_threshold(rs, seed, x0, bx), st_blue_threshold(rs, seed, x0 + 1u, bx));
            } else {
                // row seeds differ between frames only in the frame term
                const uint32_t seed_s = seed ^ ((rng.frame * 1973u) ^ (frame * 1973u));
                u = f2_unpack(f2_sub(f2_pack(__uint_as_float(st_threshold_bits(seed_s, x0)),
                                             __uint_as_float(st_threshold_bits(seed_s, x0 + 1u))),
                                     f2_pack(1.0f, 1.0f)));
            }
            red_min_if(px_s, key, ok0 && u.x < alpha.x);
            red_min_if(px_s + 1, key, ok1 && u.y < alpha.y);
        }
    }
}

// Each lane walks segment `seg` of `1 << log_segs` equal parts of the span of its row y (when
// valid), two pixels per step; the warp takes as many steps as its longest segment needs. Used for
// queued Gaussians' chunks, rows longer than the pair stream takes, and the queue's overflow.
template <bool kBlue, bool kHybrid, bool kMulti>
__device__ __forceinline__ void walk_rows(const AccumulateParams& a, const FrameRng& rng, const bool valid,
                                          const RowGaussian& G, const uint32_t y, const uint32_t seg = 0,
                                          const uint32_t log_segs = 0) {
    uint32_t xs = 0, len = 0;
    float dy = 0.0f;
    if (valid) {
        dy = __fsub_rn(static_cast<float>(y), G.my);
        row_span(G.x_min, G.w, G.mx, G.span, dy, xs, len);
        if (log_segs > 0) {
            const uint32_t part = (len + (1u << log_segs) - 1u) >> log_segs;
            const uint32_t skip = min(seg * part, len);
            xs += skip;
            len = min(len - skip, part);
        }
    }
    const uint32_t steps = __reduce_max_sync(kFullMask, len);
    if (steps == 0) return;
    const float cydy = __fmul_rn(G.cy, dy);
    const float czdy = __fmul_rn(G.cz, dy);
    uint32_t bx;
    const uint32_t seed = row_seed<kBlue>(rng, G.key_lo, y, bx);
    const unsigned long long key = (static_cast<unsigned long long>(G.key_hi) << 32) | G.key_lo;
    const bool gather_form = kHybrid && (G.flags & kGatherFormFlag);
    unsigned long long* row = a.framebuffer + (static_cast<size_t>(y) * a.cam.width_int + xs);
    const unsigned long long mx2 = f2_pack(G.mx, G.mx), cx2 = f2_pack(G.cx, G.cx), cydy2 = f2_pack(cydy, cydy);
    const unsigned long long czdy2 = f2_pack(czdy, czdy), dy2 = f2_pack(dy, dy);
    const unsigned long long opacity2 = f2_pack(G.opacity, G.opacity);
    const unsigned long long two = f2_pack(2.0f, 2.0f);
    const float fxs = static_cast<float>(xs);  // pixel coordinates are exact in float
    unsigned long long fx = f2_pack(fxs, fxs + 1.0f);
    for (uint32_t i = 0; i < steps; i += 2) {
        eval_pair<kBlue, kHybrid, kMulti>(a, rng, row + i, xs + i, fx, mx2, cx2, cydy2, czdy2, dy2, opacity2, key,
                                          seed, bx, gather_form, i < len, i + 1u < len);
        fx = f2_add(fx, two);
    }
}

// One window of the pair stream: pairs [window, window + 32) of the warp's published rows, pair
// window + lane on this lane. `bits` marks the rows that start in the window (bit i: a row's first
// pair is window + i) and `rows_before` counts the rows that start before it, so the lane's row is
// row rows_before + popc(bits up to the lane) - 1 of the ring. Pairs at or past `end` are not
// evaluated.
template <bool kBlue, bool kHybrid, bool kMulti>
__device__ __forceinline__ void consume_pairs(const AccumulateParams& a, const FrameRng& rng,
                                              const StreamRow* __restrict__ ring, const uint32_t window,
                                              const uint32_t end, const uint32_t bits, const uint32_t rows_before,
                                              const uint32_t lane) {
    // Lanes past `end` in the last window may read a ring entry no row has written yet; the masks keep
    // their blue-noise texel inside the slice (their REDs are predicated off).
    constexpr uint32_t kBlueRowMask = (kBlueNoiseHeight - 1u) * kBlueNoiseWidth;
    const uint32_t q = window + lane;
    const uint32_t owner = rows_before + __popc(bits & (kFullMask >> (31u - lane))) - 1u;
    const ulonglong2* r = reinterpret_cast<const ulonglong2*>(ring + (owner & (kStreamRows - 1u)));
    const ulonglong2 w0 = r[0];
    const ulonglong2 w1 = r[1];
    const uint4 w2 = reinterpret_cast<const uint4*>(r)[2];
    const uint4 w3 = reinterpret_cast<const uint4*>(r)[3];
    const uint32_t start = w3.z & 0xffffffu;
    const uint32_t len = w3.z >> 24;
    const uint32_t j2 = 2u * (q - start);
    const uint32_t x = (w3.y & ~kGatherFormFlag) + j2;
    const float dy = __uint_as_float(w2.x);
    const float opacity = __uint_as_float(w2.y);
    const unsigned long long key = (static_cast<unsigned long long>(w2.w) << 32) | w2.z;
    const float fx = static_cast<float>(x);  // pixel coordinates are exact in float
    const bool in = q < end;
    eval_pair<kBlue, kHybrid, kMulti>(a, rng, a.framebuffer + (static_cast<size_t>(w3.w) + j2), x,
                                      f2_pack(fx, fx + 1.0f), w0.x, w0.y, w1.x, w1.y, f2_pack(dy, dy),
                                      f2_pack(opacity, opacity), key, kBlue ? (w3.x & kBlueRowMask) : w3.x,
                                      (w3.x >> 16) & (kBlueNoiseWidth - 1u), (w3.y & kGatherFormFlag) != 0, in,
                                      in && j2 + 1u < len);
}

// Rows per chunk of a queued Gaussian of AABB width w: about kChunkPixels pixels, a power of two
// between 1 and 32; each row of the chunk is walked in 32 / rows segments.
__device__ __forceinline__ uint32_t log_chunk_rows(const uint32_t w) {
    const uint32_t rows = max(1u, min(32u, kChunkPixels / max(w, 1u)));
    return 31u - __clz(rows);
}

// Rows [r0, r0 + (1 << log_rows)) of G, clipped to r_end: lane l walks segment l >> log_rows of row
// r0 + (l & (rows - 1)).
template <bool kBlue, bool kHybrid, bool kMulti>
__device__ __forceinline__ void walk_chunk(const AccumulateParams& a, const FrameRng& rng, const uint32_t lane,
                                           const RowGaussian& G, const uint32_t r0, const uint32_t log_rows,
                                           const uint32_t r_end) {
    const uint32_t r = r0 + (lane & ((1u << log_rows) - 1u));
    walk_rows<kBlue, kHybrid, kMulti>(a, rng, r < r_end, G, G.y_min + r, lane >> log_rows, 5u - log_rows);
}

// One thread per Gaussian (accumulate_scatter.cu:19-77 for the projection and the AABB).
template <bool kBlue, bool kHybrid, bool kMulti>
__global__ void __launch_bounds__(kScatterBlock, kScatterBlocksPerSM) st_scatter_kernel(const AccumulateParams a) {
    __shared__ RowGaussian s_gauss[kScatterWarps][32];
    __shared__ StreamRow s_ring[kScatterWarps][kStreamRows];
    __shared__ uint32_t s_bits[kScatterWarps][kStreamWords];

    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t wib = threadIdx.x >> 5;
    const uint32_t lt_mask = (1u << lane) - 1u;
    const uint32_t upto_mask = kFullMask >> (31u - lane);
    const uint32_t idx = blockIdx.x * kScatterBlock + threadIdx.x;
    bool active = idx < a.n;
    const uint32_t g = active ? idx : a.n - 1;

    Projected p;
    if (!project_gaussian(active, g, a.means, a.scales, a.rotations, a.opacities, a.w2c, a.cam, p, a.pre, a.quant)) return;
    const FrameRng rng = frame_rng(a);

    const PixelRect rect = pixel_rect(p.bounds, a.cam);
    const uint32_t count = active ? rect.width * rect.height : 0u;
    RowGaussian G;
    G.mx = p.mean2d.x - 0.5f;
    G.my = p.mean2d.y - 0.5f;
    const float3 ce = conic_for_exp2(p.conic);
    G.cx = ce.x;
    G.cy = ce.y;
    G.cz = ce.z;
    G.opacity = p.opacity;
    const unsigned long long key = pack_fragment(p.depth, g);
    G.key_lo = static_cast<uint32_t>(key);
    G.key_hi = static_cast<uint32_t>(key >> 32);
    G.x_min = rect.x_min;
    G.y_min = rect.y_min;
    G.w = rect.width;
    G.row_first = 0;
    G.flags = 0;
    G.span = span_constants(G.cx, G.cy, G.cz, G.opacity);

    if (kHybrid) {
        // the reference gathers the first min(N, 2^20) Gaussians with more than 512 pixels
        const bool binned = active && count > kBinningPixelThreshold;
        const uint32_t ballot = __ballot_sync(kFullMask, binned);
        if (ballot != 0) {
            const uint32_t leader = __ffs(ballot) - 1;
            uint32_t base = 0;
            if (lane == leader) base = atomicAdd(&a.queue->binned, static_cast<unsigned>(__popc(ballot)));
            base = __shfl_sync(kFullMask, base, leader);
            if (binned && base + __popc(ballot & lt_mask) < a.max_binned) G.flags = kGatherFormFlag;
        }
    }

    // large footprints: reserve row chunks in the work queue (or keep them when it is full)
    bool keep_big = false;
    bool has_rows = count > 0;
    if (count > kBigFragments) {
        has_rows = false;
        const uint32_t log_rpc = log_chunk_rows(rect.width);
        const uint32_t chunks = (rect.height + (1u << log_rpc) - 1u) >> log_rpc;
        const unsigned long long old = atomicAdd(&a.queue->packed, (1ull << kQueueEntryShift) | chunks);
        const uint32_t e = static_cast<uint32_t>(old >> kQueueEntryShift);
        const unsigned long long first_chunk = old & kQueueChunkMask;
        if (e < a.q.capacity && first_chunk + chunks <= kMaxQueueChunks) {
            a.q.key[e] = key;
            a.q.geom[e] = make_float4(G.mx, G.my, G.cx, G.cy);
            a.q.geom2[e] = make_float4(G.cz, G.opacity, __uint_as_float(rect.x_min), __uint_as_float(rect.width));
            a.q.meta[e] = make_uint4(rect.y_min, rect.height, log_rpc | G.flags, static_cast<uint32_t>(first_chunk));
        } else {
            keep_big = true;
            atomicAdd(&a.queue->overflow, 1u);
            // an entry past 32-bit chunk indices is marked unused (the marked entries are the last ones:
            // entries and chunks are reserved together)
            if (e < a.q.capacity) a.q.meta[e] = make_uint4(0u, 0u, 0u, kUnusedQueueEntry);
        }
    }

    // level 1: the rows of this warp's Gaussians, end to end in lane order, 32 rows at a time. A row's
    // owner is found as the ordinal of its Gaussian among the warp's Gaussians with rows (the count of
    // row starts up to it), so each Gaussian's constants are stored at that ordinal
    const uint32_t h = has_rows ? rect.height : 0u;
    const uint32_t incl_rows = warp_inclusive_sum(h, lane);
    const uint32_t total_rows = __shfl_sync(kFullMask, incl_rows, 31);
    const uint32_t row_first = incl_rows - h;
    const uint32_t with_rows = __ballot_sync(kFullMask, has_rows);
    if (has_rows) {
        RowGaussian st = G;
        st.row_first = row_first;
        s_gauss[wib][__popc(with_rows & lt_mask)] = st;
    }
    StreamRow* ring = s_ring[wib];
    uint32_t* bitmap = s_bits[wib];
#pragma unroll
    for (uint32_t i = 0; i < kStreamWords / 32; ++i) bitmap[i * 32 + lane] = 0u;
    __syncwarp();

    // level 2: the pixel-pair stream of the rows' spans (see the file comment)
    uint32_t rows_head = 0;    // rows published
    uint32_t pairs_head = 0;   // pairs published
    uint32_t window = 0;       // first pair not yet consumed (a multiple of 32)
    uint32_t rows_before = 0;  // rows starting before `window`
    int prev = -1;
    for (uint32_t base = 0; base < total_rows; base += 32) {
        const uint32_t rel = row_first - base;
        const uint32_t bits = __reduce_or_sync(kFullMask, (has_rows && rel < 32u) ? (1u << rel) : 0u);
        const int owner = prev + __popc(bits & upto_mask);
        prev += __popc(bits);
        const uint32_t r = base + lane;
        const bool valid = r < total_rows;
        const RowGaussian rg = s_gauss[wib][valid ? owner : 0];
        const uint32_t y = rg.y_min + (r - rg.row_first);
        uint32_t xs = 0, len = 0;
        float dy = 0.0f;
        if (valid) {
            dy = __fsub_rn(static_cast<float>(y), rg.my);
            row_span(rg.x_min, rg.w, rg.mx, rg.span, dy, xs, len);
        }
        const bool long_row = len > 2u * kStreamMaxPairs;
        const uint32_t pairs = long_row ? 0u : (len + 1u) >> 1;
        const uint32_t published = __ballot_sync(kFullMask, pairs != 0u);
        const uint32_t incl_pairs = warp_inclusive_sum(pairs, lane);
        if (pairs != 0u) {
            const uint32_t start = pairs_head + incl_pairs - pairs;
            uint32_t bx;
            const uint32_t seed = row_seed<kBlue>(rng, rg.key_lo, y, bx);
            const float cydy = __fmul_rn(rg.cy, dy);
            const float czdy = __fmul_rn(rg.cz, dy);
            StreamRow sr;
            sr.mx[0] = sr.mx[1] = rg.mx;
            sr.cx[0] = sr.cx[1] = rg.cx;
            sr.cydy[0] = sr.cydy[1] = cydy;
            sr.czdy[0] = sr.czdy[1] = czdy;
            sr.dy = dy;
            sr.opacity = rg.opacity;
            sr.key_lo = rg.key_lo;
            sr.key_hi = rg.key_hi;
            sr.seed = kBlue ? (seed | (bx << 16)) : seed;
            sr.x0 = xs | (kHybrid ? (rg.flags & kGatherFormFlag) : 0u);
            sr.start_len = start | (len << 24);
            sr.index = y * a.cam.width_int + xs;
            ring[(rows_head + __popc(published & lt_mask)) & (kStreamRows - 1u)] = sr;
            atomicOr(&bitmap[(start >> 5) & (kStreamWords - 1u)], 1u << (start & 31u));
        }
        rows_head += __popc(published);
        pairs_head += __shfl_sync(kFullMask, incl_pairs, 31);
        __syncwarp();
        // consume every full window of 32 pairs
        while (pairs_head - window >= 32u) {
            const uint32_t word = (window >> 5) & (kStreamWords - 1u);
            const uint32_t starts = bitmap[word];
            consume_pairs<kBlue, kHybrid, kMulti>(a, rng, ring, window, pairs_head, starts, rows_before, lane);
            rows_before += __popc(starts);
            window += 32u;
            __syncwarp();
            if (lane == 0) bitmap[word] = 0u;
        }
        // the few rows longer than the stream takes: one row per lane
        if (__any_sync(kFullMask, long_row)) walk_rows<kBlue, kHybrid, kMulti>(a, rng, long_row, rg, y);
        __syncwarp();
    }
    if (pairs_head > window) {
        const uint32_t starts = bitmap[(window >> 5) & (kStreamWords - 1u)];
        consume_pairs<kBlue, kHybrid, kMulti>(a, rng, ring, window, pairs_head, starts, rows_before, lane);
    }

    // queue overflow: the warp processes its kept large Gaussians, 32 rows at a time
    uint32_t pending = __ballot_sync(kFullMask, keep_big);
    while (pending) {
        const uint32_t src = __ffs(pending) - 1;
        pending &= pending - 1;
        const uint32_t bh = __shfl_sync(kFullMask, rect.height, src);
        __syncwarp();
        if (lane == src) s_gauss[wib][0] = G;
        __syncwarp();
        const RowGaussian bg = s_gauss[wib][0];
        for (uint32_t r0 = 0; r0 < bh; r0 += 32)
            walk_rows<kBlue, kHybrid, kMulti>(a, rng, r0 + lane < bh, bg, bg.y_min + r0 + lane);
    }
}

// Persistent consumer of the large-Gaussian queue: each warp steals one chunk of rows at a time.
template <bool kBlue, bool kHybrid, bool kMulti>
__global__ void __launch_bounds__(kBlock) st_queue_kernel(const AccumulateParams a) {
    const uint32_t lane = threadIdx.x & 31u;
    const unsigned long long packed = a.queue->packed;
    const FrameRng rng = frame_rng(a);
    const uint32_t n_entries =
        static_cast<uint32_t>(min(packed >> kQueueEntryShift, static_cast<unsigned long long>(a.q.capacity)));
    if (n_entries == 0) return;
    uint32_t last_entry = n_entries - 1;  // the last used entry; entry 0 starts at chunk 0 and always is
    if (a.q.meta[last_entry].w == kUnusedQueueEntry)
        last_entry = queue_entry_of_chunk(a.q.meta, n_entries, kUnusedQueueEntry - 1u, lane);
    const uint4 last = a.q.meta[last_entry];
    const uint32_t last_log_rpc = last.z & ~kGatherFormFlag;
    const uint32_t n_chunks = last.w + ((last.y + (1u << last_log_rpc) - 1u) >> last_log_rpc);
    for (;;) {
        uint32_t c = 0;
        if (lane == 0) c = atomicAdd(&a.queue->next_chunk, 1u);
        c = __shfl_sync(kFullMask, c, 0);
        if (c >= n_chunks) break;
        const uint32_t lo = queue_entry_of_chunk(a.q.meta, n_entries, c, lane);
        const uint4 m = a.q.meta[lo];
        const float4 gm = a.q.geom[lo];
        const float4 gm2 = a.q.geom2[lo];
        const unsigned long long key = a.q.key[lo];
        RowGaussian G;
        G.mx = gm.x;
        G.my = gm.y;
        G.cx = gm.z;
        G.cy = gm.w;
        G.cz = gm2.x;
        G.opacity = gm2.y;
        G.key_lo = static_cast<uint32_t>(key);
        G.key_hi = static_cast<uint32_t>(key >> 32);
        G.x_min = __float_as_uint(gm2.z);
        G.w = __float_as_uint(gm2.w);
        G.y_min = m.x;
        G.row_first = 0;
        G.flags = m.z & kGatherFormFlag;
        G.span = span_constants(G.cx, G.cy, G.cz, G.opacity);
        const uint32_t log_rpc = m.z & ~kGatherFormFlag;
        const uint32_t r0 = (c - m.w) << log_rpc;
        if (r0 >= m.y || G.w == 0 || log_rpc > 5u) {
            if (lane == 0) atomicOr(&a.queue->error, 1u);
            continue;
        }
        walk_chunk<kBlue, kHybrid, kMulti>(a, rng, lane, G, r0, log_rpc, m.y);
    }
}

__global__ void clear_kernel(unsigned long long* __restrict__ fb, const size_t n_fb, WorkQueue* __restrict__ queue) {
    const size_t stride = static_cast<size_t>(gridDim.x) * blockDim.x;
    const size_t tid = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    ulonglong2* fb2 = reinterpret_cast<ulonglong2*>(fb);
    const size_t n2 = n_fb / 2;
    for (size_t i = tid; i < n2; i += stride) fb2[i] = make_ulonglong2(kEmptyFragment, kEmptyFragment);
    if (tid == 0) {
        if (n_fb & 1) fb[n_fb - 1] = kEmptyFragment;
        if (queue != nullptr) {
            queue->packed = 0;
            queue->next_chunk = 0;
            queue->overflow = 0;
            queue->error = 0;
            queue->binned = 0;
        }
    }
}

template <bool kBlue, bool kHybrid, bool kMulti>
void launch_st(const AccumulateParams& p, const unsigned grid, const unsigned queue_grid, cudaStream_t stream) {
    st_scatter_kernel<kBlue, kHybrid, kMulti><<<grid, kScatterBlock, 0, stream>>>(p);
    st_queue_kernel<kBlue, kHybrid, kMulti><<<queue_grid, kBlock, 0, stream>>>(p);
}

template <bool kMulti>
void launch_st_variant(const AccumulateParams& p, const unsigned grid, const unsigned queue_grid, cudaStream_t stream) {
    const bool blue = p.blue_noise != nullptr;
    if (blue && p.hybrid) launch_st<true, true, kMulti>(p, grid, queue_grid, stream);
    else if (blue) launch_st<true, false, kMulti>(p, grid, queue_grid, stream);
    else if (p.hybrid) launch_st<false, true, kMulti>(p, grid, queue_grid, stream);
    else launch_st<false, false, kMulti>(p, grid, queue_grid, stream);
}

}  // namespace

cudaError_t launch_clear(unsigned long long* framebuffer, const size_t n_fb, WorkQueue* queue, const int num_sms,
                         cudaStream_t stream) {
    size_t need = (n_fb / 2 + 255) / 256;
    const size_t cap = static_cast<size_t>(num_sms) * 16;
    if (need > cap) need = cap;
    if (need < 1) need = 1;
    clear_kernel<<<static_cast<unsigned>(need), 256, 0, stream>>>(framebuffer, n_fb, queue);
    return cudaGetLastError();
}

cudaError_t launch_accumulate_st(const AccumulateParams& p, const int num_sms, cudaStream_t stream) {
    if (p.n == 0) return cudaSuccess;
    const unsigned grid = (p.n + kScatterBlock - 1) / kScatterBlock;
    const unsigned queue_grid = static_cast<unsigned>(num_sms) * kQueueBlocksPerSM;
    if (p.n_samples > 1) launch_st_variant<true>(p, grid, queue_grid, stream);
    else launch_st_variant<false>(p, grid, queue_grid, stream);
    return cudaGetLastError();
}

}  // namespace sgs
