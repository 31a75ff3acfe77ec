// Stochastic-transparency accumulation: the closest accepted fragment per (sub)pixel.
//
// Semantics follow accumulate_scatter.cu:19-77 and scatter_utils.cuh:14-95 of the reference:
// every pixel of a Gaussian's clipped AABB with alpha >= 1/255 accepts the Gaussian when a
// threshold u(frame, Gaussian, pixel) < alpha, and the framebuffer keeps the minimum packed
// (depth_bits << 32 | index) key. The threshold is a stateless function of (frame, Gaussian,
// pixel) and the merge is a minimum, so the result does not depend on which thread evaluates
// which fragment. This file uses that freedom for a B200-oriented schedule:
//
//  * rows, then spans: a warp sorts its 32 Gaussians by their widest span (a bitonic network over
//    the lanes), expands them into AABB rows in that order, 32 rows at a time, and each lane
//    computes the conservative x-span of the alpha >= 1/255 ellipse on its row (the AABB corners,
//    ~45% of its pixels, are never evaluated);
//  * each lane then walks its own row two pixels per step, the alpha exponent of both pixels in
//    packed FP32x2 instructions (fma/mul/sub .f32x2 of sm_100a, each element rounded like the scalar
//    instruction), with no per-pixel owner lookup or shared-memory traffic; the warp steps as often
//    as its longest row needs, and each accepted pixel issues one predicated RED;
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

constexpr uint32_t kBlock = 256;
constexpr uint32_t kWarpsPerBlock = kBlock / 32;
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

// Sorting key of Gaussians without rows (they go after every Gaussian with rows).
constexpr uint32_t kNoRowsKey = (1u << 26) - 1u;

// Bitonic sort of one 32-bit value per lane, ascending over the lanes (values distinct).
__device__ __forceinline__ uint32_t warp_sort_ascending(uint32_t v, const uint32_t lane) {
#pragma unroll
    for (uint32_t k = 2; k <= 32; k <<= 1) {
#pragma unroll
        for (uint32_t j = k >> 1; j > 0; j >>= 1) {
            const uint32_t other = __shfl_xor_sync(kFullMask, v, j);
            const bool keep_min = ((lane & j) == 0) == ((lane & k) == 0);
            v = keep_min ? min(v, other) : max(v, other);
        }
    }
    return v;
}

// One predicated 64-bit RED.MIN (no branch around it).
__device__ __forceinline__ void red_min_if(unsigned long long* address, const unsigned long long key, const bool pred) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.u32 p, %2, 0;\n\t@p red.relaxed.gpu.global.min.u64 [%0], %1;\n\t}" ::"l"(address),
        "l"(key), "r"(static_cast<uint32_t>(pred))
        : "memory");
}

// Each lane walks segment `seg` of `1 << log_segs` equal parts of the span of its row y (when
// valid), two pixels per step; the warp takes as many steps as its longest segment needs
// (scatter_utils.cuh:35-46 per pixel).
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
        // alpha of pixels xs + i and xs + i + 1 with the reference's contraction of the exponent
        const unsigned long long dx = f2_sub(fx, mx2);
        const unsigned long long inner = f2_fma(cx2, dx, cydy2);
        const unsigned long long e2 =
            gather_form ? f2_fma(dx, inner, f2_mul(czdy2, dy2)) : f2_fma(czdy2, dy2, f2_mul(dx, inner));
        const float2 e = f2_unpack(e2);
        const float2 alpha =
            f2_unpack(f2_mul(opacity2, f2_pack(exp2f(fminf(e.x, 0.0f)), exp2f(fminf(e.y, 0.0f)))));
        const uint32_t x0 = xs + i;
        if (!kMulti) {
            float2 u;
            if (kBlue) {
                u = make_float2(st_blue_threshold(rng, seed, x0, bx), st_blue_threshold(rng, seed, x0 + 1u, bx));
            } else {
                u = f2_unpack(f2_sub(f2_pack(__uint_as_float(st_threshold_bits(seed, x0)),
                                             __uint_as_float(st_threshold_bits(seed, x0 + 1u))),
                                     f2_pack(1.0f, 1.0f)));
            }
            red_min_if(row + i, key, i < len && alpha.x >= kMinAlpha && u.x < alpha.x);
            red_min_if(row + i + 1u, key, i + 1u < len && alpha.y >= kMinAlpha && u.y < alpha.y);
        } else {
            // the same two pixels in every sample of the call: alpha once, one threshold per frame
            const bool in_x = i < len && alpha.x >= kMinAlpha;
            const bool in_y = i + 1u < len && alpha.y >= kMinAlpha;
            unsigned long long* row_s = row;
            for (uint32_t sm = 0; sm < a.n_samples; ++sm, row_s += a.fb_stride) {
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
                red_min_if(row_s + i, key, in_x && u.x < alpha.x);
                red_min_if(row_s + i + 1u, key, in_y && u.y < alpha.y);
            }
        }
        fx = f2_add(fx, two);
    }
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
__global__ void __launch_bounds__(kBlock, 4) st_scatter_kernel(const AccumulateParams a) {
    __shared__ RowGaussian s_gauss[kWarpsPerBlock][32];
    __shared__ uint32_t s_rank[kWarpsPerBlock][32];

    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t wib = threadIdx.x >> 5;
    const uint32_t lt_mask = (1u << lane) - 1u;
    const uint32_t upto_mask = kFullMask >> (31u - lane);
    const uint32_t idx = blockIdx.x * kBlock + threadIdx.x;
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

    // level 1: the rows of this warp's Gaussians, end to end, the Gaussians ordered by their widest
    // span so that the 32 rows walked together have similar lengths (a warp walks as long as its
    // longest row); Gaussians without rows go last
    uint32_t width_key = kNoRowsKey;
    if (has_rows) {
        uint32_t widest = G.w;
        if (G.span.k2 > 0.0f) {
            const float est = 2.0f * sqrtf(G.span.k2 * G.span.dymax2) + 2.0f;
            if (est < static_cast<float>(widest)) widest = static_cast<uint32_t>(est);
        }
        width_key = min(widest, kNoRowsKey - 1u);
    }
    const uint32_t sorted = warp_sort_ascending((width_key << 5) | lane, lane);  // lane i: i-th smallest
    const uint32_t src_lane = sorted & 31u;
    s_rank[wib][src_lane] = lane;
    const uint32_t h = has_rows ? rect.height : 0u;
    const uint32_t h_sorted = __shfl_sync(kFullMask, h, src_lane);
    const uint32_t incl_sorted = warp_inclusive_sum(h_sorted, lane);
    const uint32_t total_rows = __shfl_sync(kFullMask, incl_sorted, 31);
    __syncwarp();
    const uint32_t rank = s_rank[wib][lane];
    const uint32_t row_first = __shfl_sync(kFullMask, incl_sorted - h_sorted, rank);
    if (has_rows) {
        RowGaussian st = G;
        st.row_first = row_first;
        s_gauss[wib][rank] = st;
    }
    __syncwarp();
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
        walk_rows<kBlue, kHybrid, kMulti>(a, rng, valid, rg, y);
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
    st_scatter_kernel<kBlue, kHybrid, kMulti><<<grid, kBlock, 0, stream>>>(p);
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
    const unsigned grid = (p.n + kBlock - 1) / kBlock;
    const unsigned queue_grid = static_cast<unsigned>(num_sms) * kQueueBlocksPerSM;
    if (p.n_samples > 1) launch_st_variant<true>(p, grid, queue_grid, stream);
    else launch_st_variant<false>(p, grid, queue_grid, stream);
    return cudaGetLastError();
}

}  // namespace sgs
