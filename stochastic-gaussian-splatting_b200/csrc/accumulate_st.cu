// Stochastic-transparency accumulation: the closest accepted fragment per (sub)pixel.
//
// Semantics follow accumulate_scatter.cu:19-77 and scatter_utils.cuh:14-95 of the reference:
// every pixel of a Gaussian's clipped AABB with alpha >= 1/255 accepts the Gaussian when a
// threshold u(frame, Gaussian, pixel) < alpha, and the framebuffer keeps the minimum packed
// (depth_bits << 32 | index) key. The threshold is a stateless function of (frame, Gaussian,
// pixel) and the merge is a minimum, so the result does not depend on which thread evaluates
// which fragment. This file uses that freedom for a B200-oriented schedule:
//
//  * rows, then spans: a warp expands its 32 Gaussians into AABB rows, each lane computes the
//    conservative x-span of the alpha >= 1/255 ellipse on one row (the AABB corners, ~45% of
//    its pixels, are never evaluated), and the span pixels of 32 rows are laid end to end
//    across the lanes, so every lane evaluates one pixel per step whatever the footprint sizes;
//    the owner of a position is found with one redux.sync OR over the starts and a popc;
//  * a device-side work queue for Gaussians covering more than kBigFragments pixels: their rows
//    are cut into chunks that a persistent kernel steals across all SMs (no cross-warp tail,
//    no host synchronisation);
//  * u64 atomicMin (fire-and-forget RED) on the L2-resident framebuffer; consecutive lanes hit
//    consecutive pixels of a row, so each RED touches few L2 sectors.
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

namespace sgs {
namespace {

constexpr uint32_t kBlock = 256;
constexpr uint32_t kWarpsPerBlock = kBlock / 32;
constexpr uint32_t kFullMask = 0xffffffffu;
// Gaussians whose AABB exceeds this many pixels go to the work queue.
constexpr uint32_t kBigFragments = 2048;
// Target pixels per stolen chunk (whole rows; a single row wider than this is one chunk).
constexpr uint32_t kChunkFragments = 2048;
constexpr uint32_t kQueueBlocksPerSM = 8;
// Hybrid scheduling: AABBs above this many pixels are gathered by the reference (accumulate_hybrid.cu:26).
constexpr uint32_t kBinningPixelThreshold = 512;
// Safety margins of the row spans: exponent units (log2 of alpha) and pixels.
constexpr float kSpanExpMargin = 0.125f;
constexpr float kSpanPixelMargin = 0.02f;
// Flag in RowSlot::c.w: evaluate with the hybrid gather's contraction.
constexpr uint32_t kGatherFormFlag = 0x80000000u;

// Per-Gaussian constants of the row/span expansion (64 bytes, four 16-byte words).
struct RowGaussian {
    float mx, my;       // mean2d - 0.5: pixel (x, y) has delta (x - mx, y - my)
    float cx, cy;       // exp2-scaled conic (x, y)
    float cz;           // exp2-scaled conic z
    float opacity;
    float slope;        // row centre shift per unit dy
    float k2;           // squared half-width per unit of (dymax2 - dy^2); 0 disables spans
    float dymax2;       // rows with dy^2 > dymax2 hold no pixel with alpha >= 1/255
    uint32_t key_lo, key_hi;
    uint32_t x_min;
    uint32_t y_min, w;
    uint32_t row_first; // first row position in the warp's row list (level 1)
    uint32_t flags;     // kGatherFormFlag
};

// Span constants. For a row at offset dy the exponent is the concave quadratic
// e(dx) = cx dx^2 + cy dy dx + cz dy^2 with its maximum at dx = slope * dy; pixels with
// alpha >= 1/255 need e >= T = -log2(255 opacity). Using T minus kSpanExpMargin (far above the
// float error of e or of these constants, which enter only relative to |T|) and widening by
// kSpanPixelMargin gives a superset of the accepted pixels of every row.
__device__ __forceinline__ void span_constants(RowGaussian& G) {
    const float T = -log2f(G.opacity * kMinAlphaRcp) - kSpanExpMargin;
    const float P = 4.0f * G.cx * G.cz - G.cy * G.cy;  // > 0 for a positive-definite conic
    G.slope = 0.0f;
    G.k2 = 0.0f;
    G.dymax2 = 0.0f;
    if (P > 0.0f && G.cx < 0.0f && T < 0.0f) {
        const float inv_cx = 1.0f / G.cx;
        const float k2 = 0.25f * P * inv_cx * inv_cx;
        const float dymax2 = 4.0f * G.cx * T / P;
        const float slope = -0.5f * G.cy * inv_cx;
        if (isfinite(k2) && isfinite(dymax2) && isfinite(slope) && k2 > 0.0f) {
            G.k2 = k2;
            G.dymax2 = dymax2;
            G.slope = slope;
        }
    }
}

// Inclusive warp prefix sum.
__device__ __forceinline__ uint32_t warp_inclusive_sum(uint32_t v, const uint32_t lane) {
#pragma unroll
    for (uint32_t o = 1; o < 32; o <<= 1) {
        const uint32_t t = __shfl_up_sync(kFullMask, v, o);
        if (lane >= o) v += t;
    }
    return v;
}

// One row of span pixels ready for evaluation (48 bytes).
struct RowSlot {
    float4 a;  // mx, cx, cy * dy, cz * dy
    uint4 b;   // x offset (first x - first position), row base index (y * width), row seed / blue-noise row, dy bits
    uint4 c;   // opacity bits, key low, key high, blue-noise x offset | kGatherFormFlag
};

// Evaluates flattened position p (< total) of the row `r` that owns it (scatter_utils.cuh:35-46).
// Positions past the end evaluate a valid pixel of the same row and do not merge.
template <bool kBlue, bool kHybrid>
__device__ __forceinline__ void st_position(const AccumulateParams& a, const FrameRng& rng, const RowSlot& r,
                                            const uint32_t p, const uint32_t total) {
    const float4 ra = r.a;
    const uint4 rb = r.b;
    const uint4 rc = r.c;
    const bool in_range = p < total;
    const uint32_t x = (in_range ? p : total - 1u) + rb.x;
    const float dx = __fsub_rn(static_cast<float>(x), ra.x);
    const float rdy = __uint_as_float(rb.w);
    const float inner = __fmaf_rn(ra.y, dx, ra.z);
    float e = __fmaf_rn(ra.w, rdy, __fmul_rn(dx, inner));
    if (kHybrid && (rc.w & kGatherFormFlag)) e = __fmaf_rn(dx, inner, __fmul_rn(ra.w, rdy));
    const float alpha = __fmul_rn(__uint_as_float(rc.x), exp2f(fminf(e, 0.0f)));
    float u;
    if (kBlue) {
        const uint32_t texel = rb.z + ((x + (rc.w & 0x7fu)) % kBlueNoiseWidth);
        const uint32_t value =
            (static_cast<uint32_t>(rng.slice[texel]) << 24u) + (1u << 23u) + rng.rotation;
        u = static_cast<float>(value >> 8u) * 5.9604644775390625e-8f;
    } else {
        u = __uint_as_float(0x3f800000u | (pcg_hash(rb.z ^ (x * 9277u)) >> 9u)) - 1.0f;
    }
    if (in_range && alpha >= kMinAlpha && u < alpha) {
        const unsigned long long key = (static_cast<unsigned long long>(rc.z) << 32) | rc.y;
        atomicMin(&a.framebuffer[rb.y + x], key);
    }
}

// Each lane holds one row (valid) of Gaussian G at image row y. Computes the spans, lays the span
// pixels of the 32 rows end to end and evaluates them with all lanes (scatter_utils.cuh:35-46).
template <bool kBlue, bool kHybrid>
__device__ __forceinline__ void scatter_rows(const AccumulateParams& a, const FrameRng& rng, const uint32_t lane,
                                             const uint32_t lt_mask, const uint32_t upto_mask, RowSlot* s_rows,
                                             const bool valid, const RowGaussian& G, const uint32_t y) {
    uint32_t xs = 0, len = 0;
    float dy = 0.0f, cydy = 0.0f, czdy = 0.0f;
    if (valid) {
        dy = __fsub_rn(static_cast<float>(y), G.my);
        cydy = __fmul_rn(G.cy, dy);
        czdy = __fmul_rn(G.cz, dy);
        int lo = static_cast<int>(G.x_min);
        int hi = static_cast<int>(G.x_min + G.w) - 1;
        if (G.k2 > 0.0f) {
            const float rem = fmaf(-dy, dy, G.dymax2);
            if (rem < 0.0f) {
                hi = lo - 1;
            } else {
                const float hw = sqrtf(G.k2 * rem);
                const float c = fmaf(G.slope, dy, G.mx);
                const float eps = kSpanPixelMargin + 4.0e-6f * (fabsf(c) + hw);
                const float fl = ceilf(c - hw - eps);
                const float fh = floorf(c + hw + eps);
                // compare in float first: the span may lie far outside the int range of the AABB
                if (fl > static_cast<float>(hi) || fh < static_cast<float>(lo)) {
                    hi = lo - 1;
                } else {
                    if (fl > static_cast<float>(lo)) lo = static_cast<int>(fl);
                    if (fh < static_cast<float>(hi)) hi = static_cast<int>(fh);
                }
            }
        }
        if (hi >= lo) {
            xs = static_cast<uint32_t>(lo);
            len = static_cast<uint32_t>(hi - lo + 1);
        }
    }
    // compact the non-empty rows into shared memory, in lane order
    const uint32_t rmask = __ballot_sync(kFullMask, len > 0);
    if (rmask == 0) return;
    const uint32_t incl = warp_inclusive_sum(len, lane);
    const uint32_t total = __shfl_sync(kFullMask, incl, 31);
    const uint32_t first = incl - len;
    if (len > 0) {
        const uint32_t slot = __popc(rmask & lt_mask);
        uint32_t seed, bx = 0;
        if (kBlue) {
            const uint32_t oy = (G.key_lo * 0x91E10DA5u) >> 25u;
            bx = (G.key_lo * 0xC13FA9A9u) >> 25u;
            seed = ((y + oy) % kBlueNoiseHeight) * kBlueNoiseWidth;
        } else {
            seed = G.key_lo ^ (rng.frame * 1973u) ^ (y * 2699u);
        }
        RowSlot r;
        r.a = make_float4(G.mx, G.cx, cydy, czdy);
        r.b = make_uint4(xs - first, y * a.cam.width_int, seed, __float_as_uint(dy));
        r.c = make_uint4(__float_as_uint(G.opacity), G.key_lo, G.key_hi, bx | G.flags);
        s_rows[slot] = r;
    }
    __syncwarp();
    // two positions per lane and step (p and p + 32): one pass over 64 positions; the body is
    // straight-line code ending in one predicated RED
    int prev = -1;
    for (uint32_t base = 0; base < total; base += 64) {
        const uint32_t rel = first - base;
        const bool starts = len > 0 && rel < 64u;
        const uint32_t bits_lo = __reduce_or_sync(kFullMask, (starts && rel < 32u) ? (1u << rel) : 0u);
        const uint32_t bits_hi = __reduce_or_sync(kFullMask, (starts && rel >= 32u) ? (1u << (rel - 32u)) : 0u);
        const int n_lo = __popc(bits_lo);
        const int owner0 = prev + __popc(bits_lo & upto_mask);
        const int owner1 = prev + n_lo + __popc(bits_hi & upto_mask);
        prev += n_lo + __popc(bits_hi);
        st_position<kBlue, kHybrid>(a, rng, s_rows[owner0], base + lane, total);
        st_position<kBlue, kHybrid>(a, rng, s_rows[owner1], base + 32u + lane, total);
    }
    __syncwarp();
}

__device__ __forceinline__ uint32_t rows_per_chunk(const uint32_t w) { return max(1u, kChunkFragments / w); }

// One thread per Gaussian (accumulate_scatter.cu:19-77 for the projection and the AABB).
template <bool kBlue, bool kHybrid>
__global__ void __launch_bounds__(kBlock, 4) st_scatter_kernel(const AccumulateParams a) {
    __shared__ RowGaussian s_gauss[kWarpsPerBlock][32];
    __shared__ RowSlot s_rows[kWarpsPerBlock][32];

    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t wib = threadIdx.x >> 5;
    const uint32_t lt_mask = (1u << lane) - 1u;
    const uint32_t upto_mask = kFullMask >> (31u - lane);
    const uint32_t idx = blockIdx.x * kBlock + threadIdx.x;
    bool active = idx < a.n;
    const uint32_t g = active ? idx : a.n - 1;

    Projected p;
    if (!project_gaussian(active, g, a.means, a.scales, a.rotations, a.opacities, a.w2c, a.cam, p)) return;
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
    span_constants(G);

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
        const uint32_t rpc = rows_per_chunk(rect.width);
        const uint32_t chunks = (rect.height + rpc - 1) / rpc;
        const unsigned long long old = atomicAdd(&a.queue->packed, (1ull << kQueueEntryShift) | chunks);
        const uint32_t e = static_cast<uint32_t>(old >> kQueueEntryShift);
        const unsigned long long first_chunk = old & kQueueChunkMask;
        if (e < a.q.capacity && first_chunk + chunks <= 0xffffffffull) {
            a.q.key[e] = key;
            a.q.geom[e] = make_float4(G.mx, G.my, G.cx, G.cy);
            a.q.geom2[e] = make_float4(G.cz, G.opacity, __uint_as_float(rect.x_min), __uint_as_float(rect.width));
            a.q.meta[e] = make_uint4(rect.y_min, rect.height, rpc | G.flags, static_cast<uint32_t>(first_chunk));
        } else {
            keep_big = true;
            atomicAdd(&a.queue->overflow, 1u);
        }
    }

    // level 1: the rows of this warp's Gaussians, end to end
    const uint32_t gmask = __ballot_sync(kFullMask, has_rows);
    const uint32_t h = has_rows ? rect.height : 0u;
    const uint32_t row_incl = warp_inclusive_sum(h, lane);
    const uint32_t total_rows = __shfl_sync(kFullMask, row_incl, 31);
    const uint32_t row_first = row_incl - h;
    if (has_rows) {
        RowGaussian st = G;
        st.row_first = row_first;
        s_gauss[wib][__popc(gmask & lt_mask)] = st;
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
        scatter_rows<kBlue, kHybrid>(a, rng, lane, lt_mask, upto_mask, s_rows[wib], valid, rg, y);
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
        for (uint32_t r0 = 0; r0 < bh; r0 += 32) {
            const bool valid = r0 + lane < bh;
            scatter_rows<kBlue, kHybrid>(a, rng, lane, lt_mask, upto_mask, s_rows[wib], valid, bg, bg.y_min + r0 + lane);
        }
    }
}

// Persistent consumer of the large-Gaussian queue: each warp steals one chunk of rows at a time.
template <bool kBlue, bool kHybrid>
__global__ void __launch_bounds__(kBlock) st_queue_kernel(const AccumulateParams a) {
    __shared__ RowSlot s_rows[kWarpsPerBlock][32];
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t wib = threadIdx.x >> 5;
    const uint32_t lt_mask = (1u << lane) - 1u;
    const uint32_t upto_mask = kFullMask >> (31u - lane);
    const unsigned long long packed = a.queue->packed;
    const FrameRng rng = frame_rng(a);
    const uint32_t n_entries =
        static_cast<uint32_t>(min(packed >> kQueueEntryShift, static_cast<unsigned long long>(a.q.capacity)));
    if (n_entries == 0) return;
    const uint4 last = a.q.meta[n_entries - 1];
    const uint32_t last_rpc = last.z & ~kGatherFormFlag;
    const uint32_t n_chunks = last.w + (last.y + last_rpc - 1) / last_rpc;
    for (;;) {
        uint32_t c = 0;
        if (lane == 0) c = atomicAdd(&a.queue->next_chunk, 1u);
        c = __shfl_sync(kFullMask, c, 0);
        if (c >= n_chunks) break;
        // entry owning chunk c: the last one whose first chunk is <= c
        uint32_t lo = 0, hi = n_entries - 1;
        while (lo < hi) {
            const uint32_t mid = (lo + hi + 1) >> 1;
            if (a.q.meta[mid].w <= c) lo = mid;
            else hi = mid - 1;
        }
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
        span_constants(G);
        const uint32_t rpc = m.z & ~kGatherFormFlag;
        const uint32_t r0 = (c - m.w) * rpc;
        if (r0 >= m.y || G.w == 0 || rpc == 0) {
            if (lane == 0) atomicOr(&a.queue->error, 1u);
            continue;
        }
        const uint32_t r1 = min(r0 + rpc, m.y);
        for (uint32_t r = r0; r < r1; r += 32) {
            const bool valid = r + lane < r1;
            scatter_rows<kBlue, kHybrid>(a, rng, lane, lt_mask, upto_mask, s_rows[wib], valid, G, G.y_min + r + lane);
        }
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

template <bool kBlue, bool kHybrid>
void launch_st(const AccumulateParams& p, const unsigned grid, const unsigned queue_grid, cudaStream_t stream) {
    st_scatter_kernel<kBlue, kHybrid><<<grid, kBlock, 0, stream>>>(p);
    st_queue_kernel<kBlue, kHybrid><<<queue_grid, kBlock, 0, stream>>>(p);
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
    const bool blue = p.blue_noise != nullptr;
    if (blue && p.hybrid) launch_st<true, true>(p, grid, queue_grid, stream);
    else if (blue) launch_st<true, false>(p, grid, queue_grid, stream);
    else if (p.hybrid) launch_st<false, true>(p, grid, queue_grid, stream);
    else launch_st<false, false>(p, grid, queue_grid, stream);
    return cudaGetLastError();
}

}  // namespace sgs
