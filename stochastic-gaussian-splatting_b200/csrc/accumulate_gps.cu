// Gaussian point splatting accumulation (USE_GPS), scatter and hybrid scheduling.
//
// Follows accumulate_scatter.cu:79-146, scatter_utils.cuh:98-183 and accumulate_hybrid_gps.cu:27-181.
// Each Gaussian emits min(Poisson(2 pi sqrt(det) dilog(opacity)), cap) points drawn from its
// opacity-truncated 2-D distribution; a point that lands in the framebuffer and whose pixel
// centre lies inside the alpha threshold merges the Gaussian's key with a u64 atomicMin.
//
// The scatter path's random numbers are a per-lane stream: lane l of the warp that owns
// Gaussians [32w, 32w + 32) draws from seed(32w + l) for its own first <= 4 points and then,
// in the cooperative phase, for every point it evaluates of the warp's larger Gaussians, in lane
// order. The winners therefore depend on that exact warp grouping and draw order, and this
// kernel keeps both (culled and padding lanes still draw their Poisson sample). It evaluates the
// points in another order where that pays: the last partial row of each cooperative Gaussian is
// drawn in stream order, parked as stream states in a per-warp buffer and evaluated 32 at a time
// whatever Gaussian it belongs to.
//
// Hybrid scheduling bins the Gaussians with more than 512 points (up to max_binned of them) into
// the device-side work queue; their points use counter-based seeds (seed ^ point * golden
// ratio), so the queue's persistent consumer may process their 256-point chunks in any order.
// Unlike the reference there is no host synchronisation between the passes.
#include <cstdint>
#include <cuda_runtime.h>
#include "sgs_internal.h"

namespace sgs {
namespace {

constexpr uint32_t kBlock = 256;
constexpr uint32_t kFullMask = 0xffffffffu;
constexpr uint32_t kBinningPointThreshold = 512;  // accumulate_hybrid_gps.cu:21
constexpr uint32_t kChunkPoints = 256;             // accumulate_hybrid_gps.cu:19
constexpr uint32_t kQueueBlocksPerSM = 8;
constexpr uint32_t kItemsPerWarp = 128;  // parked cooperative points per warp (multiple of 32)
constexpr uint32_t kChunksPerClaim = 8;  // chunks a consumer warp takes per atomic on the cursor

struct PointSource {
    float2 mean2d;
    float3 conic;
    float3 L;  // Cholesky factor of the 2-D covariance: (l11, l21, l22)
    float power_threshold;
    float opacity_rcp;
    float opacity_dilog;
    unsigned long long key;
};

// Merges the point drawn from uniforms `u` (scatter_utils.cuh:116-129; gps_point draws them from
// `seed` first). kFilter first reads the
// pixel's current key (a relaxed load at GPU scope) and skips the atomic when that key is already
// <= the point's: keys only decrease during a pass, so such a point cannot change the minimum, and
// the framebuffer ends with the same bits while the L2 atomic units see far fewer operations.
template <bool kFilter = false>
__device__ __forceinline__ void gps_point_at(const AccumulateParams& a, unsigned long long* __restrict__ fb,
                                             const float2 u, const PointSource& s) {
    const float2 xy = truncated_box_muller(u.x, u.y, s.opacity_rcp, s.opacity_dilog);
    const float sx = s.mean2d.x + s.L.x * xy.x;
    const float sy = s.mean2d.y + (s.L.y * xy.x + s.L.z * xy.y);
    if (sx >= a.cam.width || sx < 0.0f || sy >= a.cam.height || sy < 0.0f) return;
    const float dcx = truncf(sx) + 0.5f - s.mean2d.x;
    const float dcy = truncf(sy) + 0.5f - s.mean2d.y;
    const float power = 0.5f * (s.conic.x * dcx * dcx + s.conic.z * dcy * dcy) + s.conic.y * dcx * dcy;
    if (power > s.power_threshold) return;
    const uint32_t px = __float2uint_rd(sx);
    const uint32_t py = __float2uint_rd(sy);
    unsigned long long* const pixel = &fb[py * a.cam.width_int + px];
    if constexpr (kFilter) {
        unsigned long long current;
        asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(current) : "l"(pixel));
        if (current <= s.key) return;
    }
    atomicMin(pixel, s.key);
}

template <bool kFilter = false>
__device__ __forceinline__ void gps_point(const AccumulateParams& a, unsigned long long* __restrict__ fb, uint2& seed,
                                          const PointSource& s) {
    gps_point_at<kFilter>(a, fb, pcg2d_uniform(seed), s);
}

// The pixel the point drawn from uniforms `u` lands on, or null when it leaves the image or fails the
// power test (the tests of gps_point_at).
__device__ __forceinline__ unsigned long long* gps_point_pixel(const AccumulateParams& a,
                                                                unsigned long long* __restrict__ fb, const float2 u,
                                                                const PointSource& s) {
    const float2 xy = truncated_box_muller(u.x, u.y, s.opacity_rcp, s.opacity_dilog);
    const float sx = s.mean2d.x + s.L.x * xy.x;
    const float sy = s.mean2d.y + (s.L.y * xy.x + s.L.z * xy.y);
    if (sx >= a.cam.width || sx < 0.0f || sy >= a.cam.height || sy < 0.0f) return nullptr;
    const float dcx = truncf(sx) + 0.5f - s.mean2d.x;
    const float dcy = truncf(sy) + 0.5f - s.mean2d.y;
    const float power = 0.5f * (s.conic.x * dcx * dcx + s.conic.z * dcy * dcy) + s.conic.y * dcx * dcy;
    if (power > s.power_threshold) return nullptr;
    return &fb[__float2uint_rd(sy) * a.cam.width_int + __float2uint_rd(sx)];
}

// `n` points per lane (the same n on every lane) drawn in order from the lane's stream, kGroup at a
// time: the group's pixels first, then their keys read together (relaxed loads at GPU scope), then the
// atomics the keys leave (the filter of gps_point_at, its loads overlapped instead of one per point).
constexpr uint32_t kFilterGroup = 4;
__device__ __forceinline__ void gps_points_filtered(const AccumulateParams& a, unsigned long long* __restrict__ fb,
                                                    uint2& seed, const PointSource& s, const uint32_t n) {
    uint32_t i = 0;
    for (; i + kFilterGroup <= n; i += kFilterGroup) {
        unsigned long long* pixel[kFilterGroup];
#pragma unroll
        for (uint32_t k = 0; k < kFilterGroup; ++k) pixel[k] = gps_point_pixel(a, fb, pcg2d_uniform(seed), s);
        unsigned long long current[kFilterGroup];
#pragma unroll
        for (uint32_t k = 0; k < kFilterGroup; ++k) {
            current[k] = 0ull;
            if (pixel[k] != nullptr) asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(current[k]) : "l"(pixel[k]));
        }
#pragma unroll
        for (uint32_t k = 0; k < kFilterGroup; ++k)
            if (pixel[k] != nullptr && current[k] > s.key) atomicMin(pixel[k], s.key);
    }
    for (; i < n; ++i) gps_point<true>(a, fb, seed, s);
}

__device__ __forceinline__ PointSource shfl_source(const PointSource& s, const uint32_t src) {
    PointSource o;
    o.mean2d = make_float2(__shfl_sync(kFullMask, s.mean2d.x, src), __shfl_sync(kFullMask, s.mean2d.y, src));
    o.conic = make_float3(__shfl_sync(kFullMask, s.conic.x, src), __shfl_sync(kFullMask, s.conic.y, src),
                          __shfl_sync(kFullMask, s.conic.z, src));
    o.L = make_float3(__shfl_sync(kFullMask, s.L.x, src), __shfl_sync(kFullMask, s.L.y, src),
                      __shfl_sync(kFullMask, s.L.z, src));
    o.power_threshold = __shfl_sync(kFullMask, s.power_threshold, src);
    o.opacity_rcp = __shfl_sync(kFullMask, s.opacity_rcp, src);
    o.opacity_dilog = __shfl_sync(kFullMask, s.opacity_dilog, src);
    o.key = __shfl_sync(kFullMask, s.key, src);
    return o;
}

// Evaluates the n parked points of the warp's cooperative phase, 32 at a time: buffer item b holds
// the stepped stream state of its point and the lane whose Gaussian it belongs to.
__device__ __forceinline__ void evaluate_parked(const AccumulateParams& a, unsigned long long* __restrict__ fb,
                                                const PointSource& s, const uint2* __restrict__ states,
                                                const uint8_t* __restrict__ srcs, const uint32_t n,
                                                const uint32_t lane) {
    __syncwarp();
    for (uint32_t base = 0; base < n; base += 32) {
        const uint32_t b = base + lane;
        const bool valid = b < n;
        const uint32_t src = valid ? srcs[b] : lane;
        const PointSource t = shfl_source(s, src);
        if (valid) gps_point_at(a, fb, pcg2d_to_uniform(states[b]), t);
    }
    __syncwarp();
}

// kHybrid: bins the Gaussians with many points into the queue; kMulti: a.n_samples frames, one
// framebuffer each (scatter scheduling only). Both are template switches so that the one-sample
// scatter kernel carries neither the frame loop nor the binning code.
template <bool kHybrid, bool kMulti>
__device__ __forceinline__ void gps_scatter(const AccumulateParams& a) {
    static_assert(!(kHybrid && kMulti), "several samples per call use scatter scheduling");
    __shared__ uint2 s_state[kBlock / 32][kItemsPerWarp];
    __shared__ uint8_t s_src[kBlock / 32][kItemsPerWarp];
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t warp = threadIdx.x >> 5;
    const uint32_t idx = blockIdx.x * kBlock + threadIdx.x;
    bool active = idx < a.n;
    const uint32_t g = active ? idx : a.n - 1;

    Projected p;
    if (!project_gaussian(active, g, a.means, a.scales, a.rotations, a.opacities, a.w2c, a.cam, p, a.pre, a.quant)) return;

    // expected point count from the truncated footprint's area and opacity, then its Poisson draw
    // (accumulate_scatter.cu:104-112)
    PointSource s;
    s.opacity_dilog = gps_dilog(p.opacity);
    const float importance = kTwoPi * sqrtf(p.determinant) * s.opacity_dilog;
    const uint32_t cap = a.max_fragments != 0
                             ? a.max_fragments
                             : __float2uint_rn(a.cam.width * a.cam.height / (2.0f * a.cam.ss * a.cam.ss));
    const float c0 = sqrtf(p.cov2d.x);
    const float c1 = p.cov2d.y / c0;
    const float c2 = sqrtf(p.cov2d.z - c1 * c1);
    s.mean2d = p.mean2d;
    s.conic = p.conic;
    s.L = make_float3(c0, c1, c2);
    s.power_threshold = p.power_threshold;
    s.opacity_rcp = 1.0f / fmaxf(p.opacity, 1.0e-37f);
    s.key = pack_fragment(p.depth, g);
    const bool projected = active;
    const uint32_t frame0 = frame_rng(a).frame;
    // several samples of one call (scatter scheduling only): the projection once, then each frame's
    // own point draws into its own framebuffer
    const uint32_t n_frames = kMulti ? a.n_samples : 1u;
    for (uint32_t sm = 0; sm < n_frames; ++sm) {
        unsigned long long* fb = kMulti ? a.framebuffer + sm * a.fb_stride : a.framebuffer;
        // every lane, culled or padding, draws its Poisson sample (accumulate_scatter.cu:104-124)
        uint2 seed = gps_seed(g, frame0 + sm);
        const uint32_t true_count = poisson_count(seed, importance);
        bool act = projected && true_count != 0;
        const uint32_t count = min(true_count, cap);
        if (__ballot_sync(kFullMask, act) == 0) continue;

        if constexpr (kHybrid) {
            // bin Gaussians with many points: one 64-bit atomic per warp reserves entries and chunks
            const bool want = act && count > kBinningPointThreshold;
            const uint32_t ballot = __ballot_sync(kFullMask, want);
            if (ballot != 0) {
                const uint32_t chunks = want ? (count + kChunkPoints - 1) / kChunkPoints : 0u;
                uint32_t incl = chunks;
#pragma unroll
                for (uint32_t o = 1; o < 32; o <<= 1) {
                    const uint32_t v = __shfl_up_sync(kFullMask, incl, o);
                    if (lane >= o) incl += v;
                }
                const uint32_t warp_chunks = __shfl_sync(kFullMask, incl, 31);
                const uint32_t leader = __ffs(ballot) - 1;
                unsigned long long base = 0;
                if (lane == leader)
                    base = atomicAdd(&a.queue->packed,
                                     (static_cast<unsigned long long>(__popc(ballot)) << kQueueEntryShift) | warp_chunks);
                base = __shfl_sync(kFullMask, base, leader);
                const uint32_t e = static_cast<uint32_t>(base >> kQueueEntryShift) + __popc(ballot & ((1u << lane) - 1u));
                const unsigned long long first_chunk = (base & kQueueChunkMask) + (incl - chunks);
                if (want && e < a.max_binned && e < a.q.capacity) {
                    if (first_chunk + chunks <= kMaxQueueChunks) {
                        a.q.key[e] = s.key;
                        a.q.geom[e] = make_float4(s.mean2d.x, s.mean2d.y, s.L.x, s.L.y);
                        a.q.geom2[e] = make_float4(s.L.z, s.power_threshold, s.opacity_rcp, s.opacity_dilog);
                        a.q.meta[e] = make_uint4(__float_as_uint(s.conic.x), __float_as_uint(s.conic.y),
                                                 __float_as_uint(s.conic.z), static_cast<uint32_t>(first_chunk));
                        a.q.count[e] = count;
                        act = false;
                    } else {
                        // past 32-bit chunk indices (where the reference's own chunk offsets wrap): the
                        // entry is marked unused and the Gaussian scattered. Entries and chunks are
                        // reserved together, so the marked entries are the queue's last ones.
                        a.q.meta[e] = make_uint4(0u, 0u, 0u, kUnusedQueueEntry);
                        a.q.count[e] = 0u;
                    }
                }
            }
        }

        // own first points, sequentially per lane (scatter_utils.cuh:34-47)
        for (uint32_t i = 0; act && i < count && i < kSequentialFragments; ++i) gps_point(a, fb, seed, s);

        // The rest cooperatively, the warp's larger Gaussians in lane order: point j (after the first
        // kSequentialFragments) of Gaussian src is drawn by lane j % 32 from its own stream, in (src, j)
        // order (scatter_utils.cuh:140-183). Whole rows of 32 points are evaluated as they are drawn;
        // the last partial row (fewer than 32 points, most of a short Gaussian's) is drawn in order but
        // parked in the warp's buffer, and full buffers are evaluated 32 points at a time whatever
        // Gaussian they belong to, so short Gaussians no longer leave most lanes idle.
        uint32_t pending = __ballot_sync(kFullMask, act && count > kSequentialFragments);
        uint32_t fill = 0;
        while (pending) {
            const uint32_t src = __ffs(pending) - 1;
            pending &= pending - 1;
            const uint32_t n_items = __shfl_sync(kFullMask, count, src) - kSequentialFragments;
            const uint32_t full = n_items & ~31u;
            if (full != 0) {
                const PointSource t = shfl_source(s, src);
                // Gaussians with more points than the binning threshold (heavy-tailed scenes; in hybrid
                // mode those beyond a full bin) mostly land on pixels that already hold a nearer key:
                // their points read the key first and skip those atomics. The hybrid kernel, which
                // meets them by the hundred thousand with a small max_binned, reads four points' keys
                // at a time; for the many small Gaussians of other scenes the extra loads would cost
                // more than they save.
                if (n_items + kSequentialFragments > kBinningPointThreshold) {
                    if (kHybrid) {
                        gps_points_filtered(a, fb, seed, t, full / 32u);
                    } else {
                        for (uint32_t j = lane; j < full; j += 32) gps_point<true>(a, fb, seed, t);
                    }
                } else {
                    for (uint32_t j = lane; j < full; j += 32) gps_point(a, fb, seed, t);
                }
            }
            const uint32_t rest = n_items - full;
            if (rest == 0) continue;
            if (fill + rest > kItemsPerWarp) {
                evaluate_parked(a, fb, s, s_state[warp], s_src[warp], fill, lane);
                fill = 0;
            }
            if (lane < rest) {
                pcg2d_step(seed);
                s_state[warp][fill + lane] = seed;
                s_src[warp][fill + lane] = static_cast<uint8_t>(src);
            }
            fill += rest;
        }
        if (fill != 0) evaluate_parked(a, fb, s, s_state[warp], s_src[warp], fill, lane);
    }
}

template <bool kMulti>
__global__ void __launch_bounds__(kBlock) gps_scatter_kernel(const AccumulateParams a) {
    gps_scatter<false, kMulti>(a);
}

// The hybrid kernel carries the key filter of overflowing large Gaussians; held to 5 resident blocks
// per SM (at most 51 registers, no spills) like the plain kernel's 47-48 registers give.
__global__ void __launch_bounds__(kBlock, 5) gps_scatter_hybrid_kernel(const AccumulateParams a) {
    gps_scatter<true, false>(a);
}

// Persistent consumer of the binned Gaussians: each warp steals kChunksPerClaim 256-point chunks at
// a time (accumulate_hybrid_gps.cu:126-181 with per-point counter-based seeds, so which warp draws
// which chunk does not change the winners).
__global__ void __launch_bounds__(kBlock, kQueueBlocksPerSM) gps_queue_kernel(const AccumulateParams a) {
    const uint32_t lane = threadIdx.x & 31u;
    const unsigned long long packed = a.queue->packed;
    const uint32_t cap = min(a.max_binned, a.q.capacity);
    const uint32_t n_entries = static_cast<uint32_t>(min(packed >> kQueueEntryShift, static_cast<unsigned long long>(cap)));
    if (n_entries == 0) return;
    // the last used entry (entry 0, which starts at chunk 0, always is); marked entries start past
    // every chunk, so the search below never lands on one
    uint32_t last = n_entries - 1;
    if (a.q.meta[last].w == kUnusedQueueEntry) last = queue_entry_of_chunk(a.q.meta, n_entries, kUnusedQueueEntry - 1u, lane);
    const uint32_t n_chunks = a.q.meta[last].w + (a.q.count[last] + kChunkPoints - 1) / kChunkPoints;
    const uint32_t frame = frame_rng(a).frame;
    for (;;) {
        uint32_t c0 = 0;
        if (lane == 0) c0 = atomicAdd(&a.queue->next_chunk, kChunksPerClaim);
        c0 = __shfl_sync(kFullMask, c0, 0);
        if (c0 >= n_chunks) break;
        const uint32_t c_end = min(c0 + kChunksPerClaim, n_chunks);
        // consecutive chunks of a claim mostly belong to one entry: search and load it only when a
        // chunk lies past the current entry's last chunk
        uint32_t entry_first = 0, entry_end = 0;
        PointSource s;
        uint32_t n_points = 0;
        uint2 base_seed = make_uint2(0u, 0u);
        for (uint32_t c = c0; c < c_end; ++c) {
            if (c >= entry_end) {
                const uint32_t lo = queue_entry_of_chunk(a.q.meta, n_entries, c, lane);
                const uint4 m = a.q.meta[lo];
                const float4 gm = a.q.geom[lo];
                const float4 gm2 = a.q.geom2[lo];
                s.key = a.q.key[lo];
                s.mean2d = make_float2(gm.x, gm.y);
                s.L = make_float3(gm.z, gm.w, gm2.x);
                s.power_threshold = gm2.y;
                s.opacity_rcp = gm2.z;
                s.opacity_dilog = gm2.w;
                s.conic = make_float3(__uint_as_float(m.x), __uint_as_float(m.y), __uint_as_float(m.z));
                n_points = a.q.count[lo];
                entry_first = m.w;
                entry_end = m.w + (n_points + kChunkPoints - 1) / kChunkPoints;
                base_seed = gps_seed(static_cast<uint32_t>(s.key), frame);
            }
            const uint32_t first_point = (c - entry_first) * kChunkPoints;
            for (uint32_t k = lane; k < kChunkPoints; k += 32) {
                const uint32_t point = first_point + k;
                if (point >= n_points) break;
                uint2 seed = base_seed;
                seed.x ^= point * 0x9E3779B9u;
                gps_point<true>(a, a.framebuffer, seed, s);
            }
        }
    }
}

}  // namespace

cudaError_t launch_accumulate_gps(const AccumulateParams& p, const int num_sms, cudaStream_t stream) {
    if (p.n == 0) return cudaSuccess;
    const unsigned grid = (p.n + kBlock - 1) / kBlock;
    if (p.hybrid) gps_scatter_hybrid_kernel<<<grid, kBlock, 0, stream>>>(p);
    else if (p.n_samples > 1) gps_scatter_kernel<true><<<grid, kBlock, 0, stream>>>(p);
    else gps_scatter_kernel<false><<<grid, kBlock, 0, stream>>>(p);
    if (p.hybrid) gps_queue_kernel<<<static_cast<unsigned>(num_sms) * kQueueBlocksPerSM, kBlock, 0, stream>>>(p);
    return cudaGetLastError();
}

}  // namespace sgs
