// Sample and resolve passes: colour of each (sub)pixel's winner, optional spatial reuse with the
// k-buffer, then the supersampling box filter and the temporal (Reset / Static / Reproject) merge.
//
// The arithmetic of every output follows resolve.cu:27-349 of the reference expression for
// expression, so that the outputs match it bit for bit when the winners match. The schedule is
// this file's own:
//  * Reset / Static without spatial reuse: one fused pass per image pixel
//    (sample_resolve_fused_kernel), several samples per call in one pass (samples_resolve_kernel);
//  * spatial reuse: reuse_sample_kernel evaluates each subpixel's winner, its resampling weights
//    and the k-buffer update, loading a k-buffer entry's occlusion factors only where they are
//    used; the neighbours' weights depend on their k-buffer before this sample's update, so the
//    resolve is a second pass;
//  * the resolve of spatial reuse and of Reproject (tile_resolve_kernel): one block per 32 x 8
//    image pixels stages the tile's samples and weights with a halo in shared memory once, instead of
//    every pixel gathering its neighbours from global memory; for Reproject it computes each pixel's
//    box-filtered YCoCg colour once for the 3 x 3 moment windows (the reference recomputes it in
//    all nine windows that contain it) and stages the history texels under the tile's reprojected
//    Catmull-Rom taps; without spatial reuse it evaluates the winners' colours itself from the
//    framebuffer (halo included), so sample and resolve are one pass.
#include <cstdint>
#include <cuda_runtime.h>
#include "sgs_internal.h"

namespace sgs {
namespace {

constexpr uint32_t kBlock = 256;
// spatio-temporal reuse constants (resolve.cu:16-23)
constexpr float kMaxAlpha = 0.99f;
constexpr float kHistoryWeight = 0.7f;
constexpr float kGammaStatic = 4.0f;
constexpr float kGammaMotion = 1.0f;
constexpr float kVelocityThreshold = 4.0f;
constexpr float kMinExtentLuma = 0.01f;
constexpr float kMinExtentChroma = 0.005f;
constexpr float kBorderMargin = 2.0f;

// Colour of Gaussian g in the quantised layout: its decoded position and half-precision SH. A
// separate, non-inlined function, so that the float32 path's code (whose rounding the reference's
// bits depend on) is compiled exactly as without it.
__device__ __noinline__ float3 quantized_color(const QuantizedModel q, const float* __restrict__ cam_position,
                                              const uint32_t sh_bases, const uint32_t g) {
    const float3 m = quant_position(q, g, q.records[g].x);
    const float vx = m.x - cam_position[0];
    const float vy = m.y - cam_position[1];
    const float vz = m.z - cam_position[2];
    const float inv_len = rsqrtf(vx * vx + vy * vy + vz * vz);
    float c[48];
    const uint32_t nc = sh_bases * 3;
    const __half* src = q.sh + static_cast<size_t>(g) * nc;
    for (uint32_t i = 0; i < nc; ++i) c[i] = __half2float(src[i]);
    return eval_sh(c, vx * inv_len, vy * inv_len, vz * inv_len, sh_bases);
}

// View-dependent colour of Gaussian g seen from the camera (resolve.cu:71-76).
__device__ __forceinline__ float3 winner_color(const ResolveParams& a, const uint32_t g) {
    if (a.quant.records != nullptr) return quantized_color(a.quant, a.cam_position, a.sh_bases, g);
    const float vx = a.means[3 * g + 0] - a.cam_position[0];
    const float vy = a.means[3 * g + 1] - a.cam_position[1];
    const float vz = a.means[3 * g + 2] - a.cam_position[2];
    const float inv_len = rsqrtf(vx * vx + vy * vy + vz * vz);
    const float x = vx * inv_len, y = vy * inv_len, z = vz * inv_len;
    if (a.sh_vec4) {
        // 48 coefficients as twelve 16-byte loads
        float c[48];
        const float4* src = reinterpret_cast<const float4*>(a.sh + static_cast<size_t>(g) * 48);
#pragma unroll
        for (int i = 0; i < 12; ++i) {
            const float4 v = __ldg(src + i);
            c[4 * i + 0] = v.x;
            c[4 * i + 1] = v.y;
            c[4 * i + 2] = v.z;
            c[4 * i + 3] = v.w;
        }
        return eval_sh(c, x, y, z, 16);
    }
    return eval_sh(a.sh + static_cast<size_t>(g) * a.sh_bases * 3, x, y, z, a.sh_bases);
}

// (rgb, depth) sample of a packed framebuffer entry, depth 0 = background (resolve.cu:65-78).
// Neighbouring pixels mostly share their winner: one lane per distinct winner of the warp
// evaluates the colour and shares it. Every lane of the warp must call this.
__device__ __forceinline__ float4 warp_sample(const ResolveParams& a, const unsigned long long data,
                                              const uint32_t lane) {
    const uint32_t depth_key = static_cast<uint32_t>(data >> 32);
    const bool has_sample = depth_key != 0xffffffffu;
    const uint32_t g = static_cast<uint32_t>(data);
    const uint32_t peers = __match_any_sync(0xffffffffu, has_sample ? g : 0xffffffffu);
    const uint32_t leader = __ffs(peers) - 1;
    float3 color = make_float3(0.0f, 0.0f, 0.0f);
    if (has_sample && lane == leader) color = winner_color(a, g);
    color.x = __shfl_sync(0xffffffffu, color.x, leader);
    color.y = __shfl_sync(0xffffffffu, color.y, leader);
    color.z = __shfl_sync(0xffffffffu, color.z, leader);
    return has_sample ? make_float4(color.x, color.y, color.z, __uint_as_float(depth_key))
                      : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
}

// Winner colour and depth of every framebuffer subpixel, the spatial-reuse weights towards its four
// neighbours and the k-buffer update (resolve.cu:27-144). A k-buffer entry's occlusion factors are
// loaded only when they are used: the entry occludes this sample, or the insertion of a new
// primitive shifts it. The pass is bound by the k-buffer traffic.
__global__ void __launch_bounds__(kBlock) reuse_sample_kernel(const ResolveParams a) {
    const uint32_t idx = blockIdx.x * kBlock + threadIdx.x;
    const bool active = idx < a.n_fb;
    const uint32_t pixel = active ? idx : a.n_fb - 1;

    const unsigned long long data = a.framebuffer[pixel];
    const uint32_t depth_key = static_cast<uint32_t>(data >> 32);
    const bool has_sample = depth_key != 0xffffffffu;
    const uint32_t g = has_sample ? static_cast<uint32_t>(data) : 0u;
    const float4 sample = warp_sample(a, data, threadIdx.x & 31u);
    if (active) a.samples[pixel] = sample;

    // alpha of this subpixel's winner at the subpixel and at its four neighbours needs its 2-D conic again
    bool projected = active && has_sample;
    Projected p;
    // lanes without a winner project Gaussian 0 alongside the others (the call is warp-collective);
    // a warp without any winner skips it, so an empty scene reads no Gaussian at all
    if (__any_sync(0xffffffffu, projected))
        project_gaussian(projected, g, a.means, a.scales, a.rotations, a.opacities, a.w2c, a.cam, p, nullptr, a.quant);
    if (!active) return;

    // per-neighbour weight = neighbour alpha over own alpha; a subpixel without a winner behaves as an
    // opaque surface at infinite depth
    float alpha = 1.0f;
    float4 na = make_float4(1.0f, 1.0f, 1.0f, 1.0f);
    float sample_depth = __uint_as_float(0x7f800000u);
    if (projected) {
        const float dx = static_cast<float>(pixel % a.cam.width_int) - (p.mean2d.x - 0.5f);
        const float dy = static_cast<float>(pixel / a.cam.width_int) - (p.mean2d.y - 0.5f);
        const float3 ce = conic_for_exp2(p.conic);
        auto eval = [&](const float ex, const float ey) {
            const float fa = fragment_alpha(ce, p.opacity, ex, ey);
            return fa < kMinAlpha ? 0.0f : fa;
        };
        alpha = fmaxf(eval(dx, dy), kMinAlpha);
        na = make_float4(eval(dx - 1.0f, dy), eval(dx + 1.0f, dy), eval(dx, dy - 1.0f), eval(dx, dy + 1.0f));
        sample_depth = sample.w;
    }
    float4 weights = has_sample && !projected
                         ? make_float4(0.0f, 0.0f, 0.0f, 0.0f)
                         : make_float4(na.x / alpha, na.y / alpha, na.z / alpha, na.w / alpha);

    // the k-buffer's primitives first: whether this winner is new decides which occlusions are read
    uint2 prims[kKBufferSize];
    bool unique = projected;
#pragma unroll
    for (uint32_t k = 0; k < kKBufferSize; ++k) {
        prims[k] = a.k_prims[static_cast<size_t>(k) * a.n_fb + pixel];
        if (prims[k].x == g) unique = false;
    }
    float4 occl[kKBufferSize];
#pragma unroll
    for (uint32_t k = 0; k < kKBufferSize; ++k) {
        // an unused slot's depth bits are a NaN, so the depth test below is false for it
        const bool occludes = __uint_as_float(prims[k].y) < sample_depth;
        occl[k] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        if (occludes || (unique && k + 1u < kKBufferSize)) occl[k] = a.k_occl[static_cast<size_t>(k) * a.n_fb + pixel];
        if (occludes) {
            weights.x *= occl[k].x;
            weights.y *= occl[k].y;
            weights.z *= occl[k].z;
            weights.w *= occl[k].w;
        }
    }
    // a winner not yet in the k-buffer shifts the entries down one slot (the last is lost) and takes slot 0
    if (unique) {
#pragma unroll
        for (uint32_t k = kKBufferSize - 1; k > 0; --k) {
            const size_t e = static_cast<size_t>(k) * a.n_fb + pixel;
            a.k_prims[e] = prims[k - 1];
            a.k_occl[e] = occl[k - 1];
        }
        a.k_prims[pixel] = make_uint2(g, depth_key);
        const float denom = 1.0f - fminf(alpha, kMaxAlpha);
        a.k_occl[pixel] = make_float4((1.0f - fminf(na.x, kMaxAlpha)) / denom, (1.0f - fminf(na.y, kMaxAlpha)) / denom,
                                      (1.0f - fminf(na.z, kMaxAlpha)) / denom, (1.0f - fminf(na.w, kMaxAlpha)) / denom);
    }
    a.reuse_weights[pixel] = weights;
}

// Winner colour and depth of every framebuffer subpixel (resolve.cu:65-78) for the resolve passes
// that read them from memory: Reproject without spatial reuse at supersampling factors whose tile
// does not fit in shared memory.
__global__ void __launch_bounds__(kBlock) plain_sample_kernel(const ResolveParams a) {
    const uint32_t idx = blockIdx.x * kBlock + threadIdx.x;
    const bool active = idx < a.n_fb;
    const uint32_t pixel = active ? idx : a.n_fb - 1;
    const float4 sample = warp_sample(a, a.framebuffer[pixel], threadIdx.x & 31u);
    if (active) a.samples[pixel] = sample;
}

// Advances a device-resident frame index once per call. The last pass of a call does it: every
// pass that reads the index (accumulate) has finished by then in stream order.
__device__ __forceinline__ void advance_frame(const ResolveParams& a) {
    if (a.frame_counter != nullptr && blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.x == 0) *a.frame_counter += 1u;
}

__device__ __forceinline__ float3 rgb_to_ycocg(const float3 c) {
    return make_float3(0.25f * c.x + 0.5f * c.y + 0.25f * c.z, 0.5f * c.x - 0.5f * c.z,
                       -0.25f * c.x + 0.5f * c.y - 0.25f * c.z);
}

__device__ __forceinline__ float4 catmull_rom_weights(const float t) {
    const float t2 = t * t;
    return make_float4(t * (-0.5f + t * (1.0f - 0.5f * t)), 1.0f + t2 * (-2.5f + 1.5f * t),
                       t * (0.5f + t * (2.0f - 1.5f * t)), t2 * (-0.5f + 0.5f * t));
}

// ---- tiled resolve of spatial reuse and Reproject ----

constexpr uint32_t kTileW = 32;  // image pixels per tile, one thread each
constexpr uint32_t kTileH = kBlock / kTileW;
constexpr uint32_t kRingW = kTileW + 2;  // the tile's pixels and a ring of one pixel (moment windows)
constexpr uint32_t kRingH = kTileH + 2;
constexpr uint32_t kHistFloats = 5;            // staged history texel: rgb, depth, alpha
constexpr size_t kMinHistBytes = 24u << 10;    // at least 1228 staged history texels per tile
constexpr size_t kMaxTileBytes = 200u << 10;   // larger tiles (supersampling >= 5) read global memory

// Shared-memory layout of one tile: the samples (and weights) of its subpixels with a halo of
// `halo` subpixels, the box-filtered YCoCg colours of its pixels and their one-pixel ring, and the
// staged history texels, which reuse the samples' space once the box filter and the colours are done.
struct TileLayout {
    uint32_t halo, sw, sh;  // staged subpixel rectangle: sw x sh, from (tile origin - halo)
    uint32_t hist_cap;      // staged history texels
    uint32_t samples, weights, hist, ycc, bytes;
};

TileLayout tile_layout(const uint32_t ss, const bool reuse, const bool reproject) {
    TileLayout L{};
    L.halo = reproject ? ss : (reuse ? 1u : 0u);
    L.sw = kTileW * ss + 2u * L.halo;
    L.sh = kTileH * ss + 2u * L.halo;
    const size_t n = static_cast<size_t>(L.sw) * L.sh;
    size_t off = 0;
    L.samples = 0;
    off += n * sizeof(float4);
    L.weights = static_cast<uint32_t>(off);
    if (reuse) off += n * sizeof(float4);
    L.hist = 0;
    if (reproject) {
        const size_t region = off > kMinHistBytes ? off : kMinHistBytes;
        L.hist_cap = static_cast<uint32_t>(region / (kHistFloats * sizeof(float)));
        off = region;
        L.ycc = static_cast<uint32_t>(off);
        off += kRingW * kRingH * sizeof(float3);
    }
    L.bytes = static_cast<uint32_t>(off);
    return L;
}

// One block per kTileW x kTileH image pixels (resolve.cu:164-349). kReuse: the samples and weights
// of reuse_sample_kernel with the neighbour resampling; kFused: the winners' colours are evaluated
// here from the framebuffer; kReproject: the temporal mode is Reproject (otherwise Reset or
// Static); kStaged: the tile's subpixels, colours and history come from shared memory (otherwise
// every read goes to global memory, for tiles too large to stage).
template <bool kReuse, bool kFused, bool kReproject, bool kStaged>
__global__ void __launch_bounds__(kBlock) tile_resolve_kernel(const ResolveParams a, const TileLayout L) {
    extern __shared__ __align__(16) unsigned char smem[];
    float4* s_samples = reinterpret_cast<float4*>(smem + L.samples);
    float4* s_weights = reinterpret_cast<float4*>(smem + L.weights);
    float* s_hist = reinterpret_cast<float*>(smem + L.hist);
    float3* s_ycc = reinterpret_cast<float3*>(smem + L.ycc);
    __shared__ uint32_t s_box[4];  // staged history rectangle: x0, x1, y0, y1 (inclusive)

    advance_frame(a);
    const uint32_t ss = a.ss;
    const uint32_t fbw = a.width * ss;
    const uint32_t fbh = a.height * ss;
    const float norm = 1.0f / static_cast<float>(ss * ss);
    const uint32_t tx0 = blockIdx.x * kTileW;
    const uint32_t ty0 = blockIdx.y * kTileH;
    const int ox = static_cast<int>(tx0 * ss) - static_cast<int>(L.halo);  // framebuffer position of staged (0, 0)
    const int oy = static_cast<int>(ty0 * ss) - static_cast<int>(L.halo);
    const uint32_t lane = threadIdx.x & 31u;

    if constexpr (kStaged) {
        if (kReproject && threadIdx.x == 0) {  // ordered before the atomics by the barrier below
            s_box[0] = s_box[2] = 0xffffffffu;
            s_box[1] = s_box[3] = 0u;
        }
        // stage the subpixels (uniform rounds: every lane of a warp takes part in warp_sample)
        const uint32_t n = L.sw * L.sh;
        for (uint32_t base = 0; base < n; base += kBlock) {
            const uint32_t i = base + threadIdx.x;
            const int fx = ox + static_cast<int>(i % L.sw);
            const int fy = oy + static_cast<int>(i / L.sw);
            const bool in = i < n && fx >= 0 && fy >= 0 && fx < static_cast<int>(fbw) && fy < static_cast<int>(fbh);
            const uint32_t fi = in ? static_cast<uint32_t>(fy) * fbw + static_cast<uint32_t>(fx) : 0u;
            float4 v;
            if constexpr (kFused) {
                v = warp_sample(a, in ? a.framebuffer[fi] : kEmptyFragment, lane);
                // the tile's own subpixels are written for inspection (each by exactly one tile)
                const bool own = in && fx >= static_cast<int>(tx0 * ss) && fx < static_cast<int>((tx0 + kTileW) * ss) &&
                                 fy >= static_cast<int>(ty0 * ss) && fy < static_cast<int>((ty0 + kTileH) * ss);
                if (own) a.samples[fi] = v;
            } else {
                v = in ? a.samples[fi] : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            }
            if (i < n) {
                s_samples[i] = v;
                if constexpr (kReuse) s_weights[i] = in ? a.reuse_weights[fi] : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            }
        }
        __syncthreads();
    }
    // subpixel (fx, fy) of the framebuffer: staged or from memory
    auto sample_at = [&](const uint32_t fx, const uint32_t fy) -> float4 {
        if constexpr (kStaged)
            return s_samples[(static_cast<int>(fy) - oy) * static_cast<int>(L.sw) + (static_cast<int>(fx) - ox)];
        return a.samples[fy * fbw + fx];
    };
    auto weight_at = [&](const uint32_t fx, const uint32_t fy) -> float4 {
        if constexpr (kStaged)
            return s_weights[(static_cast<int>(fy) - oy) * static_cast<int>(L.sw) + (static_cast<int>(fx) - ox)];
        return a.reuse_weights[fy * fbw + fx];
    };

    const uint32_t x = tx0 + threadIdx.x % kTileW;
    const uint32_t y = ty0 + threadIdx.x / kTileW;
    const bool active = x < a.width && y < a.height;
    const uint32_t px = min(x, a.width - 1u);  // inactive threads of an edge tile compute a clamped pixel
    const uint32_t py = min(y, a.height - 1u);
    const uint32_t pixel = py * a.width + px;

    // box filter over the ss x ss subpixels, each resampled from its neighbours with spatial reuse
    float3 cs = make_float3(0.0f, 0.0f, 0.0f);
    float ds = 0.0f, as = 0.0f, ws = 0.0f, depth_out = 0.0f;
    uint32_t valid = 0;
    for (uint32_t sy = 0; sy < ss; ++sy) {
        for (uint32_t sx = 0; sx < ss; ++sx) {
            const uint32_t fx = px * ss + sx;
            const uint32_t fy = py * ss + sy;
            const float4 s = sample_at(fx, fy);
            if (s.w > 0.0f) {
                depth_out += s.w;
                valid++;
            }
            float3 csum = make_float3(s.x, s.y, s.z);
            float dsum = s.w;
            float asum = s.w > 0.0f ? 1.0f : 0.0f;
            float wsum = 1.0f;
            if constexpr (kReuse) {
                // neighbours stored their weights towards this subpixel (resolve.cu:218-230)
                auto add = [&](const float4 n, const float w) {
                    csum.x += w * n.x;
                    csum.y += w * n.y;
                    csum.z += w * n.z;
                    dsum += w * n.w;
                    asum += n.w > 0.0f ? w : 0.0f;
                    wsum += w;
                };
                if (fx > 0) add(sample_at(fx - 1, fy), weight_at(fx - 1, fy).y);
                if (fx < fbw - 1) add(sample_at(fx + 1, fy), weight_at(fx + 1, fy).x);
                if (fy > 0) add(sample_at(fx, fy - 1), weight_at(fx, fy - 1).w);
                if (fy < fbh - 1) add(sample_at(fx, fy + 1), weight_at(fx, fy + 1).z);
            }
            const float rcp = 1.0f / wsum;
            cs.x += csum.x * rcp;
            cs.y += csum.y * rcp;
            cs.z += csum.z * rcp;
            ds += dsum * rcp;
            as += asum * rcp;
            ws += wsum;
        }
    }
    cs.x *= norm;
    cs.y *= norm;
    cs.z *= norm;
    ds *= norm;
    as *= norm;
    ws *= norm;

    float3 color = cs;
    float depth = ds, alpha = as, weight_mass = ws;
    if constexpr (!kReproject) {
        if (a.temporal_mode == 1 && active) {
            // Static: merge with the history weighted by the accumulated weight mass (resolve.cu:250-258)
            const float hm = a.hist_weight_mass[pixel];
            weight_mass = hm + ws;
            const float hf = hm / weight_mass;
            color.x = cs.x + hf * (a.hist_image[3 * pixel + 0] - cs.x);
            color.y = cs.y + hf * (a.hist_image[3 * pixel + 1] - cs.y);
            color.z = cs.z + hf * (a.hist_image[3 * pixel + 2] - cs.z);
            depth = ds + hf * (a.hist_depth[pixel] - ds);
            alpha = as + hf * (a.hist_alpha[pixel] - as);
        }
    } else {
        // box-filtered YCoCg colour of pixel (qx, qy) (resolve.cu:314-318)
        auto box_ycc = [&](const uint32_t qx, const uint32_t qy) {
            float3 nc = make_float3(0.0f, 0.0f, 0.0f);
            for (uint32_t sy = 0; sy < ss; ++sy) {
                for (uint32_t sx = 0; sx < ss; ++sx) {
                    const float4 s = sample_at(qx * ss + sx, qy * ss + sy);
                    nc.x += s.x;
                    nc.y += s.y;
                    nc.z += s.z;
                }
            }
            return rgb_to_ycocg(make_float3(nc.x * norm, nc.y * norm, nc.z * norm));
        };
        if constexpr (kStaged) {
            // once per pixel of the tile and its ring, clamped to the image like the moment windows
            for (uint32_t j = threadIdx.x; j < kRingW * kRingH; j += kBlock) {
                const int qx = min(max(static_cast<int>(tx0) - 1 + static_cast<int>(j % kRingW), 0),
                                   static_cast<int>(a.width) - 1);
                const int qy = min(max(static_cast<int>(ty0) - 1 + static_cast<int>(j / kRingW), 0),
                                   static_cast<int>(a.height) - 1);
                s_ycc[j] = box_ycc(static_cast<uint32_t>(qx), static_cast<uint32_t>(qy));
            }
        }

        // where this pixel's sampled surface was in the previous view: mean winner depth of the valid
        // subpixels, the far plane where none is valid (resolve.cu:261-283)
        const float z = valid > 0 ? depth_out / static_cast<float>(valid) : a.far_plane;
        const float fpx = static_cast<float>(px) + 0.5f;
        const float fpy = static_cast<float>(py) + 0.5f;
        const float vx = (fpx - a.center_x) / a.focal_x * z;
        const float vy = (fpy - a.center_y) / a.focal_y * z;
        const float vz = z;
        const float4 m1 = a.v2pv[0], m2 = a.v2pv[1], m3 = a.v2pv[2];
        const float pz = m3.x * vx + m3.y * vy + m3.z * vz + m3.w;
        bool use_history = active && pz > 0.0f;
        float ppx = 0.0f, ppy = 0.0f;
        if (use_history) {
            ppx = a.focal_x * (m1.x * vx + m1.y * vy + m1.z * vz + m1.w) / pz + a.center_x;
            ppy = a.focal_y * (m2.x * vx + m2.y * vy + m2.z * vz + m2.w) / pz + a.center_y;
            // points within the margin of the image edge take no history, so the 4 x 4 taps below never
            // leave the image
            use_history = ppx >= kBorderMargin && ppx <= static_cast<float>(a.width) - kBorderMargin &&
                          ppy >= kBorderMargin && ppy <= static_cast<float>(a.height) - kBorderMargin;
        }
        const float tx = ppx - 0.5f, ty = ppy - 0.5f;
        const float tbx = floorf(tx), tby = floorf(ty);
        const uint32_t hx = use_history ? static_cast<uint32_t>(tbx) - 1 : 0u;
        const uint32_t hy = use_history ? static_cast<uint32_t>(tby) - 1 : 0u;

        // stage the history texels under the tile's taps when their rectangle fits
        bool staged_history = false;
        uint32_t bx0 = 0, by0 = 0, bw = 0;
        if constexpr (kStaged) {
            const uint32_t any = __ballot_sync(0xffffffffu, use_history);
            if (any != 0u) {
                const uint32_t mnx = __reduce_min_sync(0xffffffffu, use_history ? hx : 0xffffffffu);
                const uint32_t mxx = __reduce_max_sync(0xffffffffu, use_history ? hx + 3u : 0u);
                const uint32_t mny = __reduce_min_sync(0xffffffffu, use_history ? hy : 0xffffffffu);
                const uint32_t mxy = __reduce_max_sync(0xffffffffu, use_history ? hy + 3u : 0u);
                if (lane == 0) {
                    atomicMin(&s_box[0], mnx);
                    atomicMax(&s_box[1], mxx);
                    atomicMin(&s_box[2], mny);
                    atomicMax(&s_box[3], mxy);
                }
            }
            __syncthreads();  // also: every read of the staged subpixels is done
            bx0 = s_box[0];
            by0 = s_box[2];
            const bool some = bx0 <= s_box[1];
            bw = some ? s_box[1] - bx0 + 1u : 0u;
            const uint32_t bh = some ? s_box[3] - by0 + 1u : 0u;
            staged_history = some && static_cast<size_t>(bw) * bh <= L.hist_cap;
            if (staged_history) {
                const uint32_t cap = L.hist_cap;
                for (uint32_t k = threadIdx.x; k < bw * bh; k += kBlock) {
                    const uint32_t hi = (by0 + k / bw) * a.width + bx0 + k % bw;
                    s_hist[k] = a.hist_image[3 * hi + 0];
                    s_hist[cap + k] = a.hist_image[3 * hi + 1];
                    s_hist[2 * cap + k] = a.hist_image[3 * hi + 2];
                    s_hist[3 * cap + k] = a.hist_depth[hi];
                    s_hist[4 * cap + k] = a.hist_alpha[hi];
                }
            }
            __syncthreads();
        }

        if (use_history) {
            // bicubic (Catmull-Rom) filter of the previous outputs around that point, unclamped
            // (resolve.cu:285-305)
            const float4 wx4 = catmull_rom_weights(tx - tbx);
            const float4 wy4 = catmull_rom_weights(ty - tby);
            const float wx[4] = {wx4.x, wx4.y, wx4.z, wx4.w};
            const float wy[4] = {wy4.x, wy4.y, wy4.z, wy4.w};
            float3 ch = make_float3(0.0f, 0.0f, 0.0f);
            float dh = 0.0f, ah = 0.0f;
#pragma unroll
            for (uint32_t j = 0; j < 4; ++j) {
#pragma unroll
                for (uint32_t i = 0; i < 4; ++i) {
                    const float w = wx[i] * wy[j];
                    // the texel from shared memory or from the history arrays, then one accumulation for
                    // both (the same operations either way)
                    float hr, hg, hb, hd, ha;
                    if (staged_history) {
                        const uint32_t k = (hy + j - by0) * bw + (hx + i - bx0);
                        const uint32_t cap = L.hist_cap;
                        hr = s_hist[k];
                        hg = s_hist[cap + k];
                        hb = s_hist[2 * cap + k];
                        hd = s_hist[3 * cap + k];
                        ha = s_hist[4 * cap + k];
                    } else {
                        const uint32_t hi = (hy + j) * a.width + hx + i;
                        hr = a.hist_image[3 * hi + 0];
                        hg = a.hist_image[3 * hi + 1];
                        hb = a.hist_image[3 * hi + 2];
                        hd = a.hist_depth[hi];
                        ha = a.hist_alpha[hi];
                    }
                    ch.x += w * hr;
                    ch.y += w * hg;
                    ch.z += w * hb;
                    dh += w * hd;
                    ah += w * ha;
                }
            }

            // mean and mean square, in YCoCg, of this sample's box-filtered colours over the pixel and its 8
            // neighbours (clamped at the edges) (resolve.cu:307-326)
            float3 mean = make_float3(0.0f, 0.0f, 0.0f);
            float3 mean_sq = make_float3(0.0f, 0.0f, 0.0f);
            for (int wy = -1; wy <= 1; ++wy) {
                for (int wx = -1; wx <= 1; ++wx) {
                    float3 ycc;
                    if constexpr (kStaged) {
                        ycc = s_ycc[(static_cast<int>(py - ty0) + 1 + wy) * static_cast<int>(kRingW) +
                                    static_cast<int>(px - tx0) + 1 + wx];
                    } else {
                        const int qx = max(0, min(static_cast<int>(px) + wx, static_cast<int>(a.width) - 1));
                        const int qy = max(0, min(static_cast<int>(py) + wy, static_cast<int>(a.height) - 1));
                        ycc = box_ycc(static_cast<uint32_t>(qx), static_cast<uint32_t>(qy));
                    }
                    mean.x += ycc.x;
                    mean.y += ycc.y;
                    mean.z += ycc.z;
                    mean_sq.x += ycc.x * ycc.x;
                    mean_sq.y += ycc.y * ycc.y;
                    mean_sq.z += ycc.z * ycc.z;
                }
            }
            mean.x /= 9.0f;
            mean.y /= 9.0f;
            mean.z /= 9.0f;
            mean_sq.x /= 9.0f;
            mean_sq.y /= 9.0f;
            mean_sq.z /= 9.0f;
            const float sdx = sqrtf(fmaxf(mean_sq.x - mean.x * mean.x, 0.0f));
            const float sdy = sqrtf(fmaxf(mean_sq.y - mean.y * mean.y, 0.0f));
            const float sdz = sqrtf(fmaxf(mean_sq.z - mean.z * mean.z, 0.0f));

            // how far the history colour lies outside a box of gamma standard deviations around the mean
            // (gamma falls from the static to the moving value as the pixel moves faster), as a
            // discount of the history weight (resolve.cu:328-339)
            const float dvx = fpx - ppx, dvy = fpy - ppy;
            const float velocity = sqrtf(dvx * dvx + dvy * dvy);
            const float gamma = kGammaStatic + fminf(velocity / kVelocityThreshold, 1.0f) * (kGammaMotion - kGammaStatic);
            const float ex = fmaxf(gamma * sdx, kMinExtentLuma);
            const float ey = fmaxf(gamma * sdy, kMinExtentChroma);
            const float ez = fmaxf(gamma * sdz, kMinExtentChroma);
            const float3 hyc = rgb_to_ycocg(ch);
            const float qx = fabsf(hyc.x - mean.x) / ex;
            const float qy = fabsf(hyc.y - mean.y) / ey;
            const float qz = fabsf(hyc.z - mean.z) / ez;
            const float distance = fmaxf(qx, fmaxf(qy, qz));
            const float discount = distance > 1.0f ? kHistoryWeight / distance : kHistoryWeight;
            color.x = cs.x + discount * (ch.x - cs.x);
            color.y = cs.y + discount * (ch.y - cs.y);
            color.z = cs.z + discount * (ch.z - cs.z);
            depth = ds + discount * (dh - ds);
            alpha = as + discount * (ah - as);
            // weight mass of a sum that kept this discount forever: Static merges start from it when the
            // view stops moving
            weight_mass = ws / (1.0f - discount);
        }
    }
    if (!active) return;
    a.image[3 * pixel + 0] = color.x;
    a.image[3 * pixel + 1] = color.y;
    a.image[3 * pixel + 2] = color.z;
    a.depth[pixel] = depth;
    a.alpha[pixel] = alpha;
    a.weight_mass[pixel] = weight_mass;
}

// Sample and resolve in one pass when no neighbour is read (no spatial reuse, Reset or Static):
// one thread per image pixel evaluates its ss x ss subpixels' winners (warp-deduplicated),
// box-filters them and merges the history with resolve.cu:191-258's arithmetic. The samples are
// still written for inspection. The pass waits on its dependent gathers (key, then the winner's SH),
// so it is held to 40 registers for 6 resident blocks per SM.
__global__ void __launch_bounds__(kBlock, 6) sample_resolve_fused_kernel(const ResolveParams a) {
    advance_frame(a);
    const uint32_t idx = blockIdx.x * kBlock + threadIdx.x;
    const bool active = idx < a.n_pixels;
    const uint32_t pixel = active ? idx : a.n_pixels - 1;
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t ss = a.ss;
    const uint32_t bx = (pixel % a.width) * ss;
    const uint32_t by = (pixel / a.width) * ss;
    const uint32_t fbw = a.width * ss;
    const float norm = 1.0f / static_cast<float>(ss * ss);

    float3 cs = make_float3(0.0f, 0.0f, 0.0f);
    float ds = 0.0f, as = 0.0f, ws = 0.0f;
    for (uint32_t oy = 0; oy < ss; ++oy) {
        for (uint32_t ox = 0; ox < ss; ++ox) {
            const uint32_t fi = (by + oy) * fbw + bx + ox;
            const float4 s = warp_sample(a, a.framebuffer[fi], lane);
            if (active) a.samples[fi] = s;
            const float3 csum = make_float3(s.x, s.y, s.z);
            const float dsum = s.w;
            const float asum = s.w > 0.0f ? 1.0f : 0.0f;
            const float wsum = 1.0f;
            const float rcp = 1.0f / wsum;
            cs.x += csum.x * rcp;
            cs.y += csum.y * rcp;
            cs.z += csum.z * rcp;
            ds += dsum * rcp;
            as += asum * rcp;
            ws += wsum;
        }
    }
    if (!active) return;
    cs.x *= norm;
    cs.y *= norm;
    cs.z *= norm;
    ds *= norm;
    as *= norm;
    ws *= norm;

    float3 color = cs;
    float depth = ds, alpha = as, weight_mass = ws;
    if (a.temporal_mode == 1) {
        const float hm = a.hist_weight_mass[pixel];
        weight_mass = hm + ws;
        const float hf = hm / weight_mass;
        color.x = cs.x + hf * (a.hist_image[3 * pixel + 0] - cs.x);
        color.y = cs.y + hf * (a.hist_image[3 * pixel + 1] - cs.y);
        color.z = cs.z + hf * (a.hist_image[3 * pixel + 2] - cs.z);
        depth = ds + hf * (a.hist_depth[pixel] - ds);
        alpha = as + hf * (a.hist_alpha[pixel] - as);
    }
    a.image[3 * pixel + 0] = color.x;
    a.image[3 * pixel + 1] = color.y;
    a.image[3 * pixel + 2] = color.z;
    a.depth[pixel] = depth;
    a.alpha[pixel] = alpha;
    a.weight_mass[pixel] = weight_mass;
}

// Several samples of one call merged in order (the first in the call's temporal mode, Reset or
// Static, the rest Static): per pixel the same box filter and the same merge as
// sample_resolve_fused_kernel once per sample, the history carried in registers between samples, so
// the outputs equal those of one call per sample bit for bit.
__global__ void __launch_bounds__(kBlock) samples_resolve_kernel(const ResolveParams a) {
    if (a.frame_counter != nullptr && blockIdx.x == 0 && threadIdx.x == 0) *a.frame_counter += a.n_samples;
    const uint32_t idx = blockIdx.x * kBlock + threadIdx.x;
    const bool active = idx < a.n_pixels;
    const uint32_t pixel = active ? idx : a.n_pixels - 1;
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t ss = a.ss;
    const uint32_t bx = (pixel % a.width) * ss;
    const uint32_t by = (pixel / a.width) * ss;
    const uint32_t fbw = a.width * ss;
    const float norm = 1.0f / static_cast<float>(ss * ss);

    float3 color = make_float3(0.0f, 0.0f, 0.0f);
    float depth = 0.0f, alpha = 0.0f, weight_mass = 0.0f;
    if (a.temporal_mode == 1 && active) {
        color = make_float3(a.hist_image[3 * pixel + 0], a.hist_image[3 * pixel + 1], a.hist_image[3 * pixel + 2]);
        depth = a.hist_depth[pixel];
        alpha = a.hist_alpha[pixel];
        weight_mass = a.hist_weight_mass[pixel];
    }
    for (uint32_t sm = 0; sm < a.n_samples; ++sm) {
        const unsigned long long* fb = a.framebuffer + sm * a.fb_stride;
        float3 cs = make_float3(0.0f, 0.0f, 0.0f);
        float ds = 0.0f, as = 0.0f, ws = 0.0f;
        for (uint32_t oy = 0; oy < ss; ++oy) {
            for (uint32_t ox = 0; ox < ss; ++ox) {
                const uint32_t fi = (by + oy) * fbw + bx + ox;
                const float4 smp = warp_sample(a, fb[fi], lane);
                const float wsum = 1.0f;
                const float rcp = 1.0f / wsum;
                cs.x += smp.x * rcp;
                cs.y += smp.y * rcp;
                cs.z += smp.z * rcp;
                ds += smp.w * rcp;
                as += (smp.w > 0.0f ? 1.0f : 0.0f) * rcp;
                ws += wsum;
            }
        }
        cs.x *= norm;
        cs.y *= norm;
        cs.z *= norm;
        ds *= norm;
        as *= norm;
        ws *= norm;
        if (sm == 0 && a.temporal_mode == 0) {
            color = cs;
            depth = ds;
            alpha = as;
            weight_mass = ws;
        } else {
            const float hm = weight_mass;
            weight_mass = hm + ws;
            const float hf = hm / weight_mass;
            color.x = cs.x + hf * (color.x - cs.x);
            color.y = cs.y + hf * (color.y - cs.y);
            color.z = cs.z + hf * (color.z - cs.z);
            depth = ds + hf * (depth - ds);
            alpha = as + hf * (alpha - as);
        }
    }
    if (!active) return;
    a.image[3 * pixel + 0] = color.x;
    a.image[3 * pixel + 1] = color.y;
    a.image[3 * pixel + 2] = color.z;
    a.depth[pixel] = depth;
    a.alpha[pixel] = alpha;
    a.weight_mass[pixel] = weight_mass;
}

}  // namespace

namespace {

template <bool kReuse, bool kFused, bool kReproject, bool kStaged>
cudaError_t launch_tile(const ResolveParams& p, const TileLayout& L, cudaStream_t stream) {
    auto kernel = tile_resolve_kernel<kReuse, kFused, kReproject, kStaged>;
    const size_t bytes = kStaged ? L.bytes : 0u;
    if (bytes > (48u << 10)) {
        const cudaError_t err = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                     static_cast<int>(bytes));
        if (err != cudaSuccess) return err;
    }
    const dim3 grid((p.width + kTileW - 1) / kTileW, (p.height + kTileH - 1) / kTileH);
    kernel<<<grid, kBlock, bytes, stream>>>(p, L);
    return cudaGetLastError();
}

}  // namespace

cudaError_t launch_sample_resolve(const ResolveParams& p, cudaStream_t stream) {
    if (p.n_samples > 1) {
        samples_resolve_kernel<<<(p.n_pixels + kBlock - 1) / kBlock, kBlock, 0, stream>>>(p);
        return cudaGetLastError();
    }
    const bool reproject = p.temporal_mode == 2;
    if (!p.spatial_reuse && !reproject) {
        sample_resolve_fused_kernel<<<(p.n_pixels + kBlock - 1) / kBlock, kBlock, 0, stream>>>(p);
        return cudaGetLastError();
    }
    const TileLayout L = tile_layout(p.ss, p.spatial_reuse, reproject);
    const bool staged = L.bytes <= kMaxTileBytes;
    const unsigned grid_sample = (p.n_fb + kBlock - 1) / kBlock;
    if (p.spatial_reuse) {
        reuse_sample_kernel<<<grid_sample, kBlock, 0, stream>>>(p);
        const cudaError_t err = cudaGetLastError();
        if (err != cudaSuccess) return err;
        if (reproject) return staged ? launch_tile<true, false, true, true>(p, L, stream)
                                     : launch_tile<true, false, true, false>(p, L, stream);
        return staged ? launch_tile<true, false, false, true>(p, L, stream)
                      : launch_tile<true, false, false, false>(p, L, stream);
    }
    // Reproject without spatial reuse: the winners' colours evaluated by the resolve tiles themselves
    if (staged) return launch_tile<false, true, true, true>(p, L, stream);
    plain_sample_kernel<<<grid_sample, kBlock, 0, stream>>>(p);
    const cudaError_t err = cudaGetLastError();
    if (err != cudaSuccess) return err;
    return launch_tile<false, false, true, false>(p, L, stream);
}

}  // namespace sgs
