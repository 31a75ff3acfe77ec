// Sample and resolve passes: colour of each (sub)pixel's winner, optional spatial reuse with the
// k-buffer, then the supersampling box filter and the temporal (Reset / Static / Reproject) merge.
//
// Follows resolve.cu:27-349 of the reference expression for expression, so that the outputs match
// it bit for bit when the winners match.
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

// View-dependent colour of Gaussian g seen from the camera (resolve.cu:71-76).
__device__ __forceinline__ float3 winner_color(const ResolveParams& a, const uint32_t g) {
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

// Winner colour and depth per (sub)pixel; with spatial reuse also the resampling weights towards
// the four neighbours and the k-buffer update (resolve.cu:27-144).
template <bool kReuse>
__global__ void __launch_bounds__(kBlock) sample_kernel(const ResolveParams a) {
    const uint32_t idx = blockIdx.x * kBlock + threadIdx.x;
    const bool active = idx < a.n_fb;
    const uint32_t pixel = active ? idx : a.n_fb - 1;

    const unsigned long long data = a.framebuffer[pixel];
    const uint32_t depth_key = static_cast<uint32_t>(data >> 32);
    const bool has_sample = depth_key != 0xffffffffu;
    const uint32_t g = has_sample ? static_cast<uint32_t>(data) : 0u;
    const float4 sample = warp_sample(a, data, threadIdx.x & 31u);
    if (active) a.samples[pixel] = sample;
    if constexpr (!kReuse) return;

    // project the winner again to evaluate it at the neighbours
    bool projected = active && has_sample;
    Projected p;
    project_gaussian(projected, g, a.means, a.scales, a.rotations, a.opacities, a.w2c, a.cam, p);
    if (!active) return;

    // weights start with the change in alpha; background is opaque and farthest
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

    // change in occlusion from the k-buffer of recently sampled primitives
    bool unique = projected;
    uint2 prims[kKBufferSize];
    float4 occl[kKBufferSize];
#pragma unroll
    for (uint32_t k = 0; k < kKBufferSize; ++k) {
        const size_t e = static_cast<size_t>(k) * a.n_fb + pixel;
        prims[k] = a.k_prims[e];
        occl[k] = a.k_occl[e];
        if (prims[k].x == g) unique = false;
        // empty entries hold a NaN depth and never occlude
        if (__uint_as_float(prims[k].y) < sample_depth) {
            weights.x *= occl[k].x;
            weights.y *= occl[k].y;
            weights.z *= occl[k].z;
            weights.w *= occl[k].w;
        }
    }
    // insert a new primitive at the front, evicting the oldest entry
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

// Advances a device-resident frame index once per call. The last pass of a call does it: every
// pass that reads the index (accumulate) has finished by then in stream order.
__device__ __forceinline__ void advance_frame(const ResolveParams& a) {
    if (a.frame_counter != nullptr && blockIdx.x == 0 && threadIdx.x == 0) *a.frame_counter += 1u;
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

// Box filter over the ss x ss subpixels with optional self-normalised neighbour resampling,
// then the temporal merge (resolve.cu:164-349).
template <bool kReuse>
__global__ void __launch_bounds__(kBlock) resolve_kernel(const ResolveParams a) {
    advance_frame(a);
    const uint32_t pixel = blockIdx.x * kBlock + threadIdx.x;
    if (pixel >= a.n_pixels) return;
    const uint32_t ss = a.ss;
    const uint32_t bx = (pixel % a.width) * ss;
    const uint32_t by = (pixel / a.width) * ss;
    const uint32_t fbw = a.width * ss;
    const uint32_t fbh = a.height * ss;
    const float norm = 1.0f / static_cast<float>(ss * ss);

    float3 cs = make_float3(0.0f, 0.0f, 0.0f);
    float ds = 0.0f, as = 0.0f, ws = 0.0f, depth_out = 0.0f;
    uint32_t valid = 0;
    for (uint32_t oy = 0; oy < ss; ++oy) {
        for (uint32_t ox = 0; ox < ss; ++ox) {
            const uint32_t fx = bx + ox;
            const uint32_t fy = by + oy;
            const uint32_t fi = fy * fbw + fx;
            const float4 s = a.samples[fi];
            if (s.w > 0.0f) {
                depth_out += s.w;
                valid++;
            }
            float3 csum = make_float3(s.x, s.y, s.z);
            float dsum = s.w;
            float asum = s.w > 0.0f ? 1.0f : 0.0f;
            float wsum = 1.0f;
            if constexpr (kReuse) {
                auto add = [&](const uint32_t ni, const float w) {
                    const float4 n = a.samples[ni];
                    csum.x += w * n.x;
                    csum.y += w * n.y;
                    csum.z += w * n.z;
                    dsum += w * n.w;
                    asum += n.w > 0.0f ? w : 0.0f;
                    wsum += w;
                };
                if (fx > 0) add(fi - 1, a.reuse_weights[fi - 1].y);
                if (fx < fbw - 1) add(fi + 1, a.reuse_weights[fi + 1].x);
                if (fy > 0) add(fi - fbw, a.reuse_weights[fi - fbw].w);
                if (fy < fbh - 1) add(fi + fbw, a.reuse_weights[fi + fbw].z);
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
    if (a.temporal_mode == 1) {
        // weighted cumulative moving average
        const float hm = a.hist_weight_mass[pixel];
        weight_mass = hm + ws;
        const float hf = hm / weight_mass;
        color.x = cs.x + hf * (a.hist_image[3 * pixel + 0] - cs.x);
        color.y = cs.y + hf * (a.hist_image[3 * pixel + 1] - cs.y);
        color.z = cs.z + hf * (a.hist_image[3 * pixel + 2] - cs.z);
        depth = ds + hf * (a.hist_depth[pixel] - ds);
        alpha = as + hf * (a.hist_alpha[pixel] - as);
    } else if (a.temporal_mode == 2) {
        do {
            // reproject the sampled surface point, background at the far plane
            const uint32_t x = pixel % a.width;
            const uint32_t y = pixel / a.width;
            const float z = valid > 0 ? depth_out / static_cast<float>(valid) : a.far_plane;
            const float px = static_cast<float>(x) + 0.5f;
            const float py = static_cast<float>(y) + 0.5f;
            const float vx = (px - a.center_x) / a.focal_x * z;
            const float vy = (py - a.center_y) / a.focal_y * z;
            const float vz = z;
            const float4 m1 = a.v2pv[0], m2 = a.v2pv[1], m3 = a.v2pv[2];
            const float pz = m3.x * vx + m3.y * vy + m3.z * vz + m3.w;
            if (!(pz > 0.0f)) break;
            const float ppx = a.focal_x * (m1.x * vx + m1.y * vy + m1.z * vz + m1.w) / pz + a.center_x;
            const float ppy = a.focal_y * (m2.x * vx + m2.y * vy + m2.z * vz + m2.w) / pz + a.center_y;
            // no history near the border, keeps every Catmull-Rom tap inside
            const bool inside = ppx >= kBorderMargin && ppx <= static_cast<float>(a.width) - kBorderMargin &&
                                ppy >= kBorderMargin && ppy <= static_cast<float>(a.height) - kBorderMargin;
            if (!inside) break;

            const float tx = ppx - 0.5f, ty = ppy - 0.5f;
            const float tbx = floorf(tx), tby = floorf(ty);
            const float4 wx4 = catmull_rom_weights(tx - tbx);
            const float4 wy4 = catmull_rom_weights(ty - tby);
            const float wx[4] = {wx4.x, wx4.y, wx4.z, wx4.w};
            const float wy[4] = {wy4.x, wy4.y, wy4.z, wy4.w};
            const uint32_t hx = static_cast<uint32_t>(tbx) - 1;
            const uint32_t hy = static_cast<uint32_t>(tby) - 1;
            float3 ch = make_float3(0.0f, 0.0f, 0.0f);
            float dh = 0.0f, ah = 0.0f;
#pragma unroll
            for (uint32_t j = 0; j < 4; ++j) {
#pragma unroll
                for (uint32_t i = 0; i < 4; ++i) {
                    const uint32_t hi = (hy + j) * a.width + hx + i;
                    const float w = wx[i] * wy[j];
                    ch.x += w * a.hist_image[3 * hi + 0];
                    ch.y += w * a.hist_image[3 * hi + 1];
                    ch.z += w * a.hist_image[3 * hi + 2];
                    dh += w * a.hist_depth[hi];
                    ah += w * a.hist_alpha[hi];
                }
            }

            // YCoCg moments of the current samples in a 3x3 window
            float3 mean = make_float3(0.0f, 0.0f, 0.0f);
            float3 mean_sq = make_float3(0.0f, 0.0f, 0.0f);
            for (int oy = -1; oy <= 1; ++oy) {
                for (int ox = -1; ox <= 1; ++ox) {
                    const uint32_t nx = static_cast<uint32_t>(max(0, min(static_cast<int>(x) + ox, static_cast<int>(a.width) - 1)));
                    const uint32_t ny = static_cast<uint32_t>(max(0, min(static_cast<int>(y) + oy, static_cast<int>(a.height) - 1)));
                    float3 nc = make_float3(0.0f, 0.0f, 0.0f);
                    for (uint32_t sy = 0; sy < ss; ++sy) {
                        for (uint32_t sx = 0; sx < ss; ++sx) {
                            const float4 s = a.samples[(ny * ss + sy) * fbw + nx * ss + sx];
                            nc.x += s.x;
                            nc.y += s.y;
                            nc.z += s.z;
                        }
                    }
                    const float3 ycc = rgb_to_ycocg(make_float3(nc.x * norm, nc.y * norm, nc.z * norm));
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

            // soft history rejection with velocity-adaptive confidence half-extents
            const float dvx = px - ppx, dvy = py - ppy;
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
            // steady-state weight mass, used once the camera stops
            weight_mass = ws / (1.0f - discount);
        } while (false);
    }
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

cudaError_t launch_sample_resolve(const ResolveParams& p, cudaStream_t stream) {
    if (p.n_samples > 1) {
        samples_resolve_kernel<<<(p.n_pixels + kBlock - 1) / kBlock, kBlock, 0, stream>>>(p);
        return cudaGetLastError();
    }
    if (!p.spatial_reuse && p.temporal_mode != 2) {
        sample_resolve_fused_kernel<<<(p.n_pixels + kBlock - 1) / kBlock, kBlock, 0, stream>>>(p);
        return cudaGetLastError();
    }
    const unsigned grid_sample = (p.n_fb + kBlock - 1) / kBlock;
    const unsigned grid_resolve = (p.n_pixels + kBlock - 1) / kBlock;
    if (p.spatial_reuse) {
        sample_kernel<true><<<grid_sample, kBlock, 0, stream>>>(p);
        resolve_kernel<true><<<grid_resolve, kBlock, 0, stream>>>(p);
    } else {
        sample_kernel<false><<<grid_sample, kBlock, 0, stream>>>(p);
        resolve_kernel<false><<<grid_resolve, kBlock, 0, stream>>>(p);
    }
    return cudaGetLastError();
}

}  // namespace sgs
