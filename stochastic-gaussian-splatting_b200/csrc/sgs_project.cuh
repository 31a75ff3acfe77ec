// Per-Gaussian projection (EWA splatting) and degree <= 3 spherical-harmonics colour.
//
// Restates gs_utils.h:38-243 of the reference. Expressions keep the reference's association so
// that, compiled with -use_fast_math, depth, conic, opacity, power threshold and screen bounds
// match the reference bit for bit (the fragment keys and alpha tests depend on them).
#pragma once

#include <cstdint>
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include "sgs_common.cuh"

namespace sgs {

// Camera of one accumulate/sample pass, already scaled to (sub)pixels of the framebuffer.
struct PassCamera {
    float width, height;        // framebuffer size in (sub)pixels
    float focal_x, focal_y;
    float center_x, center_y;
    float near_plane, far_plane;
    float ss;                   // supersampling factor as float
    uint32_t width_int;         // framebuffer width as integer
    bool proper_aa;
};

// Everything the accumulation and reuse passes need about one projected Gaussian.
struct Projected {
    float depth;
    float opacity;
    float determinant;
    float power_threshold;
    float2 mean2d;
    float3 conic;
    float3 cov2d;
    float4 bounds;  // x_min, x_max, y_min, y_max in (sub)pixels
};

// Upper triangle of the 3-D covariance R diag(exp(2 s)) R^T of Gaussian g (gs_utils.h:82-110);
// clears `valid` for a degenerate quaternion. The projection and the preactivated layout both take
// it from here, so the two hold the same bits.
struct Cov3d {
    float c11, c12, c13, c22, c23, c33;
};

__device__ __forceinline__ Cov3d cov3d_from(const float s0, const float s1, const float s2, const float4 q,
                                            bool& valid) {
    const float vx = expf(2.0f * s0);
    const float vy = expf(2.0f * s1);
    const float vz = expf(2.0f * s2);
    const float r = q.x, i = q.y, j = q.z, k = q.w;
    const float ii = i * i, jj = j * j, kk = k * k;
    const float ij = i * j, ik = i * k, jk = j * k;
    const float ri = r * i, rj = r * j, rk = r * k;
    const float norm_sq = r * r + ii + jj + kk;
    if (norm_sq < 1e-8f) valid = false;
    const float n_rcp = 1.0f / norm_sq;
    const float R11 = 1.0f - 2.0f * (jj + kk) * n_rcp, R12 = 2.0f * (ij - rk) * n_rcp, R13 = 2.0f * (ik + rj) * n_rcp;
    const float R21 = 2.0f * (ij + rk) * n_rcp, R22 = 1.0f - 2.0f * (ii + kk) * n_rcp, R23 = 2.0f * (jk - ri) * n_rcp;
    const float R31 = 2.0f * (ik - rj) * n_rcp, R32 = 2.0f * (jk + ri) * n_rcp, R33 = 1.0f - 2.0f * (ii + jj) * n_rcp;
    const float S11 = R11 * vx, S12 = R12 * vy, S13 = R13 * vz;
    const float S21 = R21 * vx, S22 = R22 * vy, S23 = R23 * vz;
    const float S31 = R31 * vx, S32 = R32 * vy, S33 = R33 * vz;
    Cov3d c;
    c.c11 = S11 * R11 + S12 * R12 + S13 * R13;
    c.c12 = S11 * R21 + S12 * R22 + S13 * R23;
    c.c13 = S11 * R31 + S12 * R32 + S13 * R33;
    c.c22 = S21 * R21 + S22 * R22 + S23 * R23;
    c.c23 = S21 * R31 + S22 * R32 + S23 * R33;
    c.c33 = S31 * R31 + S32 * R32 + S33 * R33;
    return c;
}

__device__ __forceinline__ Cov3d cov3d_of(const uint32_t g, const float* __restrict__ scales,
                                          const float4* __restrict__ rotations, bool& valid) {
    return cov3d_from(scales[3 * g + 0], scales[3 * g + 1], scales[3 * g + 2], rotations[g], valid);
}

// ---- quantised layout (sgs_quantize, quantize.cu; the README.md:143-147 improvement) ----
// A Gaussian is one 16-byte record: its position in 11-10-11 bits relative to the box of its chunk
// of kQuantChunk consecutive Gaussians (the chunk table holds (lo, 0) and (extent, 0) per chunk), its
// rotation as the three smallest components of the normalised quaternion (2 + 3 x 10 bits), its
// log-scales and opacity logit as IEEE half; the SH coefficients are IEEE half. records == nullptr
// selects the float32 arrays.
constexpr uint32_t kQuantChunk = 256;

struct QuantizedModel {
    const uint4* records;
    const float4* chunks;
    const __half* sh;
};

__device__ __forceinline__ float quant_half(const uint32_t bits16) {
    return __half2float(__ushort_as_half(static_cast<unsigned short>(bits16 & 0xffffu)));
}

__device__ __forceinline__ float3 quant_position(const QuantizedModel& q, const uint32_t g, const uint32_t w) {
    const float4 lo = q.chunks[2 * (g / kQuantChunk)];
    const float4 ext = q.chunks[2 * (g / kQuantChunk) + 1];
    return make_float3(lo.x + static_cast<float>(w >> 21) * (ext.x * (1.0f / 2047.0f)),
                       lo.y + static_cast<float>((w >> 11) & 1023u) * (ext.y * (1.0f / 1023.0f)),
                       lo.z + static_cast<float>(w & 2047u) * (ext.z * (1.0f / 2047.0f)));
}

__device__ __forceinline__ float4 quant_rotation(const uint32_t w) {
    const uint32_t big = w >> 30;
    const float c0 = (static_cast<float>((w >> 20) & 1023u) * (2.0f / 1022.0f) - 1.0f) * 0.70710678f;
    const float c1 = (static_cast<float>((w >> 10) & 1023u) * (2.0f / 1022.0f) - 1.0f) * 0.70710678f;
    const float c2 = (static_cast<float>(w & 1023u) * (2.0f / 1022.0f) - 1.0f) * 0.70710678f;
    const float l = sqrtf(fmaxf(0.0f, 1.0f - (c0 * c0 + c1 * c1 + c2 * c2)));
    return make_float4(big == 0 ? l : c0, big == 1 ? l : (big == 0 ? c0 : c1), big == 2 ? l : (big <= 1 ? c1 : c2),
                       big == 3 ? l : c2);
}

// Sigmoid of the opacity logit (gs_utils.h:77-79).
__device__ __forceinline__ float opacity_of(const float raw_opacity) { return 1.0f / (1.0f + expf(-raw_opacity)); }

// Preactivated layout of one Gaussian: two float4, (c11, c12, c13, c22) and (c23, c33, opacity,
// 1 when the quaternion is usable else 0), computed once by sgs_preactivate from the same code.
__device__ __forceinline__ void preactivated_of(const uint32_t g, const float* __restrict__ scales,
                                                const float4* __restrict__ rotations,
                                                const float* __restrict__ opacities, float4& v0, float4& v1) {
    bool valid = true;
    const Cov3d c = cov3d_of(g, scales, rotations, valid);
    v0 = make_float4(c.c11, c.c12, c.c13, c.c22);
    v1 = make_float4(c.c23, c.c33, opacity_of(opacities[g]), valid ? 1.0f : 0.0f);
}

// Loads and projects Gaussian `g`; clears `active` when it is culled. Returns false when no lane
// of the calling warp is active after the depth test or at the end (the warp may then skip the
// rest of its work); the early exits mirror gs_utils.h:74-75,189-190 and keep the loads of culled
// warps from happening.
// `pre` (nullable): the preactivated layout of the same Gaussians; when given, covariance and
// opacity are read from it instead of being rebuilt from scales, rotations and the opacity logit.
// `qm` (records == nullptr: unused): the quantised layout, decoded in place of every float32 array.
__device__ __forceinline__ bool project_gaussian(bool& active, const uint32_t g, const float* __restrict__ means,
                                                 const float* __restrict__ scales, const float4* __restrict__ rotations,
                                                 const float* __restrict__ opacities, const float4* __restrict__ w2c,
                                                 const PassCamera& cam, Projected& p,
                                                 const float4* __restrict__ pre = nullptr,
                                                 const QuantizedModel qm = QuantizedModel{}) {
    uint4 rec = make_uint4(0u, 0u, 0u, 0u);
    float mx, my, mz;
    if (qm.records != nullptr) {
        rec = qm.records[g];
        const float3 m = quant_position(qm, g, rec.x);
        mx = m.x, my = m.y, mz = m.z;
    } else {
        mx = means[3 * g + 0], my = means[3 * g + 1], mz = means[3 * g + 2];
    }
    const float4 r3 = w2c[2];
    p.depth = r3.x * mx + r3.y * my + r3.z * mz + r3.w;
    if (p.depth < cam.near_plane || p.depth > cam.far_plane) active = false;
    if (__ballot_sync(0xffffffffu, active) == 0) return false;

    Cov3d cv;
    if (pre != nullptr) {
        const float4 v0 = pre[2 * g], v1 = pre[2 * g + 1];
        p.opacity = v1.z;
        if (p.opacity < kMinAlpha) active = false;
        if (v1.w == 0.0f) active = false;
        cv.c11 = v0.x, cv.c12 = v0.y, cv.c13 = v0.z, cv.c22 = v0.w, cv.c23 = v1.x, cv.c33 = v1.y;
    } else if (qm.records != nullptr) {
        p.opacity = opacity_of(quant_half(rec.w >> 16));
        if (p.opacity < kMinAlpha) active = false;
        cv = cov3d_from(quant_half(rec.z), quant_half(rec.z >> 16), quant_half(rec.w), quant_rotation(rec.y), active);
    } else {
        p.opacity = opacity_of(opacities[g]);
        if (p.opacity < kMinAlpha) active = false;
        cv = cov3d_of(g, scales, rotations, active);
    }
    const float c11 = cv.c11, c12 = cv.c12, c13 = cv.c13, c22 = cv.c22, c23 = cv.c23, c33 = cv.c33;

    const float4 r1 = w2c[0];
    const float x = (r1.x * mx + r1.y * my + r1.z * mz + r1.w) / p.depth;
    const float4 r2 = w2c[1];
    const float y = (r2.x * mx + r2.y * my + r2.z * mz + r2.w) / p.depth;

    // EWA Jacobian with the position clamped to 1.15x the view frustum
    const float clip_left = (-0.15f * cam.width - cam.center_x) / cam.focal_x;
    const float clip_right = (1.15f * cam.width - cam.center_x) / cam.focal_x;
    const float clip_top = (-0.15f * cam.height - cam.center_y) / cam.focal_y;
    const float clip_bottom = (1.15f * cam.height - cam.center_y) / cam.focal_y;
    const float xc = fmaxf(clip_left, fminf(x, clip_right));
    const float yc = fmaxf(clip_top, fminf(y, clip_bottom));
    const float j11 = cam.focal_x / p.depth;
    const float j13 = -j11 * xc;
    const float j22 = cam.focal_y / p.depth;
    const float j23 = -j22 * yc;
    const float a1 = j11 * r1.x + j13 * r3.x, a2 = j11 * r1.y + j13 * r3.y, a3 = j11 * r1.z + j13 * r3.z;
    const float b1 = j22 * r2.x + j23 * r3.x, b2 = j22 * r2.y + j23 * r3.y, b3 = j22 * r2.z + j23 * r3.z;
    const float ac1 = a1 * c11 + a2 * c12 + a3 * c13;
    const float ac2 = a1 * c12 + a2 * c22 + a3 * c23;
    const float ac3 = a1 * c13 + a2 * c23 + a3 * c33;
    const float bc1 = b1 * c11 + b2 * c12 + b3 * c13;
    const float bc2 = b1 * c12 + b2 * c22 + b3 * c23;
    const float bc3 = b1 * c13 + b2 * c23 + b3 * c33;
    float cxx = ac1 * a1 + ac2 * a2 + ac3 * a3;
    const float cxy = ac1 * b1 + ac2 * b2 + ac3 * b3;
    float cyy = bc1 * b1 + bc2 * b2 + bc3 * b3;
    const float det_raw = cxx * cyy - cxy * cxy;
    const float kernel = (cam.proper_aa ? kDilationProperAA : kDilation) * cam.ss * cam.ss;
    cxx += kernel;
    cyy += kernel;
    p.cov2d = make_float3(cxx, cxy, cyy);
    p.determinant = cxx * cyy - cxy * cxy;
    if (p.determinant < kMinCov2dDeterminant) active = false;
    p.conic = make_float3(cyy / p.determinant, -cxy / p.determinant, cxx / p.determinant);
    if (cam.proper_aa) {
        p.opacity *= sqrtf(fmaxf(det_raw / p.determinant, 0.0f));
        if (p.opacity < kMinAlpha) active = false;
    }
    p.mean2d = make_float2(x * cam.focal_x + cam.center_x, y * cam.focal_y + cam.center_y);

    // screen bounds of the ellipse where alpha reaches 1/255
    p.power_threshold = logf(p.opacity * kMinAlphaRcp);
    const float cutoff = 2.0f * p.power_threshold;
    const float ex = sqrtf(cxx * cutoff);
    const float ey = sqrtf(cyy * cutoff);
    p.bounds = make_float4(p.mean2d.x - ex, p.mean2d.x + ex, p.mean2d.y - ey, p.mean2d.y + ey);
    if (p.bounds.x >= cam.width || p.bounds.y < 0.0f || p.bounds.z >= cam.height || p.bounds.w < 0.0f) active = false;
    if (__ballot_sync(0xffffffffu, active) == 0) return false;
    return true;
}

// Conic scaled by -log2(e)/2 (and -log2(e) off-diagonal) so alpha needs one exp2 (gs_utils.h:21-24).
__device__ __forceinline__ float3 conic_for_exp2(const float3 c) {
    constexpr float log2e = 1.44269504089f;
    return make_float3(-0.5f * log2e * c.x, -log2e * c.y, -0.5f * log2e * c.z);
}

// alpha of a fragment at offset (dx, dy) from the shifted mean, as scatter_utils.cuh:37-40.
__device__ __forceinline__ float fragment_alpha(const float3 ce, const float opacity, const float dx, const float dy) {
    const float exponent = dx * (ce.x * dx + ce.y * dy) + ce.z * dy * dy;
    return opacity * exp2f(fminf(exponent, 0.0f));
}

// Integer AABB of the projected ellipse clipped to the framebuffer (accumulate_scatter.cu:63-70).
struct PixelRect {
    uint32_t x_min, y_min, width, height;
};

__device__ __forceinline__ PixelRect pixel_rect(const float4 b, const PassCamera& cam) {
    const uint32_t x_min = __float2uint_rd(fmaxf(b.x, 0.0f));
    const uint32_t x_max = __float2uint_ru(fminf(b.y, cam.width));
    const uint32_t y_min = __float2uint_rd(fmaxf(b.z, 0.0f));
    const uint32_t y_max = __float2uint_ru(fminf(b.w, cam.height));
    return PixelRect{x_min, y_min, x_max - x_min, y_max - y_min};
}

// ---- spherical harmonics (gs_utils.h:196-243) ----
constexpr float kSH0 = 0.28209479177387814f;
constexpr float kSH1 = 0.48860251190291987f;
constexpr float kSH2a = 1.0925484305920792f;
constexpr float kSH2b = 0.94617469575755997f;
constexpr float kSH2c = 0.31539156525251999f;
constexpr float kSH2d = 0.54627421529603959f;
constexpr float kSH3a = 0.59004358992664352f;
constexpr float kSH3b = 1.7701307697799304f;
constexpr float kSH3c = 2.8906114426405538f;
constexpr float kSH3d = 0.45704579946446572f;
constexpr float kSH3e = 2.2852289973223288f;
constexpr float kSH3f = 1.865881662950577f;
constexpr float kSH3g = 1.1195289977703462f;
constexpr float kSH3h = 1.4453057213202769f;

// Accumulates `w * c` into colour with the reference's left-to-right association
// (colour +/- scalar * coefficient, one component at a time).
__device__ __forceinline__ void sh_add(float3& color, const float w, const float* c) {
    color.x = color.x + w * c[0];
    color.y = color.y + w * c[1];
    color.z = color.z + w * c[2];
}
__device__ __forceinline__ void sh_sub(float3& color, const float w, const float* c) {
    color.x = color.x - w * c[0];
    color.y = color.y - w * c[1];
    color.z = color.z - w * c[2];
}

// View-dependent colour of one Gaussian: `coeffs` points at its (bases, 3) coefficients, the
// direction is normalised. Degree follows the number of bases (1, 4, 9 or 16); colour + 0.5,
// clamped at zero.
__device__ __forceinline__ float3 eval_sh(const float* __restrict__ coeffs, const float x, const float y, const float z,
                                          const uint32_t bases) {
    float3 color = make_float3(0.5f + kSH0 * coeffs[0], 0.5f + kSH0 * coeffs[1], 0.5f + kSH0 * coeffs[2]);
    if (bases > 1) {
        sh_sub(color, kSH1 * y, coeffs + 3);
        sh_add(color, kSH1 * z, coeffs + 6);
        sh_sub(color, kSH1 * x, coeffs + 9);
        if (bases > 4) {
            const float xx = x * x, yy = y * y, zz = z * z;
            const float xy = x * y, xz = x * z, yz = y * z;
            sh_add(color, kSH2a * xy, coeffs + 12);
            sh_sub(color, kSH2a * yz, coeffs + 15);
            sh_add(color, kSH2b * zz - kSH2c, coeffs + 18);
            sh_sub(color, kSH2a * xz, coeffs + 21);
            sh_add(color, kSH2d * (xx - yy), coeffs + 24);
            if (bases > 9) {
                sh_add(color, y * (kSH3a * yy - kSH3b * xx), coeffs + 27);
                sh_add(color, kSH3c * xy * z, coeffs + 30);
                sh_add(color, y * (kSH3d - kSH3e * zz), coeffs + 33);
                sh_add(color, z * (kSH3f * zz - kSH3g), coeffs + 36);
                sh_add(color, x * (kSH3d - kSH3e * zz), coeffs + 39);
                sh_add(color, kSH3h * z * (xx - yy), coeffs + 42);
                sh_add(color, x * (kSH3b * yy - kSH3a * xx), coeffs + 45);
            }
        }
    }
    return make_float3(fmaxf(color.x, 0.0f), fmaxf(color.y, 0.0f), fmaxf(color.z, 0.0f));
}

}  // namespace sgs
