// Conservative per-row spans of a projected Gaussian's alpha >= 1/255 ellipse.
//
// For a row at offset dy from the shifted mean, the exp2-scaled exponent is the concave quadratic
// e(dx) = cx dx^2 + cy dy dx + cz dy^2 with its maximum at dx = slope * dy; pixels with
// alpha >= 1/255 need e >= T = -log2(255 opacity). Using T minus kSpanExpMargin (far above the float
// error of e or of these constants, which enter only relative to |T|) and widening by
// kSpanPixelMargin gives a superset of the pixels of the row with alpha >= 1/255, so evaluating only
// the span leaves every alpha test of the reference's AABB loop (scatter_utils.cuh:34-94) unchanged.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>
#include "sgs_common.cuh"

namespace sgs {

// Safety margins of the row spans: exponent units (log2 of alpha) and pixels.
constexpr float kSpanExpMargin = 0.125f;
constexpr float kSpanPixelMargin = 0.02f;

struct SpanConstants {
    float slope;   // row centre shift per unit dy
    float k2;      // squared half-width per unit of (dymax2 - dy^2); 0 disables spans (whole AABB rows)
    float dymax2;  // rows with dy^2 > dymax2 hold no pixel with alpha >= 1/255
};

// Span constants from the exp2-scaled conic (cx, cy, cz) and the opacity.
__device__ __forceinline__ SpanConstants span_constants(const float cx, const float cy, const float cz,
                                                        const float opacity) {
    SpanConstants k{0.0f, 0.0f, 0.0f};
    const float T = -log2f(opacity * kMinAlphaRcp) - kSpanExpMargin;
    const float P = 4.0f * cx * cz - cy * cy;  // > 0 for a positive-definite conic
    if (P > 0.0f && cx < 0.0f && T < 0.0f) {
        const float inv_cx = 1.0f / cx;
        const float k2 = 0.25f * P * inv_cx * inv_cx;
        const float dymax2 = 4.0f * cx * T / P;
        const float slope = -0.5f * cy * inv_cx;
        if (isfinite(k2) && isfinite(dymax2) && isfinite(slope) && k2 > 0.0f) {
            k.slope = slope;
            k.k2 = k2;
            k.dymax2 = dymax2;
        }
    }
    return k;
}

// Span [xs, xs + len) of the row at offset dy inside the AABB columns [x_min, x_min + w), for the
// shifted mean x coordinate mx; clamped in floating point first, since the ellipse may lie far
// outside the integer range of the AABB (a non-finite bound leaves the whole AABB row, still a
// superset).
__device__ __forceinline__ void row_span(const uint32_t x_min, const uint32_t w, const float mx,
                                         const SpanConstants& k, const float dy, uint32_t& xs, uint32_t& len) {
    const float lo_f = static_cast<float>(x_min);
    const float hi_f = static_cast<float>(x_min + w - 1u);
    float fl = lo_f, fh = hi_f;
    if (k.k2 > 0.0f) {
        const float rem = fmaf(-dy, dy, k.dymax2);
        const float hw = sqrtf(k.k2 * fmaxf(rem, 0.0f));
        const float c = fmaf(k.slope, dy, mx);
        const float eps = kSpanPixelMargin + 4.0e-6f * (fabsf(c) + hw);
        fl = fmaxf(ceilf(c - hw - eps), lo_f);
        fh = fminf(floorf(c + hw + eps), hi_f);
        if (rem < 0.0f) fh = fl - 1.0f;
    }
    xs = 0;
    len = 0;
    if (fh >= fl) {
        xs = static_cast<uint32_t>(fl);
        len = static_cast<uint32_t>(fh) - xs + 1u;
    }
}

// Inclusive prefix sum over the 32 lanes of a warp (all lanes active).
__device__ __forceinline__ uint32_t warp_inclusive_sum(uint32_t v, const uint32_t lane) {
#pragma unroll
    for (uint32_t o = 1; o < 32; o <<= 1) {
        const uint32_t t = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += t;
    }
    return v;
}

}  // namespace sgs
