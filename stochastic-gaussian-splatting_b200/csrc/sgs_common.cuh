// Device-side building blocks of the per-sample stochastic render path: constants, random
// number generators and the packed fragment key.
//
// Bit-exactness contract: every floating-point expression below keeps the operand order and
// association of the reference (StochasticGSCudaBackend/StochasticGSCudaBackend/*.h), and the
// library is compiled with the reference's flags (-O3 -use_fast_math), so the compiler forms the
// same fused multiply-adds and calls the same intrinsics. The integer generators are exact.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace sgs {

// ---- Gaussian splatting constants (gs_utils.h:13-18) ----
constexpr float kDilation = 0.3f;
constexpr float kDilationProperAA = 0.1f;
constexpr float kMinCov2dDeterminant = 1e-6f;
constexpr float kMinAlphaRcp = 255.0f;
constexpr float kMinAlpha = 1.0f / kMinAlphaRcp;
constexpr float kTwoPi = 2.0f * 3.14159265358979323846f;  // math_utils.h:10
constexpr uint32_t kSequentialFragments = 4;               // scatter_utils.cuh:11
constexpr uint32_t kKBufferSize = 4;                        // resolve.h:9

// ---- blue noise volume (math_utils.h:123-125) ----
constexpr uint32_t kBlueNoiseWidth = 128;
constexpr uint32_t kBlueNoiseHeight = 128;
constexpr uint32_t kBlueNoiseDepth = 64;

// Empty framebuffer entry: every bit set, so any accepted fragment is smaller.
constexpr unsigned long long kEmptyFragment = ~0ull;

// Packs the closest-fragment key: view depth bits in the high word (non-negative floats order
// like their bit patterns), Gaussian index in the low word (accumulate_scatter.cu:71-72).
__device__ __forceinline__ unsigned long long pack_fragment(float depth, uint32_t gaussian_idx) {
    return (static_cast<unsigned long long>(__float_as_uint(depth)) << 32) | gaussian_idx;
}

// ---- white-noise threshold of stochastic transparency (math_utils.h:113-122) ----
__device__ __forceinline__ uint32_t pcg_hash(uint32_t seed) {
    const uint32_t state = seed * 747796405u + 2891336453u;
    const uint32_t word = ((state >> ((state >> 28u) + 4u)) ^ state) * 277803737u;
    return (word >> 22u) ^ word;
}

// u in [0, 1) from (frame, Gaussian, pixel): 23 random mantissa bits under exponent 0.
__device__ __forceinline__ float st_uniform(uint32_t frame, uint32_t gaussian, uint32_t x, uint32_t y) {
    const uint32_t seed = gaussian ^ (frame * 1973u) ^ (x * 9277u) ^ (y * 2699u);
    return __uint_as_float(0x3f800000u | (pcg_hash(seed) >> 9u)) - 1.0f;
}

// Spatio-temporal blue-noise threshold (math_utils.h:125-136): per-Gaussian R2 offsets into the
// 128x128 slice, the byte as the top 8 bits of a 0.32 fixed-point value plus half an LSB of the
// byte and the per-pass rotation, converted with 24-bit precision.
__device__ __forceinline__ float st_blue_noise(const uint8_t* __restrict__ slice, uint32_t rotation, uint32_t gaussian,
                                               uint32_t x, uint32_t y) {
    const uint32_t ox = (gaussian * 0xC13FA9A9u) >> 25u;
    const uint32_t oy = (gaussian * 0x91E10DA5u) >> 25u;
    const uint32_t texel = ((y + oy) % kBlueNoiseHeight) * kBlueNoiseWidth + (x + ox) % kBlueNoiseWidth;
    const uint32_t value = (static_cast<uint32_t>(slice[texel]) << 24u) + (1u << 23u) + rotation;
    return static_cast<float>(value >> 8u) * 5.9604644775390625e-8f;
}

// ---- Gaussian point splatting generators (math_utils.h:45-111) ----
__device__ __forceinline__ uint32_t hash32(uint32_t x) {
    x ^= x >> 16;
    x *= 0x7feb352du;
    x ^= x >> 15;
    x *= 0x846ca68bu;
    x ^= x >> 16;
    return x;
}

__device__ __forceinline__ uint2 gps_seed(uint32_t idx, uint32_t frame) {
    uint32_t h1 = hash32(idx ^ (frame * 0x9E3779B9u));
    uint32_t h2 = hash32((idx * 0xBB67AE85u) ^ frame);
    h1 ^= h2 * 0x3C6EF372u;
    h2 ^= h1 * 0xA54FF53Au;
    return make_uint2(h1, h2);
}

// One step of the 2-D PCG hash (Jarzynski & Olano), advancing the state in place.
__device__ __forceinline__ void pcg2d_step(uint2& s) {
    s.x = s.x * 1664525u + 1013904223u;
    s.y = s.y * 1664525u + 1013904223u;
    s.x += s.y * 1664525u;
    s.y += s.x * 1664525u;
    s.x ^= s.x >> 16u;
    s.y ^= s.y >> 16u;
    s.x += s.y * 1664525u;
    s.y += s.x * 1664525u;
    s.x ^= s.x >> 16u;
    s.y ^= s.y >> 16u;
}

// The two uniforms in [0, 1) of a stepped PCG2D state.
__device__ __forceinline__ float2 pcg2d_to_uniform(const uint2 s) {
    return make_float2(static_cast<float>(s.x) * 2.3283064365387e-10f, static_cast<float>(s.y) * 2.3283064365387e-10f);
}

__device__ __forceinline__ float2 pcg2d_uniform(uint2& s) {
    pcg2d_step(s);
    return pcg2d_to_uniform(s);
}

// Polynomial approximations of the dilogarithm-based radial CDF used by GPS to draw points
// from an opacity-truncated Gaussian. Coefficients from Gaussian Point Splatting
// (https://github.com/JorisAR/gaussian-point-splatting, BSD-3-Clause, Copyright (c) 2026 Joris
// Rijsdijk), as used by the reference (math_utils.h:14-43); they define the sampled distribution
// and are kept for parity.
__device__ __forceinline__ float gps_dilog(const float x) {
    float y = -0.952623943f;
    y = fmaf(y, x, 2.995873777f);
    y = fmaf(y, x, -3.762115247f);
    y = fmaf(y, x, 2.334605281f);
    y = fmaf(y, x, -0.773941317f);
    y = fmaf(y, x, 5.97506396e-02f);
    y = fmaf(y, x, -0.256617940f);
    y = fmaf(y, x, 2.000061866f);
    y *= x;
    const float s = 1.0f - x;
    if (s > 0.0f) y += s * logf(fmaxf(s, 1.0e-37f));
    return y;
}

__device__ __forceinline__ float gps_inv_dilog(const float x) {
    const float t = fminf(x / 1.6449340668482264f, 1.0f);
    float y = -1.27463503e+01f;
    y = fmaf(y, t, 5.88993459e+01f);
    y = fmaf(y, t, -1.16025780e+02f);
    y = fmaf(y, t, 1.26945827e+02f);
    y = fmaf(y, t, -8.43108826e+01f);
    y = fmaf(y, t, 3.48799862e+01f);
    y = fmaf(y, t, -8.89606235e+00f);
    y = fmaf(y, t, 1.38640936e+00f);
    y = fmaf(y, t, -7.80640876e-01f);
    y = fmaf(y, t, 1.64841888e+00f);
    y = fmaf(y, t, -2.82836687e-05f);
    return y;
}

// Standard normal pair by the Box-Muller transform (math_utils.h:81-87).
__device__ __forceinline__ float2 box_muller(const float u1, const float u2) {
    const float r = sqrtf(fmaxf(-2.0f * logf(fmaxf(fminf(u1, 1.0f), 1.0e-37f)), 0.0f));
    const float theta = kTwoPi * u2;
    float s, c;
    sincosf(theta, &s, &c);
    return make_float2(r * c, r * s);
}

// Box-Muller with the radius drawn from the opacity-truncated distribution (math_utils.h:89-96).
__device__ __forceinline__ float2 truncated_box_muller(const float u1, const float u2, const float opacity_rcp,
                                                       const float opacity_dilog) {
    const float a = opacity_rcp * gps_inv_dilog((1.0f - u1) * opacity_dilog);
    const float r = sqrtf(fmaxf(-2.0f * logf(fmaxf(fminf(a, 1.0f), 1.0e-37f)), 0.0f));
    const float theta = kTwoPi * u2;
    float s, c;
    sincosf(theta, &s, &c);
    return make_float2(r * c, r * s);
}

// Poisson(lambda) through a normal draw and a Cornish-Fisher-type expansion, rounded
// (math_utils.h:98-111).
__device__ __forceinline__ uint32_t poisson_count(uint2& state, const float lambda) {
    const float2 u = pcg2d_uniform(state);
    const float w = box_muller(u.x, u.y).x;
    const float w2 = w * w;
    const float w3 = w2 * w;
    const float w4 = w2 * w2;
    const float s = sqrtf(lambda);
    const float s_rcp = 1.0f / s;
    const float l_rcp = 1.0f / lambda;
    float kf = lambda + s * w + (w2 - 1.0f) / 6.0f;
    kf += s_rcp * (-(1.0f / 36.0f) * w - (1.0f / 72.0f) * w3);
    kf += l_rcp * (-(8.0f / 405.0f) + (7.0f / 810.0f) * w2 + (1.0f / 270.0f) * w4);
    return __float2uint_rn(fmaxf(kf, 0.0f));
}

}  // namespace sgs
