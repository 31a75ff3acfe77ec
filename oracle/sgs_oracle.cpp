// CPU restatement of the reference's per-sample stochastic render path (TEST INFRASTRUCTURE).
//
// This oracle is the checker of the B200 kernels and the CPU baseline of the benchmark. Only the
// tests, the smoke check and the benchmark's CPU legs load it; the product never does.
//
// It restates, function by function, the reference StochasticGSCudaBackend:
//   project()            gs_utils.h:38-193         alpha/exponent  scatter_utils.cuh:37-41, accumulate_hybrid.cu:308-311
//   st_uniform()         math_utils.h:113-122      st_blue_noise() math_utils.h:125-136
//   gps_*                math_utils.h:14-111       accumulate_st() accumulate_scatter.cu:19-77 + scatter_utils.cuh:14-95
//   accumulate_gps()     accumulate_scatter.cu:79-146 + scatter_utils.cuh:98-183 (per-lane warp streams)
//   hybrid GPS binning   accumulate_hybrid_gps.cu:27-181      hybrid ST binning accumulate_hybrid.cu:34-321
//   eval_sh()            gs_utils.h:197-243        sample()        resolve.cu:27-144
//   resolve()            resolve.cu:146-349
// in IEEE single precision with libm. The reference runs with -use_fast_math, whose approximate
// exp/log/sqrt/division this file does not imitate, so agreement is a tolerance, except for the
// view depth, whose fused multiply-add form (fma(c, z, fma(a, x, b*y)) + w) is reproduced exactly so
// that winners carry the same depth bits. Where the reference's own kernels contract the alpha
// exponent differently (scatter loops vs hybrid gather) the two forms are reproduced with fmaf.
//
// The pinned state of this oracle: tests/test_oracle_golden.py checks it against golden outputs
// that the reference's own CUDA kernels produced on a B200 (tests/golden/, made by
// tests/golden/make_golden.py).
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

constexpr float kDilation = 0.3f;
constexpr float kDilationAA = 0.1f;
constexpr float kMinDet = 1e-6f;
constexpr float kMinAlphaRcp = 255.0f;
constexpr float kMinAlpha = 1.0f / kMinAlphaRcp;
constexpr float kTwoPi = 2.0f * 3.14159265358979323846f;
constexpr uint32_t kSeq = 4;
constexpr uint32_t kK = 4;
constexpr uint64_t kEmpty = ~0ull;

struct Cam {
    float width, height, fx, fy, cx, cy, near_plane, far_plane, ss;
    uint32_t width_int;
    bool aa;
};

struct Proj {
    bool active;
    float depth, opacity, det, power;
    float mx, my;       // mean2d
    float conic[3];
    float cov[3];
    float bounds[4];    // x_min, x_max, y_min, y_max
};

inline float fmaf_(float a, float b, float c) { return std::fmaf(a, b, c); }

// gs_utils.h:38-193 (the culled flag is per Gaussian; warp-level early exits do not change results)
Proj project(const float* means, const float* scales, const float* rot, const float* opac, const float* w2c,
             uint32_t g, const Cam& cam) {
    Proj p{};
    p.active = true;
    const float mx = means[3 * g], my = means[3 * g + 1], mz = means[3 * g + 2];
    const float* r1 = w2c;
    const float* r2 = w2c + 4;
    const float* r3 = w2c + 8;
    p.depth = fmaf_(r3[2], mz, fmaf_(r3[0], mx, r3[1] * my)) + r3[3];
    if (p.depth < cam.near_plane || p.depth > cam.far_plane) p.active = false;
    p.opacity = 1.0f / (1.0f + std::exp(-opac[g]));
    if (p.opacity < kMinAlpha) p.active = false;
    const float vx = std::exp(2.0f * scales[3 * g]), vy = std::exp(2.0f * scales[3 * g + 1]),
                vz = std::exp(2.0f * scales[3 * g + 2]);
    const float r = rot[4 * g], i = rot[4 * g + 1], j = rot[4 * g + 2], k = rot[4 * g + 3];
    const float ii = i * i, jj = j * j, kk = k * k, ij = i * j, ik = i * k, jk = j * k, ri = r * i, rj = r * j, rk = r * k;
    const float nsq = r * r + ii + jj + kk;
    if (nsq < 1e-8f) p.active = false;
    const float n = 1.0f / nsq;
    const float R[3][3] = {{1.0f - 2.0f * (jj + kk) * n, 2.0f * (ij - rk) * n, 2.0f * (ik + rj) * n},
                           {2.0f * (ij + rk) * n, 1.0f - 2.0f * (ii + kk) * n, 2.0f * (jk - ri) * n},
                           {2.0f * (ik - rj) * n, 2.0f * (jk + ri) * n, 1.0f - 2.0f * (ii + jj) * n}};
    const float v[3] = {vx, vy, vz};
    float S[3][3];
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) S[a][b] = R[a][b] * v[b];
    auto row_dot = [](const float* x, const float* y) { return x[0] * y[0] + x[1] * y[1] + x[2] * y[2]; };
    const float c11 = row_dot(S[0], R[0]), c12 = row_dot(S[0], R[1]), c13 = row_dot(S[0], R[2]);
    const float c22 = row_dot(S[1], R[1]), c23 = row_dot(S[1], R[2]), c33 = row_dot(S[2], R[2]);
    const float x = (r1[0] * mx + r1[1] * my + r1[2] * mz + r1[3]) / p.depth;
    const float y = (r2[0] * mx + r2[1] * my + r2[2] * mz + r2[3]) / p.depth;
    const float cl = (-0.15f * cam.width - cam.cx) / cam.fx, cr = (1.15f * cam.width - cam.cx) / cam.fx;
    const float ct = (-0.15f * cam.height - cam.cy) / cam.fy, cb = (1.15f * cam.height - cam.cy) / cam.fy;
    const float xc = std::max(cl, std::min(x, cr)), yc = std::max(ct, std::min(y, cb));
    const float j11 = cam.fx / p.depth, j13 = -j11 * xc, j22 = cam.fy / p.depth, j23 = -j22 * yc;
    const float a[3] = {j11 * r1[0] + j13 * r3[0], j11 * r1[1] + j13 * r3[1], j11 * r1[2] + j13 * r3[2]};
    const float b[3] = {j22 * r2[0] + j23 * r3[0], j22 * r2[1] + j23 * r3[1], j22 * r2[2] + j23 * r3[2]};
    const float ac[3] = {a[0] * c11 + a[1] * c12 + a[2] * c13, a[0] * c12 + a[1] * c22 + a[2] * c23,
                         a[0] * c13 + a[1] * c23 + a[2] * c33};
    const float bc[3] = {b[0] * c11 + b[1] * c12 + b[2] * c13, b[0] * c12 + b[1] * c22 + b[2] * c23,
                         b[0] * c13 + b[1] * c23 + b[2] * c33};
    float cxx = row_dot(ac, a);
    const float cxy = row_dot(ac, b);
    float cyy = row_dot(bc, b);
    const float det_raw = cxx * cyy - cxy * cxy;
    const float kernel = (cam.aa ? kDilationAA : kDilation) * cam.ss * cam.ss;
    cxx += kernel;
    cyy += kernel;
    p.cov[0] = cxx;
    p.cov[1] = cxy;
    p.cov[2] = cyy;
    p.det = cxx * cyy - cxy * cxy;
    if (p.det < kMinDet) p.active = false;
    p.conic[0] = cyy / p.det;
    p.conic[1] = -cxy / p.det;
    p.conic[2] = cxx / p.det;
    if (cam.aa) {
        p.opacity *= std::sqrt(std::max(det_raw / p.det, 0.0f));
        if (p.opacity < kMinAlpha) p.active = false;
    }
    p.mx = x * cam.fx + cam.cx;
    p.my = y * cam.fy + cam.cy;
    p.power = std::log(p.opacity * kMinAlphaRcp);
    const float cut = 2.0f * p.power;
    const float ex = std::sqrt(cxx * cut), ey = std::sqrt(cyy * cut);
    p.bounds[0] = p.mx - ex;
    p.bounds[1] = p.mx + ex;
    p.bounds[2] = p.my - ey;
    p.bounds[3] = p.my + ey;
    if (p.bounds[0] >= cam.width || p.bounds[1] < 0.0f || p.bounds[2] >= cam.height || p.bounds[3] < 0.0f)
        p.active = false;
    return p;
}

struct Rect {
    uint32_t x0, y0, w, h;
};

// accumulate_scatter.cu:63-70 (float -> uint conversions round down / up, negatives to 0)
uint32_t to_uint_rd(float v) { return v <= 0.0f ? 0u : static_cast<uint32_t>(std::floor(v)); }
uint32_t to_uint_ru(float v) { return v <= 0.0f ? 0u : static_cast<uint32_t>(std::ceil(v)); }

Rect rect_of(const Proj& p, const Cam& cam) {
    const uint32_t x0 = to_uint_rd(std::max(p.bounds[0], 0.0f));
    const uint32_t x1 = to_uint_ru(std::min(p.bounds[1], cam.width));
    const uint32_t y0 = to_uint_rd(std::max(p.bounds[2], 0.0f));
    const uint32_t y1 = to_uint_ru(std::min(p.bounds[3], cam.height));
    return Rect{x0, y0, x1 - x0, y1 - y0};
}

// exponent of alpha with the fused forms of the reference's compiled kernels:
// scatter loops: fma(cz*dy, dy, dx*fma(cx, dx, cy*dy)); hybrid gather: fma(dx, fma(cx, dx, cy*dy), (cz*dy)*dy)
float st_alpha(const Proj& p, float px, float py, bool gather_form) {
    constexpr float log2e = 1.44269504089f;
    const float cx = -0.5f * log2e * p.conic[0], cy = -log2e * p.conic[1], cz = -0.5f * log2e * p.conic[2];
    const float dx = px - (p.mx - 0.5f), dy = py - (p.my - 0.5f);
    const float inner = fmaf_(cx, dx, cy * dy);
    const float czdy = cz * dy;
    const float e = gather_form ? fmaf_(dx, inner, czdy * dy) : fmaf_(czdy, dy, dx * inner);
    return p.opacity * std::exp2(std::min(e, 0.0f));
}

uint32_t pcg_hash(uint32_t seed) {
    const uint32_t state = seed * 747796405u + 2891336453u;
    const uint32_t word = ((state >> ((state >> 28u) + 4u)) ^ state) * 277803737u;
    return (word >> 22u) ^ word;
}

float bits_to_float(uint32_t u) {
    float f;
    std::memcpy(&f, &u, 4);
    return f;
}
uint32_t float_to_bits(float f) {
    uint32_t u;
    std::memcpy(&u, &f, 4);
    return u;
}

float st_uniform(uint32_t frame, uint32_t g, uint32_t x, uint32_t y) {
    const uint32_t seed = g ^ (frame * 1973u) ^ (x * 9277u) ^ (y * 2699u);
    return bits_to_float(0x3f800000u | (pcg_hash(seed) >> 9u)) - 1.0f;
}

float st_blue(const uint8_t* slice, uint32_t rotation, uint32_t g, uint32_t x, uint32_t y) {
    const uint32_t ox = (g * 0xC13FA9A9u) >> 25u, oy = (g * 0x91E10DA5u) >> 25u;
    const uint32_t texel = ((y + oy) % 128u) * 128u + (x + ox) % 128u;
    const uint32_t value = (static_cast<uint32_t>(slice[texel]) << 24u) + (1u << 23u) + rotation;
    return static_cast<float>(value >> 8u) * 5.9604644775390625e-8f;
}

uint32_t hash32(uint32_t x) {
    x ^= x >> 16;
    x *= 0x7feb352du;
    x ^= x >> 15;
    x *= 0x846ca68bu;
    x ^= x >> 16;
    return x;
}

struct Seed {
    uint32_t x, y;
};

Seed gps_seed(uint32_t idx, uint32_t frame) {
    uint32_t h1 = hash32(idx ^ (frame * 0x9E3779B9u));
    uint32_t h2 = hash32((idx * 0xBB67AE85u) ^ frame);
    h1 ^= h2 * 0x3C6EF372u;
    h2 ^= h1 * 0xA54FF53Au;
    return Seed{h1, h2};
}

void pcg2d(Seed& s, float& u1, float& u2) {
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
    u1 = static_cast<float>(s.x) * 2.3283064365387e-10f;
    u2 = static_cast<float>(s.y) * 2.3283064365387e-10f;
}

// Polynomial dilogarithm approximations of Gaussian Point Splatting (BSD-3-Clause, Copyright (c) 2026
// Joris Rijsdijk), as used by the reference (math_utils.h:14-43); they define the sampled distribution.
float gps_dilog(float x) {
    float y = -0.952623943f;
    y = std::fmaf(y, x, 2.995873777f);
    y = std::fmaf(y, x, -3.762115247f);
    y = std::fmaf(y, x, 2.334605281f);
    y = std::fmaf(y, x, -0.773941317f);
    y = std::fmaf(y, x, 5.97506396e-02f);
    y = std::fmaf(y, x, -0.256617940f);
    y = std::fmaf(y, x, 2.000061866f);
    y *= x;
    const float s = 1.0f - x;
    if (s > 0.0f) y += s * std::log(std::max(s, 1.0e-37f));
    return y;
}

float gps_inv_dilog(float x) {
    const float t = std::min(x / 1.6449340668482264f, 1.0f);
    float y = -1.27463503e+01f;
    y = std::fmaf(y, t, 5.88993459e+01f);
    y = std::fmaf(y, t, -1.16025780e+02f);
    y = std::fmaf(y, t, 1.26945827e+02f);
    y = std::fmaf(y, t, -8.43108826e+01f);
    y = std::fmaf(y, t, 3.48799862e+01f);
    y = std::fmaf(y, t, -8.89606235e+00f);
    y = std::fmaf(y, t, 1.38640936e+00f);
    y = std::fmaf(y, t, -7.80640876e-01f);
    y = std::fmaf(y, t, 1.64841888e+00f);
    y = std::fmaf(y, t, -2.82836687e-05f);
    return y;
}

void truncated_box_muller(float u1, float u2, float op_rcp, float op_dilog, float& ox, float& oy) {
    const float a = op_rcp * gps_inv_dilog((1.0f - u1) * op_dilog);
    const float R = std::sqrt(std::max(-2.0f * std::log(std::max(std::min(a, 1.0f), 1.0e-37f)), 0.0f));
    const float th = kTwoPi * u2;
    ox = R * std::cos(th);
    oy = R * std::sin(th);
}

uint32_t poisson_count(Seed& s, float lambda) {
    float u1, u2;
    pcg2d(s, u1, u2);
    const float R = std::sqrt(std::max(-2.0f * std::log(std::max(std::min(u1, 1.0f), 1.0e-37f)), 0.0f));
    const float w = R * std::cos(kTwoPi * u2);
    const float w2 = w * w, w3 = w2 * w, w4 = w2 * w2;
    const float sq = std::sqrt(lambda), s_rcp = 1.0f / sq, l_rcp = 1.0f / lambda;
    float kf = lambda + sq * w + (w2 - 1.0f) / 6.0f;
    kf += s_rcp * (-(1.0f / 36.0f) * w - (1.0f / 72.0f) * w3);
    kf += l_rcp * (-(8.0f / 405.0f) + (7.0f / 810.0f) * w2 + (1.0f / 270.0f) * w4);
    return static_cast<uint32_t>(std::nearbyint(std::max(kf, 0.0f)));
}

void atomic_min_u64(uint64_t* addr, uint64_t v) {
    uint64_t cur = __atomic_load_n(addr, __ATOMIC_RELAXED);
    while (v < cur && !__atomic_compare_exchange_n(addr, &cur, v, true, __ATOMIC_RELAXED, __ATOMIC_RELAXED)) {
    }
}

uint64_t pack(float depth, uint32_t g) { return (static_cast<uint64_t>(float_to_bits(depth)) << 32) | g; }

struct GpsSource {
    float mx, my, conic[3], L[3], power, op_rcp, op_dilog;
    uint64_t key;
};

// one point of scatter_utils.cuh:116-129 / accumulate_hybrid_gps.cu:167-180
void gps_point(Seed& seed, const GpsSource& s, const Cam& cam, uint64_t* fb) {
    float u1, u2, xx, yy;
    pcg2d(seed, u1, u2);
    truncated_box_muller(u1, u2, s.op_rcp, s.op_dilog, xx, yy);
    const float sx = s.mx + s.L[0] * xx;
    const float sy = s.my + (s.L[1] * xx + s.L[2] * yy);
    if (sx >= cam.width || sx < 0.0f || sy >= cam.height || sy < 0.0f) return;
    const float dcx = std::trunc(sx) + 0.5f - s.mx, dcy = std::trunc(sy) + 0.5f - s.my;
    const float power = 0.5f * (s.conic[0] * dcx * dcx + s.conic[2] * dcy * dcy) + s.conic[1] * dcx * dcy;
    if (power > s.power) return;
    const uint32_t px = static_cast<uint32_t>(sx), py = static_cast<uint32_t>(sy);
    atomic_min_u64(&fb[static_cast<size_t>(py) * cam.width_int + px], s.key);
}

Cam make_cam(uint32_t width, uint32_t height, float fx, float fy, float cx, float cy, float near_plane, float far_plane,
             int aa, int ss_raw) {
    const uint32_t ss = ss_raw < 1 ? 1u : static_cast<uint32_t>(ss_raw);
    const float s = static_cast<float>(ss);
    Cam c;
    c.width = static_cast<float>(width * ss);
    c.height = static_cast<float>(height * ss);
    c.fx = fx * s;
    c.fy = fy * s;
    c.cx = cx * s;
    c.cy = cy * s;
    c.near_plane = near_plane;
    c.far_plane = far_plane;
    c.ss = s;
    c.width_int = width * ss;
    c.aa = aa != 0;
    return c;
}

void set_threads(int threads) {
#ifdef _OPENMP
    if (threads > 0) omp_set_num_threads(threads);
#else
    (void)threads;
#endif
}

// degree <= 3 SH (gs_utils.h:197-243)
void eval_sh(const float* c, float x, float y, float z, uint32_t bases, float out[3]) {
    constexpr float C0 = 0.28209479177387814f, C1 = 0.48860251190291987f, C2a = 1.0925484305920792f,
                    C2b = 0.94617469575755997f, C2c = 0.31539156525251999f, C2d = 0.54627421529603959f,
                    C3a = 0.59004358992664352f, C3b = 1.7701307697799304f, C3c = 2.8906114426405538f,
                    C3d = 0.45704579946446572f, C3e = 2.2852289973223288f, C3f = 1.865881662950577f,
                    C3g = 1.1195289977703462f, C3h = 1.4453057213202769f;
    for (int ch = 0; ch < 3; ++ch) {
        float col = 0.5f + C0 * c[ch];
        if (bases > 1) {
            col = col - C1 * y * c[3 + ch] + C1 * z * c[6 + ch] - C1 * x * c[9 + ch];
            if (bases > 4) {
                const float xx = x * x, yy = y * y, zz = z * z, xy = x * y, xz = x * z, yz = y * z;
                col = col + C2a * xy * c[12 + ch] - C2a * yz * c[15 + ch] + (C2b * zz - C2c) * c[18 + ch] -
                      C2a * xz * c[21 + ch] + C2d * (xx - yy) * c[24 + ch];
                if (bases > 9) {
                    col = col + y * (C3a * yy - C3b * xx) * c[27 + ch] + C3c * xy * z * c[30 + ch] +
                          y * (C3d - C3e * zz) * c[33 + ch] + z * (C3f * zz - C3g) * c[36 + ch] +
                          x * (C3d - C3e * zz) * c[39 + ch] + C3h * z * (xx - yy) * c[42 + ch] +
                          x * (C3b * yy - C3a * xx) * c[45 + ch];
                }
            }
        }
        out[ch] = std::max(col, 0.0f);
    }
}

}  // namespace

extern "C" {

struct OracleStats {
    uint64_t fragments;  // AABB pixels evaluated (ST) or points drawn (GPS)
    uint64_t accepted;   // fragments merged into the framebuffer
    uint64_t binned;     // Gaussians handled by the hybrid pass
};

int oracle_abi_version(void) { return 1; }

// Per-Gaussian projection (18 floats: active, depth, opacity, det, power, mean2d xy, conic xyz,
// cov2d xyz, bounds x_min x_max y_min y_max, active) in framebuffer (sub)pixels.
int oracle_project(const float* means, const float* scales, const float* rotations, const float* opacities,
                   uint32_t n, const float* w2c, uint32_t width, uint32_t height, float fx, float fy, float cx,
                   float cy, float near_plane, float far_plane, int aa, int ss, float* out) {
    const Cam cam = make_cam(width, height, fx, fy, cx, cy, near_plane, far_plane, aa, ss);
    for (uint32_t g = 0; g < n; ++g) {
        const Proj p = project(means, scales, rotations, opacities, w2c, g, cam);
        float* o = out + static_cast<size_t>(g) * 18;
        o[0] = p.active ? 1.0f : 0.0f;
        o[1] = p.depth;
        o[2] = p.opacity;
        o[3] = p.det;
        o[4] = p.power;
        o[5] = p.mx;
        o[6] = p.my;
        o[7] = p.conic[0];
        o[8] = p.conic[1];
        o[9] = p.conic[2];
        o[10] = p.cov[0];
        o[11] = p.cov[1];
        o[12] = p.cov[2];
        o[13] = p.bounds[0];
        o[14] = p.bounds[1];
        o[15] = p.bounds[2];
        o[16] = p.bounds[3];
        o[17] = o[0];
    }
    return 0;
}

// Closest accepted fragment per (sub)pixel (render.cu:65-125). `blue_noise` is the (64,128,128)
// volume or null; `max_fragments` / `max_binned` 0 take the reference defaults.
int oracle_accumulate(const float* means, const float* scales, const float* rotations, const float* opacities,
                      uint32_t n, const float* w2c, uint32_t width, uint32_t height, float fx, float fy, float cx,
                      float cy, float near_plane, float far_plane, int aa, int ss, int use_gps, int hybrid,
                      const uint8_t* blue_noise, uint32_t frame, uint32_t max_fragments, uint32_t max_binned,
                      int threads, uint64_t* fb, OracleStats* stats) {
    set_threads(threads);
    const Cam cam = make_cam(width, height, fx, fy, cx, cy, near_plane, far_plane, aa, ss);
    const size_t n_fb = static_cast<size_t>(cam.width_int) * static_cast<uint32_t>(cam.height);
    std::fill(fb, fb + n_fb, kEmpty);
    std::atomic<uint64_t> n_frag{0}, n_acc{0};
    uint64_t n_binned = 0;
    const uint32_t cap_binned = std::min<uint32_t>(n, max_binned ? max_binned : (1u << 20));
    if (n == 0) {
        if (stats) *stats = OracleStats{0, 0, 0};
        return 0;
    }
    std::vector<Proj> proj(n);
#pragma omp parallel for schedule(static)
    for (int64_t g = 0; g < static_cast<int64_t>(n); ++g)
        proj[g] = project(means, scales, rotations, opacities, w2c, static_cast<uint32_t>(g), cam);

    if (!use_gps) {
        const uint8_t* slice = blue_noise ? blue_noise + static_cast<size_t>(frame % 64u) * 128u * 128u : nullptr;
        const uint32_t rotation = (frame / 64u) * 0x9E3779B9u;
        // hybrid: the first max_binned Gaussians above 512 pixels use the gather kernel's form
        std::vector<uint8_t> gathered(hybrid ? n : 0, 0);
        if (hybrid) {
            for (uint32_t g = 0; g < n && n_binned < cap_binned; ++g) {
                const Proj& p = proj[g];
                if (!p.active) continue;
                const Rect rc = rect_of(p, cam);
                if (static_cast<uint64_t>(rc.w) * rc.h > 512u) {
                    gathered[g] = 1;
                    ++n_binned;
                }
            }
        }
#pragma omp parallel for schedule(dynamic, 256)
        for (int64_t gi = 0; gi < static_cast<int64_t>(n); ++gi) {
            const uint32_t g = static_cast<uint32_t>(gi);
            const Proj& p = proj[g];
            if (!p.active) continue;
            const Rect rc = rect_of(p, cam);
            const uint64_t key = pack(p.depth, g);
            const bool gather_form = hybrid && gathered[g];
            uint64_t f = 0, acc = 0;
            for (uint32_t yy = 0; yy < rc.h; ++yy) {
                for (uint32_t xx = 0; xx < rc.w; ++xx) {
                    const uint32_t px = rc.x0 + xx, py = rc.y0 + yy;
                    ++f;
                    const float alpha = st_alpha(p, static_cast<float>(px), static_cast<float>(py), gather_form);
                    if (alpha < kMinAlpha) continue;
                    const float u = slice ? st_blue(slice, rotation, g, px, py) : st_uniform(frame, g, px, py);
                    if (u >= alpha) continue;
                    ++acc;
                    atomic_min_u64(&fb[static_cast<size_t>(py) * cam.width_int + px], key);
                }
            }
            n_frag += f;
            n_acc += acc;
        }
    } else {
        const uint32_t cap = max_fragments
                                 ? max_fragments
                                 : static_cast<uint32_t>(std::nearbyint(cam.width * cam.height / (2.0f * cam.ss * cam.ss)));
        const int64_t n_warps = (n + 31) / 32;
        std::vector<uint8_t> binned(hybrid ? n : 0, 0);
        std::vector<GpsSource> bsrc(hybrid ? n : 0);
        std::vector<uint32_t> bcount(hybrid ? n : 0, 0);
        if (hybrid) {
            // binned set: Gaussians with more than 512 points, in index order up to max_binned
            for (uint32_t g = 0; g < n && n_binned < cap_binned; ++g) {
                const Proj& p = proj[g];
                if (!p.active) continue;
                const float dl = gps_dilog(p.opacity);
                Seed sd = gps_seed(g, frame);
                const uint32_t cnt = std::min(poisson_count(sd, kTwoPi * std::sqrt(p.det) * dl), cap);
                if (cnt > 512u) {
                    binned[g] = 1;
                    ++n_binned;
                }
            }
        }
        // one emulated warp of 32 consecutive Gaussians per iteration, each lane on its own stream
#pragma omp parallel for schedule(dynamic, 64)
        for (int64_t w = 0; w < n_warps; ++w) {
            GpsSource src[32];
            Seed seed[32];
            uint32_t count[32];
            bool act[32];
            uint64_t f = 0;
            for (uint32_t l = 0; l < 32; ++l) {
                const uint64_t gi = static_cast<uint64_t>(w) * 32 + l;
                const bool in_range = gi < n;
                const uint32_t g = in_range ? static_cast<uint32_t>(gi) : n - 1;
                const Proj& p = proj[g];
                act[l] = in_range && p.active;
                GpsSource& s = src[l];
                s.op_dilog = gps_dilog(p.opacity);
                seed[l] = gps_seed(g, frame);
                const uint32_t tc = poisson_count(seed[l], kTwoPi * std::sqrt(p.det) * s.op_dilog);
                if (tc == 0) act[l] = false;
                count[l] = std::min(tc, cap);
                const float c0 = std::sqrt(p.cov[0]), c1 = p.cov[1] / c0, c2 = std::sqrt(p.cov[2] - c1 * c1);
                s.mx = p.mx;
                s.my = p.my;
                s.conic[0] = p.conic[0];
                s.conic[1] = p.conic[1];
                s.conic[2] = p.conic[2];
                s.L[0] = c0;
                s.L[1] = c1;
                s.L[2] = c2;
                s.power = p.power;
                s.op_rcp = 1.0f / std::max(p.opacity, 1.0e-37f);
                s.key = pack(p.depth, g);
                if (hybrid && act[l] && binned[g]) {
                    bsrc[g] = s;
                    bcount[g] = count[l];
                    act[l] = false;
                }
            }
            for (uint32_t l = 0; l < 32; ++l)
                for (uint32_t i = 0; act[l] && i < count[l] && i < kSeq; ++i) {
                    gps_point(seed[l], src[l], cam, fb);
                    ++f;
                }
            for (uint32_t c = 0; c < 32; ++c) {
                if (!act[c] || count[c] <= kSeq) continue;
                const uint32_t iters = (count[c] - kSeq + 31) / 32;
                for (uint32_t it = 0; it < iters; ++it)
                    for (uint32_t l = 0; l < 32; ++l) {
                        if (it * 32 + l + kSeq >= count[c]) continue;
                        gps_point(seed[l], src[c], cam, fb);
                        ++f;
                    }
            }
            n_frag += f;
        }
        if (hybrid) {
            // binned points with counter-based seeds (accumulate_hybrid_gps.cu:162-166)
#pragma omp parallel for schedule(dynamic, 16)
            for (int64_t gi = 0; gi < static_cast<int64_t>(n); ++gi) {
                if (!binned[gi]) continue;
                const uint32_t g = static_cast<uint32_t>(gi);
                const Seed base = gps_seed(g, frame);
                for (uint32_t pt = 0; pt < bcount[g]; ++pt) {
                    Seed s = base;
                    s.x ^= pt * 0x9E3779B9u;
                    gps_point(s, bsrc[g], cam, fb);
                }
                n_frag += bcount[g];
            }
        }
    }
    if (stats) {
        stats->fragments = n_frag.load();
        stats->accepted = n_acc.load();
        stats->binned = n_binned;
    }
    return 0;
}

// sample_cu + resolve_cu (resolve.cu:27-349). `samples` (P_fb, 4) and `reuse` (P_fb, 4, or null
// without spatial reuse) are outputs; the k-buffer (K, P_fb, 2|4) is updated in place.
int oracle_sample_resolve(const float* means, const float* scales, const float* rotations, const float* opacities,
                          const float* sh, uint32_t n, uint32_t bases, const float* w2c, const float* cam_pos,
                          uint32_t width, uint32_t height, float fx, float fy, float cx, float cy, float near_plane,
                          float far_plane, int aa, int ss_raw, int spatial_reuse, const uint64_t* fb,
                          int32_t* k_prims, float* k_occl, const float* h_image, const float* h_depth,
                          const float* h_alpha, const float* h_wm, const float* v2pv, int mode, int threads,
                          float* samples, float* reuse, float* image, float* depth, float* alpha, float* wm) {
    (void)n;
    set_threads(threads);
    const Cam cam = make_cam(width, height, fx, fy, cx, cy, near_plane, far_plane, aa, ss_raw);
    const uint32_t ss = static_cast<uint32_t>(cam.ss);
    const uint32_t fbw = width * ss, fbh = height * ss;
    const int64_t n_fb = static_cast<int64_t>(fbw) * fbh;
    const int64_t n_px = static_cast<int64_t>(width) * height;
    constexpr float kMaxAlpha = 0.99f;

#pragma omp parallel for schedule(static)
    for (int64_t pix = 0; pix < n_fb; ++pix) {
        const uint64_t data = fb[pix];
        const uint32_t depth_key = static_cast<uint32_t>(data >> 32);
        const bool has = depth_key != 0xffffffffu;
        const uint32_t g = has ? static_cast<uint32_t>(data) : 0u;
        float s[4] = {0, 0, 0, 0};
        if (has) {
            const float vx = means[3 * g] - cam_pos[0], vy = means[3 * g + 1] - cam_pos[1],
                        vz = means[3 * g + 2] - cam_pos[2];
            const float inv = 1.0f / std::sqrt(vx * vx + vy * vy + vz * vz);
            eval_sh(sh + static_cast<size_t>(g) * bases * 3, vx * inv, vy * inv, vz * inv, bases, s);
            s[3] = bits_to_float(depth_key);
        }
        std::memcpy(samples + 4 * pix, s, sizeof(s));
        if (!spatial_reuse) continue;
        Proj p{};
        bool projected = has;
        if (projected) {
            p = project(means, scales, rotations, opacities, w2c, g, cam);
            projected = p.active;
        }
        float a = 1.0f, na[4] = {1, 1, 1, 1}, sdepth = INFINITY;
        if (projected) {
            const float dx = static_cast<float>(pix % fbw), dy = static_cast<float>(pix / fbw);
            auto ev = [&](float ox, float oy) {
                const float v = st_alpha(p, dx + ox, dy + oy, false);
                return v < kMinAlpha ? 0.0f : v;
            };
            a = std::max(ev(0, 0), kMinAlpha);
            na[0] = ev(-1, 0);
            na[1] = ev(1, 0);
            na[2] = ev(0, -1);
            na[3] = ev(0, 1);
            sdepth = s[3];
        }
        float w[4];
        for (int k = 0; k < 4; ++k) w[k] = (has && !projected) ? 0.0f : na[k] / a;
        bool unique = projected;
        int32_t pr[kK][2];
        float oc[kK][4];
        for (uint32_t k = 0; k < kK; ++k) {
            const int64_t e = static_cast<int64_t>(k) * n_fb + pix;
            pr[k][0] = k_prims[2 * e];
            pr[k][1] = k_prims[2 * e + 1];
            std::memcpy(oc[k], k_occl + 4 * e, sizeof(oc[k]));
            if (static_cast<uint32_t>(pr[k][0]) == g) unique = false;
            if (bits_to_float(static_cast<uint32_t>(pr[k][1])) < sdepth)
                for (int c = 0; c < 4; ++c) w[c] *= oc[k][c];
        }
        if (unique) {
            for (uint32_t k = kK - 1; k > 0; --k) {
                const int64_t e = static_cast<int64_t>(k) * n_fb + pix;
                k_prims[2 * e] = pr[k - 1][0];
                k_prims[2 * e + 1] = pr[k - 1][1];
                std::memcpy(k_occl + 4 * e, oc[k - 1], sizeof(oc[k - 1]));
            }
            k_prims[2 * pix] = static_cast<int32_t>(g);
            k_prims[2 * pix + 1] = static_cast<int32_t>(depth_key);
            const float den = 1.0f - std::min(a, kMaxAlpha);
            for (int c = 0; c < 4; ++c) k_occl[4 * pix + c] = (1.0f - std::min(na[c], kMaxAlpha)) / den;
        }
        std::memcpy(reuse + 4 * pix, w, sizeof(w));
    }

    const float norm = 1.0f / static_cast<float>(ss * ss);
#pragma omp parallel for schedule(static)
    for (int64_t pix = 0; pix < n_px; ++pix) {
        const uint32_t x = static_cast<uint32_t>(pix % width), y = static_cast<uint32_t>(pix / width);
        float cs[3] = {0, 0, 0}, ds = 0, as = 0, ws = 0, dout = 0;
        uint32_t valid = 0;
        for (uint32_t oy = 0; oy < ss; ++oy)
            for (uint32_t ox = 0; ox < ss; ++ox) {
                const uint32_t fx_ = x * ss + ox, fy_ = y * ss + oy;
                const int64_t fi = static_cast<int64_t>(fy_) * fbw + fx_;
                const float* s = samples + 4 * fi;
                if (s[3] > 0.0f) {
                    dout += s[3];
                    ++valid;
                }
                float csum[3] = {s[0], s[1], s[2]}, dsum = s[3], asum = s[3] > 0.0f ? 1.0f : 0.0f, wsum = 1.0f;
                auto add = [&](int64_t ni, float wt) {
                    const float* q = samples + 4 * ni;
                    for (int c = 0; c < 3; ++c) csum[c] += wt * q[c];
                    dsum += wt * q[3];
                    asum += q[3] > 0.0f ? wt : 0.0f;
                    wsum += wt;
                };
                if (spatial_reuse) {
                    if (fx_ > 0) add(fi - 1, reuse[4 * (fi - 1) + 1]);
                    if (fx_ < fbw - 1) add(fi + 1, reuse[4 * (fi + 1) + 0]);
                    if (fy_ > 0) add(fi - fbw, reuse[4 * (fi - fbw) + 3]);
                    if (fy_ < fbh - 1) add(fi + fbw, reuse[4 * (fi + fbw) + 2]);
                }
                const float r = 1.0f / wsum;
                for (int c = 0; c < 3; ++c) cs[c] += csum[c] * r;
                ds += dsum * r;
                as += asum * r;
                ws += wsum;
            }
        for (int c = 0; c < 3; ++c) cs[c] *= norm;
        ds *= norm;
        as *= norm;
        ws *= norm;
        float col[3] = {cs[0], cs[1], cs[2]}, d = ds, al = as, wmass = ws;
        if (mode == 1) {
            const float hm = h_wm[pix];
            wmass = hm + ws;
            const float hf = hm / wmass;
            for (int c = 0; c < 3; ++c) col[c] = cs[c] + hf * (h_image[3 * pix + c] - cs[c]);
            d = ds + hf * (h_depth[pix] - ds);
            al = as + hf * (h_alpha[pix] - as);
        } else if (mode == 2) {
            do {
                const float z = valid > 0 ? dout / static_cast<float>(valid) : far_plane;
                const float px = static_cast<float>(x) + 0.5f, py = static_cast<float>(y) + 0.5f;
                const float vx = (px - cx) / fx * z, vy = (py - cy) / fy * z, vz = z;
                const float* m1 = v2pv;
                const float* m2 = v2pv + 4;
                const float* m3 = v2pv + 8;
                const float pz = m3[0] * vx + m3[1] * vy + m3[2] * vz + m3[3];
                if (!(pz > 0.0f)) break;
                const float ppx = fx * (m1[0] * vx + m1[1] * vy + m1[2] * vz + m1[3]) / pz + cx;
                const float ppy = fy * (m2[0] * vx + m2[1] * vy + m2[2] * vz + m2[3]) / pz + cy;
                if (!(ppx >= 2.0f && ppx <= static_cast<float>(width) - 2.0f && ppy >= 2.0f &&
                      ppy <= static_cast<float>(height) - 2.0f))
                    break;
                auto cr = [](float t, float out[4]) {
                    const float t2 = t * t;
                    out[0] = t * (-0.5f + t * (1.0f - 0.5f * t));
                    out[1] = 1.0f + t2 * (-2.5f + 1.5f * t);
                    out[2] = t * (0.5f + t * (2.0f - 1.5f * t));
                    out[3] = t2 * (-0.5f + 0.5f * t);
                };
                const float tx = ppx - 0.5f, ty = ppy - 0.5f, bxf = std::floor(tx), byf = std::floor(ty);
                float wx[4], wy[4];
                cr(tx - bxf, wx);
                cr(ty - byf, wy);
                const uint32_t hx = static_cast<uint32_t>(bxf) - 1, hy = static_cast<uint32_t>(byf) - 1;
                float ch[3] = {0, 0, 0}, dh = 0, ah = 0;
                for (uint32_t j = 0; j < 4; ++j)
                    for (uint32_t i = 0; i < 4; ++i) {
                        const int64_t hi = static_cast<int64_t>(hy + j) * width + hx + i;
                        const float wt = wx[i] * wy[j];
                        for (int c = 0; c < 3; ++c) ch[c] += wt * h_image[3 * hi + c];
                        dh += wt * h_depth[hi];
                        ah += wt * h_alpha[hi];
                    }
                auto ycc = [](const float c[3], float o[3]) {
                    o[0] = 0.25f * c[0] + 0.5f * c[1] + 0.25f * c[2];
                    o[1] = 0.5f * c[0] - 0.5f * c[2];
                    o[2] = -0.25f * c[0] + 0.5f * c[1] - 0.25f * c[2];
                };
                float mean[3] = {0, 0, 0}, msq[3] = {0, 0, 0};
                for (int oy = -1; oy <= 1; ++oy)
                    for (int ox = -1; ox <= 1; ++ox) {
                        const int nx = std::clamp(static_cast<int>(x) + ox, 0, static_cast<int>(width) - 1);
                        const int ny = std::clamp(static_cast<int>(y) + oy, 0, static_cast<int>(height) - 1);
                        float nc[3] = {0, 0, 0};
                        for (uint32_t sy = 0; sy < ss; ++sy)
                            for (uint32_t sx = 0; sx < ss; ++sx) {
                                const float* q = samples + 4 * (static_cast<int64_t>(ny * ss + sy) * fbw + nx * ss + sx);
                                for (int c = 0; c < 3; ++c) nc[c] += q[c];
                            }
                        for (int c = 0; c < 3; ++c) nc[c] *= norm;
                        float yv[3];
                        ycc(nc, yv);
                        for (int c = 0; c < 3; ++c) {
                            mean[c] += yv[c];
                            msq[c] += yv[c] * yv[c];
                        }
                    }
                float sd[3];
                for (int c = 0; c < 3; ++c) {
                    mean[c] /= 9.0f;
                    msq[c] /= 9.0f;
                    sd[c] = std::sqrt(std::max(msq[c] - mean[c] * mean[c], 0.0f));
                }
                const float vel = std::sqrt((px - ppx) * (px - ppx) + (py - ppy) * (py - ppy));
                const float gamma = 4.0f + std::min(vel / 4.0f, 1.0f) * (1.0f - 4.0f);
                const float ext[3] = {std::max(gamma * sd[0], 0.01f), std::max(gamma * sd[1], 0.005f),
                                      std::max(gamma * sd[2], 0.005f)};
                float hy_[3];
                ycc(ch, hy_);
                float dist = 0.0f;
                for (int c = 0; c < 3; ++c) dist = std::max(dist, std::fabs(hy_[c] - mean[c]) / ext[c]);
                const float disc = dist > 1.0f ? 0.7f / dist : 0.7f;
                for (int c = 0; c < 3; ++c) col[c] = cs[c] + disc * (ch[c] - cs[c]);
                d = ds + disc * (dh - ds);
                al = as + disc * (ah - as);
                wmass = ws / (1.0f - disc);
            } while (false);
        }
        for (int c = 0; c < 3; ++c) image[3 * pix + c] = col[c];
        depth[pix] = d;
        alpha[pix] = al;
        wm[pix] = wmass;
    }
    return 0;
}

// Alpha of Gaussian g at (sub)pixel (px, py) in single precision (the accumulate evaluation) and in
// double precision from the same projected parameters: the tests use it to show that a winner
// mismatch sits on a decision boundary.
int oracle_fragment_alpha(const float* means, const float* scales, const float* rotations, const float* opacities,
                          uint32_t g, const float* w2c, uint32_t width, uint32_t height, float fx, float fy, float cx,
                          float cy, float near_plane, float far_plane, int aa, int ss, uint32_t px, uint32_t py,
                          float* alpha_f, double* alpha_d) {
    const Cam cam = make_cam(width, height, fx, fy, cx, cy, near_plane, far_plane, aa, ss);
    const Proj p = project(means, scales, rotations, opacities, w2c, g, cam);
    *alpha_f = st_alpha(p, static_cast<float>(px), static_cast<float>(py), false);
    const double dx = static_cast<double>(px) - (static_cast<double>(p.mx) - 0.5);
    const double dy = static_cast<double>(py) - (static_cast<double>(p.my) - 0.5);
    const double e = -0.5 * (p.conic[0] * dx * dx + p.conic[2] * dy * dy) - p.conic[1] * dx * dy;
    *alpha_d = p.opacity * std::exp(std::min(e, 0.0));
    return p.active ? 1 : 0;
}

}  // extern "C"
