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

// ---------------------------------------------------------------------------------------------
// Expected image of stochastic transparency and its exact gradient (double precision).
//
// For a (sub)pixel with fragments i in key order, the expected premultiplied colour, alpha and
// depth of one sample are C = sum c_i a_i T_i, A = sum a_i T_i, D = sum z_i a_i T_i with
// T_i = prod_{j before i} (1 - a_j). The fragment support (which Gaussian reaches which pixel with
// alpha >= 1/255) and the key order are frozen at a base point given in single precision (the
// forward of the render path); within them the image is a smooth function of the parameters, whose
// derivative is what a gradient estimator must reproduce on average. This is the checker of the
// backward pass: no reference counterpart exists (the reference has no backward).
// ---------------------------------------------------------------------------------------------
namespace {

struct ProjD {
    double t[3], x, y, xc, yc;
    bool free_x, free_y;
    double qn[4], qnorm;
    double R[3][3], v[3], S[3][3], T[2][3];
    double a, b, c, det, conic[3];
    double sig;             // sigmoid of the opacity logit
    double raw_xx, raw_yy;  // diagonal of the undilated 2-D covariance
    double det_raw, ratio;  // proper antialiasing: det of the undilated covariance, det_raw / det
    bool aa;
    double op, m2[2];       // op: the opacity alpha uses (sig, times sqrt(ratio) with antialiasing)
    double dvec[3], dlen, dir[3], color[3], Y[16];
    bool cpos[3];
};

constexpr double kC0 = 0.28209479177387814, kC1 = 0.48860251190291987, kC2a = 1.0925484305920792,
                 kC2b = 0.94617469575755997, kC2c = 0.31539156525251999, kC2d = 0.54627421529603959,
                 kC3a = 0.59004358992664352, kC3b = 1.7701307697799304, kC3c = 2.8906114426405538,
                 kC3d = 0.45704579946446572, kC3e = 2.2852289973223288, kC3f = 1.865881662950577,
                 kC3g = 1.1195289977703462, kC3h = 1.4453057213202769;

// signed SH basis of the reference's eval_sh (gs_utils.h:212-243) and its gradient w.r.t. the direction
void sh_basis(const double x, const double y, const double z, double Y[16], double dY[16][3]) {
    const double xx = x * x, yy = y * y, zz = z * z;
    double v[16] = {kC0, -kC1 * y, kC1 * z, -kC1 * x, kC2a * x * y, -kC2a * y * z, kC2b * zz - kC2c, -kC2a * x * z,
                    kC2d * (xx - yy), y * (kC3a * yy - kC3b * xx), kC3c * x * y * z, y * (kC3d - kC3e * zz),
                    z * (kC3f * zz - kC3g), x * (kC3d - kC3e * zz), kC3h * z * (xx - yy), x * (kC3b * yy - kC3a * xx)};
    double g[16][3] = {{0, 0, 0}, {0, -kC1, 0}, {0, 0, kC1}, {-kC1, 0, 0},
                       {kC2a * y, kC2a * x, 0}, {0, -kC2a * z, -kC2a * y}, {0, 0, 2 * kC2b * z},
                       {-kC2a * z, 0, -kC2a * x}, {2 * kC2d * x, -2 * kC2d * y, 0},
                       {-2 * kC3b * x * y, 3 * kC3a * yy - kC3b * xx, 0}, {kC3c * y * z, kC3c * x * z, kC3c * x * y},
                       {0, kC3d - kC3e * zz, -2 * kC3e * y * z}, {0, 0, 3 * kC3f * zz - kC3g},
                       {kC3d - kC3e * zz, 0, -2 * kC3e * x * z}, {2 * kC3h * x * z, -2 * kC3h * y * z, kC3h * (xx - yy)},
                       {kC3b * yy - 3 * kC3a * xx, 2 * kC3b * x * y, 0}};
    std::memcpy(Y, v, sizeof(v));
    std::memcpy(dY, g, sizeof(g));
}

ProjD project_d(const double* m, const double* s, const double* q, const double o, const double* sh, uint32_t bases,
                const double* W, const double* cam, const double fx, const double fy, const double cx0,
                const double cy0, const double width, const double height, const double dil, const bool aa) {
    ProjD p{};
    for (int r = 0; r < 3; ++r) p.t[r] = W[4 * r] * m[0] + W[4 * r + 1] * m[1] + W[4 * r + 2] * m[2] + W[4 * r + 3];
    p.x = p.t[0] / p.t[2];
    p.y = p.t[1] / p.t[2];
    const double cl = (-0.15 * width - cx0) / fx, cr = (1.15 * width - cx0) / fx;
    const double ct = (-0.15 * height - cy0) / fy, cb = (1.15 * height - cy0) / fy;
    p.xc = std::min(std::max(p.x, cl), cr);
    p.yc = std::min(std::max(p.y, ct), cb);
    p.free_x = p.x > cl && p.x < cr;
    p.free_y = p.y > ct && p.y < cb;
    p.qnorm = std::sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
    for (int i = 0; i < 4; ++i) p.qn[i] = q[i] / p.qnorm;
    const double w = p.qn[0], X = p.qn[1], Yq = p.qn[2], Z = p.qn[3];
    const double R[3][3] = {{1 - 2 * (Yq * Yq + Z * Z), 2 * (X * Yq - w * Z), 2 * (X * Z + w * Yq)},
                            {2 * (X * Yq + w * Z), 1 - 2 * (X * X + Z * Z), 2 * (Yq * Z - w * X)},
                            {2 * (X * Z - w * Yq), 2 * (Yq * Z + w * X), 1 - 2 * (X * X + Yq * Yq)}};
    std::memcpy(p.R, R, sizeof(R));
    for (int i = 0; i < 3; ++i) p.v[i] = std::exp(2.0 * s[i]);
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            double acc = 0;
            for (int k = 0; k < 3; ++k) acc += R[i][k] * p.v[k] * R[j][k];
            p.S[i][j] = acc;
        }
    const double J[2][3] = {{fx / p.t[2], 0, -fx * p.xc / p.t[2]}, {0, fy / p.t[2], -fy * p.yc / p.t[2]}};
    for (int i = 0; i < 2; ++i)
        for (int j = 0; j < 3; ++j) {
            double acc = 0;
            for (int k = 0; k < 3; ++k) acc += J[i][k] * W[4 * k + j];
            p.T[i][j] = acc;
        }
    double cov[2][2];
    for (int i = 0; i < 2; ++i)
        for (int j = 0; j < 2; ++j) {
            double acc = 0;
            for (int k = 0; k < 3; ++k)
                for (int l = 0; l < 3; ++l) acc += p.T[i][k] * p.S[k][l] * p.T[j][l];
            cov[i][j] = acc;
        }
    p.a = cov[0][0] + dil;
    p.b = cov[0][1];
    p.c = cov[1][1] + dil;
    p.det = p.a * p.c - p.b * p.b;
    p.conic[0] = p.c / p.det;
    p.conic[1] = -p.b / p.det;
    p.conic[2] = p.a / p.det;
    p.sig = 1.0 / (1.0 + std::exp(-o));
    // proper antialiasing keeps the integral of the dilated footprint: opacity * sqrt(det / det dilated)
    // (gs_utils.h:155,165-166)
    p.aa = aa;
    p.raw_xx = cov[0][0];
    p.raw_yy = cov[1][1];
    p.det_raw = cov[0][0] * cov[1][1] - cov[0][1] * cov[0][1];
    p.ratio = p.det_raw / p.det;
    p.op = aa ? p.sig * std::sqrt(std::max(p.ratio, 0.0)) : p.sig;
    p.m2[0] = p.x * fx + cx0;
    p.m2[1] = p.y * fy + cy0;
    for (int i = 0; i < 3; ++i) p.dvec[i] = m[i] - cam[i];
    p.dlen = std::sqrt(p.dvec[0] * p.dvec[0] + p.dvec[1] * p.dvec[1] + p.dvec[2] * p.dvec[2]);
    for (int i = 0; i < 3; ++i) p.dir[i] = p.dvec[i] / p.dlen;
    double dY[16][3];
    sh_basis(p.dir[0], p.dir[1], p.dir[2], p.Y, dY);
    for (int ch = 0; ch < 3; ++ch) {
        double col = 0.5;
        for (uint32_t bb = 0; bb < bases; ++bb) col += p.Y[bb] * sh[3 * bb + ch];
        p.cpos[ch] = col > 0.0;
        p.color[ch] = std::max(col, 0.0);
    }
    return p;
}

// upstream gradients of one Gaussian's projected quantities
struct GradProj {
    double op, conic[3], m2[2], depth, color[3];
};

// chain rule from the projected quantities to the parameters (mean, log-scale, quaternion, logit, SH)
void project_d_backward(const ProjD& p, const GradProj& g, const double* sh, uint32_t bases, const double* W,
                        const double fx, const double fy, double* dm, double* ds, double* dq, double* dopac,
                        double* dsh) {
    const double f = p.aa ? std::sqrt(std::max(p.ratio, 0.0)) : 1.0;
    *dopac = g.op * f * p.sig * (1.0 - p.sig);
    // conic = inverse(cov2d + dilation): dL/dcov = -C G C
    const double C[2][2] = {{p.conic[0], p.conic[1]}, {p.conic[1], p.conic[2]}};
    const double G[2][2] = {{g.conic[0], 0.5 * g.conic[1]}, {0.5 * g.conic[1], g.conic[2]}};
    double CG[2][2], GA[2][2];
    for (int i = 0; i < 2; ++i)
        for (int j = 0; j < 2; ++j) CG[i][j] = C[i][0] * G[0][j] + C[i][1] * G[1][j];
    for (int i = 0; i < 2; ++i)
        for (int j = 0; j < 2; ++j) GA[i][j] = -(CG[i][0] * C[0][j] + CG[i][1] * C[1][j]);
    if (p.aa && p.ratio > 0.0) {
        // op = sig sqrt(r), r = det_raw / det with det_raw = xx yy - xy^2 and det = (xx + d)(yy + d) - xy^2
        // dL/dr = g.op sig / (2 sqrt(r)); dr/dxx = (yy det - det_raw (yy + d)) / det^2, likewise for yy,
        // dr/dxy = 2 xy (det_raw - det) / det^2, split over the two off-diagonal entries
        const double k = g.op * p.sig / (2.0 * f) / (p.det * p.det);
        GA[0][0] += k * (p.raw_yy * p.det - p.det_raw * p.c);
        GA[1][1] += k * (p.raw_xx * p.det - p.det_raw * p.a);
        GA[0][1] += k * (p.b * (p.det_raw - p.det));
        GA[1][0] += k * (p.b * (p.det_raw - p.det));
    }
    // G_cov symmetric with off-diagonal dL/db / 2 = GA[0][1]
    double dS[3][3], dT[2][3];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            double acc = 0;
            for (int k = 0; k < 2; ++k)
                for (int l = 0; l < 2; ++l) acc += p.T[k][i] * GA[k][l] * p.T[l][j];
            dS[i][j] = acc;
        }
    for (int i = 0; i < 2; ++i)
        for (int j = 0; j < 3; ++j) {
            double acc = 0;
            for (int k = 0; k < 2; ++k)
                for (int l = 0; l < 3; ++l) acc += GA[i][k] * p.T[k][l] * p.S[l][j];
            dT[i][j] = 2.0 * acc;
        }
    // T = J W3
    double dJ[2][3];
    for (int i = 0; i < 2; ++i)
        for (int j = 0; j < 3; ++j) {
            double acc = 0;
            for (int k = 0; k < 3; ++k) acc += dT[i][k] * W[4 * j + k];
            dJ[i][j] = acc;
        }
    const double tz = p.t[2];
    double dtx = 0, dty = 0, dtz = g.depth;
    dtz += dJ[0][0] * (-fx / (tz * tz)) + dJ[0][2] * (fx * p.xc / (tz * tz)) + dJ[1][1] * (-fy / (tz * tz)) +
           dJ[1][2] * (fy * p.yc / (tz * tz));
    double dx = g.m2[0] * fx, dy = g.m2[1] * fy;
    if (p.free_x) dx += dJ[0][2] * (-fx / tz);
    if (p.free_y) dy += dJ[1][2] * (-fy / tz);
    dtx += dx / tz;
    dty += dy / tz;
    dtz -= dx * p.t[0] / (tz * tz) + dy * p.t[1] / (tz * tz);
    for (int i = 0; i < 3; ++i) dm[i] = W[i] * dtx + W[4 + i] * dty + W[8 + i] * dtz;
    // Sigma = R V R^T
    for (int i = 0; i < 3; ++i) {
        double acc = 0;
        for (int k = 0; k < 3; ++k)
            for (int l = 0; l < 3; ++l) acc += p.R[k][i] * dS[k][l] * p.R[l][i];
        ds[i] = acc * 2.0 * p.v[i];
    }
    double dR[3][3];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            double acc = 0;
            for (int k = 0; k < 3; ++k) acc += (dS[i][k] + dS[k][i]) * p.R[k][j];
            dR[i][j] = acc * p.v[j];
        }
    const double w = p.qn[0], X = p.qn[1], Y = p.qn[2], Z = p.qn[3];
    double dqn[4];
    dqn[0] = 2 * (-Z * dR[0][1] + Y * dR[0][2] + Z * dR[1][0] - X * dR[1][2] - Y * dR[2][0] + X * dR[2][1]);
    dqn[1] = 2 * (Y * dR[0][1] + Z * dR[0][2] + Y * dR[1][0] - 2 * X * dR[1][1] - w * dR[1][2] + Z * dR[2][0] +
                  w * dR[2][1] - 2 * X * dR[2][2]);
    dqn[2] = 2 * (-2 * Y * dR[0][0] + X * dR[0][1] + w * dR[0][2] + X * dR[1][0] + Z * dR[1][2] - w * dR[2][0] +
                  Z * dR[2][1] - 2 * Y * dR[2][2]);
    dqn[3] = 2 * (-2 * Z * dR[0][0] - w * dR[0][1] + X * dR[0][2] + w * dR[1][0] - 2 * Z * dR[1][1] + Y * dR[1][2] +
                  X * dR[2][0] + Y * dR[2][1]);
    const double dot = dqn[0] * w + dqn[1] * X + dqn[2] * Y + dqn[3] * Z;
    for (int i = 0; i < 4; ++i) dq[i] = (dqn[i] - p.qn[i] * dot) / p.qnorm;
    // colour = max(0.5 + sum Y_b sh_b, 0) per channel; direction = normalize(mean - camera)
    double Yb[16], dY[16][3];
    sh_basis(p.dir[0], p.dir[1], p.dir[2], Yb, dY);
    double ddir[3] = {0, 0, 0};
    for (int ch = 0; ch < 3; ++ch) {
        const double gc = p.cpos[ch] ? g.color[ch] : 0.0;
        for (uint32_t bb = 0; bb < bases; ++bb) {
            dsh[3 * bb + ch] = gc * Yb[bb];
            for (int k = 0; k < 3; ++k) ddir[k] += gc * sh[3 * bb + ch] * dY[bb][k];
        }
    }
    const double dd = ddir[0] * p.dir[0] + ddir[1] * p.dir[1] + ddir[2] * p.dir[2];
    for (int k = 0; k < 3; ++k) dm[k] += (ddir[k] - p.dir[k] * dd) / p.dlen;
}

// ---- Gaussian point splatting: the probability that a Gaussian puts a point into a pixel ----------
//
// A Gaussian with projected opacity o, dilated 2-D covariance Sigma and mean m draws N points with
// N = rint(max(kf(w), 0)), w standard normal and kf the Cornish-Fisher expansion of a Poisson
// quantile (math_utils.h:98-111) at lambda = 2 pi sqrt(det Sigma) Li2(o) (accumulate_scatter.cu:
// 104-112). The points are independent with density -ln(1 - o G(x)) / lambda, G(x) =
// exp(-(x - m)^T Sigma^-1 (x - m) / 2): truncated_box_muller draws o G with P(o G <= t) =
// Li2(t) / Li2(o) (math_utils.h:14-43 approximate Li2 and its inverse). A point in the square of
// (sub)pixel p registers when p's centre passes the power test, so p is hit with probability
//   h = 1 - E[(1 - q)^N],  q = Lambda_p / lambda,  Lambda_p = integral over p of -ln(1 - o G),
// independently of every other Gaussian (for a Poisson N, h = 1 - exp(-Lambda_p)). The expected
// image is the stochastic-transparency one with alpha replaced by h.

double li2(const double x) {
    if (x <= 0.0) return 0.0;
    if (x >= 1.0) return 1.6449340668482264;
    if (x > 0.5) return 1.6449340668482264 - std::log(x) * std::log1p(-x) - li2(1.0 - x);
    double term = x, sum = 0.0;
    for (int k = 1; k < 200 && term > 1e-18; ++k, term *= x) sum += term / (static_cast<double>(k) * k);
    return sum;
}

// kf(w) of the count draw, and its partial derivatives in w and lambda
double cf_kf(const double w, const double lam) {
    const double s = std::sqrt(lam), w2 = w * w;
    return lam + s * w + (w2 - 1.0) / 6.0 + (-(w / 36.0) - w2 * w / 72.0) / s +
           (-(8.0 / 405.0) + (7.0 / 810.0) * w2 + w2 * w2 / 270.0) / lam;
}
double cf_kf_w(const double w, const double lam) {
    const double s = std::sqrt(lam), w2 = w * w;
    return s + w / 3.0 + (-(1.0 / 36.0) - w2 / 24.0) / s + ((14.0 / 810.0) * w + (4.0 / 270.0) * w2 * w) / lam;
}
double cf_kf_lam(const double w, const double lam) {
    const double s = std::sqrt(lam), w2 = w * w;
    return 1.0 + w / (2.0 * s) - 0.5 * (-(w / 36.0) - w2 * w / 72.0) / (lam * s) -
           (-(8.0 / 405.0) + (7.0 / 810.0) * w2 + w2 * w2 / 270.0) / (lam * lam);
}

double normal_cdf(const double x) { return 0.5 * std::erfc(-x / std::sqrt(2.0)); }
double normal_pdf(const double x) { return std::exp(-0.5 * x * x) / std::sqrt(2.0 * 3.14159265358979323846); }

// Law of the point count: P[n] = P(N = n) and dP[n] = dP(N = n) / dlambda, n = 0 .. until the rest
// is below 1e-15. F(t) = P(kf(w) < t) is a sum over the monotone pieces of the quartic kf on
// [-12, 12] (outside, kf exceeds every threshold used); its lambda-derivative is
// -sum over the roots r of kf = t of phi(r) (dkf/dlambda)(r) / |dkf/dw(r)|.
struct CountLaw {
    std::vector<double> P, dP;
};

CountLaw cf_count_law(const double lam) {
    constexpr double kW = 12.0;
    constexpr int kGrid = 4800;
    std::vector<double> cut{-kW};
    double prev = cf_kf_w(-kW, lam);
    for (int i = 1; i <= kGrid; ++i) {
        const double w = -kW + 2.0 * kW * i / kGrid;
        const double cur = cf_kf_w(w, lam);
        if ((prev < 0.0) != (cur < 0.0) && i < kGrid) {
            double lo = w - 2.0 * kW / kGrid, hi = w;
            for (int it = 0; it < 200 && hi - lo > 1e-15; ++it) {
                const double mid = 0.5 * (lo + hi);
                if ((cf_kf_w(mid, lam) < 0.0) == (cf_kf_w(lo, lam) < 0.0)) lo = mid;
                else hi = mid;
            }
            cut.push_back(0.5 * (lo + hi));
        }
        prev = cur;
    }
    cut.push_back(kW);
    double top = 0.0;
    for (const double c : cut) top = std::max(top, cf_kf(c, lam));
    // F(t) and dF/dlambda at threshold t
    auto F = [&](const double t, double& dF) {
        double f = 0.0;
        dF = 0.0;
        for (size_t i = 0; i + 1 < cut.size(); ++i) {
            const double a = cut[i], b = cut[i + 1], fa = cf_kf(a, lam), fb = cf_kf(b, lam);
            const bool up = fb >= fa;
            const double lo_v = up ? fa : fb, hi_v = up ? fb : fa;
            if (t <= lo_v) continue;
            if (t >= hi_v) {
                f += normal_cdf(b) - normal_cdf(a);
                continue;
            }
            double lo = a, hi = b;
            for (int it = 0; it < 200 && hi - lo > 1e-15; ++it) {
                const double mid = 0.5 * (lo + hi);
                if ((cf_kf(mid, lam) < t) == up) lo = mid;
                else hi = mid;
            }
            const double r = 0.5 * (lo + hi);
            f += up ? normal_cdf(r) - normal_cdf(a) : normal_cdf(b) - normal_cdf(r);
            const double slope = std::fabs(cf_kf_w(r, lam));
            if (slope > 0.0) dF -= normal_pdf(r) * cf_kf_lam(r, lam) / slope;
        }
        return f;
    };
    CountLaw law;
    double f_prev = 0.0, d_prev = 0.0;
    for (int n = 0;; ++n) {
        double d;
        const double f = F(n + 0.5, d);
        law.P.push_back(f - f_prev);
        law.dP.push_back(d - d_prev);
        f_prev = f;
        d_prev = d;
        if (1.0 - f < 1e-15 || n + 0.5 > top) break;
    }
    return law;
}

// Gauss-Legendre nodes and weights of order n on [0, 1] (Newton on the Legendre recurrence).
void gauss_legendre01(const int n, std::vector<double>& x, std::vector<double>& w) {
    x.assign(n, 0.0);
    w.assign(n, 0.0);
    for (int i = 0; i < n; ++i) {
        double z = std::cos(3.14159265358979323846 * (i + 0.75) / (n + 0.5)), dp = 0.0;
        for (int it = 0; it < 100; ++it) {
            double p0 = 1.0, p1 = 0.0;
            for (int j = 1; j <= n; ++j) {
                const double p2 = p1;
                p1 = p0;
                p0 = ((2.0 * j - 1.0) * z * p1 - (j - 1.0) * p2) / j;
            }
            dp = n * (z * p0 - p1) / (z * z - 1.0);
            const double dz = p0 / dp;
            z -= dz;
            if (std::fabs(dz) < 1e-16) break;
        }
        x[i] = 0.5 * (1.0 - z);
        w[i] = 1.0 / ((1.0 - z * z) * dp * dp);
    }
}

// Probability of one fragment (ST alpha or GPS hit probability) and its partial derivatives in the
// projected opacity, the conic (x, y, z) and the 2-D mean.
struct FragP {
    double p, d_op, d_conic[3], d_m2[2];
};

FragP st_fragment(const ProjD& p, const double px, const double py) {
    const double dx = px - (p.m2[0] - 0.5), dy = py - (p.m2[1] - 0.5);
    const double e = -0.5 * (p.conic[0] * dx * dx + p.conic[2] * dy * dy) - p.conic[1] * dx * dy;
    const double a = p.op * std::exp(std::min(e, 0.0));
    FragP f;
    f.p = a;
    f.d_op = a / p.op;
    f.d_conic[0] = a * (-0.5 * dx * dx);
    f.d_conic[1] = a * (-dx * dy);
    f.d_conic[2] = a * (-0.5 * dy * dy);
    f.d_m2[0] = a * (p.conic[0] * dx + p.conic[1] * dy);
    f.d_m2[1] = a * (p.conic[1] * dx + p.conic[2] * dy);
    return f;
}

// Per-Gaussian constants of the GPS hit probability: lambda, its derivatives in (op, conic x/y/z)
// and the law of the count (above kPoissonLambda the count is taken as Poisson, which the
// Cornish-Fisher draw matches to about 1e-5 there). With a point cap c (the render draws
// min(N, c) points, accumulate_scatter.cu:129-131), the law is truncated at c and P(N >= c) folded
// into the term of c: Q = sum_{n < c} P(N = n) Z^n + P(N >= c) Z^c.
struct GpsLaw {
    double lam, d_lam[4];
    bool poisson;
    CountLaw law;
};
constexpr double kOraclePoissonLambda = 32.0;

// Poisson law of n < cap with the rest folded into the term of cap, and its lambda-derivative
// (d pmf(n) / d lambda = pmf(n - 1) - pmf(n); the folded rest's is pmf(cap - 1)).
CountLaw poisson_law_capped(const double lam, const uint32_t cap) {
    CountLaw law;
    law.P.resize(cap + 1);
    law.dP.resize(cap + 1);
    double prev = 0.0, sum = 0.0;
    for (uint32_t n = 0; n < cap; ++n) {
        const double pmf = std::exp(n * std::log(lam) - lam - std::lgamma(n + 1.0));
        law.P[n] = pmf;
        law.dP[n] = prev - pmf;
        sum += pmf;
        prev = pmf;
    }
    law.P[cap] = std::max(1.0 - sum, 0.0);
    law.dP[cap] = prev;
    return law;
}

GpsLaw gps_law(const ProjD& p, const uint32_t cap) {
    GpsLaw g;
    const double two_pi = 2.0 * 3.14159265358979323846;
    const double sd = std::sqrt(p.det);
    g.lam = two_pi * sd * li2(p.op);
    const double D = p.conic[0] * p.conic[2] - p.conic[1] * p.conic[1];  // 1 / det
    g.d_lam[0] = two_pi * sd * (-std::log1p(-std::min(p.op, 1.0 - 1e-16)) / p.op);
    g.d_lam[1] = g.lam * (-0.5) * p.conic[2] / D;
    g.d_lam[2] = g.lam * p.conic[1] / D;
    g.d_lam[3] = g.lam * (-0.5) * p.conic[0] / D;
    g.poisson = g.lam >= kOraclePoissonLambda;
    if (!g.poisson) {
        g.law = cf_count_law(g.lam);
        if (cap > 0 && cap < g.law.P.size()) {
            double rest = 0.0, d_rest = 0.0;
            for (size_t n = cap; n < g.law.P.size(); ++n) {
                rest += g.law.P[n];
                d_rest += g.law.dP[n];
            }
            g.law.P.resize(cap + 1);
            g.law.dP.resize(cap + 1);
            g.law.P[cap] = rest;
            g.law.dP[cap] = d_rest;
        }
    } else if (cap > 0 && g.lam + 12.0 * std::sqrt(g.lam) >= cap) {
        g.poisson = false;  // the cap binds: the capped Poisson law through the general form
        g.law = poisson_law_capped(g.lam, cap);
    }
    return g;
}

// GPS hit probability of the pixel square [px, px + 1) x [py, py + 1): Lambda_p by an order-`quad`
// Gauss-Legendre rule per axis, then h and the chain through Lambda_p and lambda.
FragP gps_fragment(const ProjD& p, const GpsLaw& g, const double px, const double py, const std::vector<double>& qx,
                   const std::vector<double>& qw) {
    double Lp = 0.0, dL_op = 0.0, dL_c[3] = {0, 0, 0}, dL_m[2] = {0, 0};
    for (size_t i = 0; i < qx.size(); ++i)
        for (size_t j = 0; j < qx.size(); ++j) {
            const double W = qw[i] * qw[j];
            const double dx = px + qx[i] - p.m2[0], dy = py + qx[j] - p.m2[1];
            const double G = std::exp(-0.5 * (p.conic[0] * dx * dx + p.conic[2] * dy * dy) - p.conic[1] * dx * dy);
            const double oG = p.op * G;
            Lp += W * -std::log1p(-oG);
            const double w = W * oG / (1.0 - oG);
            dL_op += w / p.op;
            dL_c[0] += w * (-0.5 * dx * dx);
            dL_c[1] += w * (-dx * dy);
            dL_c[2] += w * (-0.5 * dy * dy);
            dL_m[0] += w * (p.conic[0] * dx + p.conic[1] * dy);
            dL_m[1] += w * (p.conic[1] * dx + p.conic[2] * dy);
        }
    double h, dh_dL, dh_dlam;
    if (g.poisson) {
        h = -std::expm1(-Lp);
        dh_dL = std::exp(-Lp);
        dh_dlam = 0.0;
    } else {
        const double Z = 1.0 - Lp / g.lam;
        double Q = 0.0, dQ_dZ = 0.0, dQ_dlam = 0.0, Zn = 1.0;
        for (size_t n = 0; n < g.law.P.size(); ++n) {
            Q += g.law.P[n] * Zn;
            dQ_dlam += g.law.dP[n] * Zn;
            if (n + 1 < g.law.P.size()) dQ_dZ += (n + 1) * g.law.P[n + 1] * Zn;
            Zn *= Z;
        }
        h = 1.0 - Q;
        dh_dL = dQ_dZ / g.lam;
        dh_dlam = -dQ_dZ * Lp / (g.lam * g.lam) - dQ_dlam;
    }
    FragP f;
    f.p = h;
    f.d_op = dh_dL * dL_op + dh_dlam * g.d_lam[0];
    for (int c = 0; c < 3; ++c) f.d_conic[c] = dh_dL * dL_c[c] + dh_dlam * g.d_lam[1 + c];
    f.d_m2[0] = dh_dL * dL_m[0];
    f.d_m2[1] = dh_dL * dL_m[1];
    return f;
}

}  // namespace

extern "C" {

// Law of the GPS point count at lambda (tests): writes up to `cap` probabilities P(N = n) and their
// lambda-derivatives, returns how many the law has (may exceed cap).
int oracle_gps_count_law(const double lambda, double* P, double* dP, const int cap) {
    const CountLaw law = cf_count_law(lambda);
    for (int n = 0; n < cap && n < static_cast<int>(law.P.size()); ++n) {
        P[n] = law.P[n];
        dP[n] = law.dP[n];
    }
    return static_cast<int>(law.P.size());
}

// Expected image (H, W, 3 / 1 / 1) of one stochastic-transparency sample, image resolution (the
// ss x ss box filter applied), and the gradient of L = sum(g_image * image + g_alpha * alpha +
// g_depth * depth) w.r.t. every parameter. Support and key order come from the single-precision
// projection of the `base_*` parameters; `d_*` may be null for the forward only.
int oracle_expected_image(const double* means, const double* scales, const double* rotations, const double* opacities,
                          const double* sh, uint32_t n, uint32_t bases, const double* w2c, const double* cam_pos,
                          uint32_t width, uint32_t height, double fx, double fy, double cx, double cy, double near_plane,
                          double far_plane, int ss_raw, int aa, const float* base_means, const float* base_scales,
                          const float* base_rotations, const float* base_opacities, const double* g_image,
                          const double* g_alpha, const double* g_depth, double* image, double* alpha, double* depth,
                          double* loss, double* d_means, double* d_scales, double* d_rotations, double* d_opacities,
                          double* d_sh);

// The same for Gaussian point splatting: each fragment's alpha is replaced by the probability that
// the Gaussian puts a point into the (sub)pixel (see gps_fragment), with the pixel integrals taken
// by an order-`quad` Gauss-Legendre rule per axis. The support is the pixels whose centre passes the
// power test at the base point, as in the render (scatter_utils.cuh:116-129). `max_fragments`: the
// point cap (0: the render's default, width x height / (2 ss^2) framebuffer pixels; < 0: none).
int oracle_expected_image_gps(const double* means, const double* scales, const double* rotations,
                              const double* opacities, const double* sh, uint32_t n, uint32_t bases, const double* w2c,
                              const double* cam_pos, uint32_t width, uint32_t height, double fx, double fy, double cx,
                              double cy, double near_plane, double far_plane, int ss_raw, int aa,
                              const float* base_means, const float* base_scales, const float* base_rotations,
                              const float* base_opacities, const double* g_image, const double* g_alpha,
                              const double* g_depth, double* image, double* alpha, double* depth, double* loss,
                              double* d_means, double* d_scales, double* d_rotations, double* d_opacities,
                              double* d_sh, int quad, int max_fragments);

}  // extern "C"

namespace {

int expected_image_impl(const double* means, const double* scales, const double* rotations, const double* opacities,
                        const double* sh, uint32_t n, uint32_t bases, const double* w2c, const double* cam_pos,
                        uint32_t width, uint32_t height, double fx, double fy, double cx, double cy, double near_plane,
                        double far_plane, int ss_raw, int aa, const float* base_means, const float* base_scales,
                        const float* base_rotations, const float* base_opacities, const double* g_image,
                        const double* g_alpha, const double* g_depth, double* image, double* alpha, double* depth,
                        double* loss, double* d_means, double* d_scales, double* d_rotations, double* d_opacities,
                        double* d_sh, const bool gps, const int quad, const int cap_arg) {
    const uint32_t ss = ss_raw < 1 ? 1u : static_cast<uint32_t>(ss_raw);
    float w2cf[12];
    for (int i = 0; i < 12; ++i) w2cf[i] = static_cast<float>(w2c[i]);
    const Cam cam = make_cam(width, height, static_cast<float>(fx), static_cast<float>(fy), static_cast<float>(cx),
                             static_cast<float>(cy), static_cast<float>(near_plane), static_cast<float>(far_plane), aa,
                             static_cast<int>(ss));
    const uint32_t fbw = width * ss, fbh = height * ss;
    const double dfx = fx * ss, dfy = fy * ss, dcx = cx * ss, dcy = cy * ss;
    const double dil = (aa ? kDilationAA : kDilation) * ss * ss;
    // frozen support and order from the single-precision forward
    std::vector<std::vector<std::pair<uint64_t, uint32_t>>> frags(static_cast<size_t>(fbw) * fbh);
    for (uint32_t g = 0; g < n; ++g) {
        const Proj p = project(base_means, base_scales, base_rotations, base_opacities, w2cf, g, cam);
        if (!p.active) continue;
        const Rect rc = rect_of(p, cam);
        const uint64_t key = pack(p.depth, g);
        for (uint32_t yy = 0; yy < rc.h; ++yy)
            for (uint32_t xx = 0; xx < rc.w; ++xx) {
                const uint32_t px = rc.x0 + xx, py = rc.y0 + yy;
                if (gps) {
                    const float dcx = static_cast<float>(px) + 0.5f - p.mx, dcy = static_cast<float>(py) + 0.5f - p.my;
                    const float power =
                        0.5f * (p.conic[0] * dcx * dcx + p.conic[2] * dcy * dcy) + p.conic[1] * dcx * dcy;
                    if (power > p.power) continue;
                } else if (st_alpha(p, static_cast<float>(px), static_cast<float>(py), false) < kMinAlpha) {
                    continue;
                }
                frags[static_cast<size_t>(py) * fbw + px].push_back({key, g});
            }
    }
    std::vector<ProjD> pd(n);
    for (uint32_t g = 0; g < n; ++g)
        pd[g] = project_d(means + 3 * g, scales + 3 * g, rotations + 4 * g, opacities[g], sh + static_cast<size_t>(g) * bases * 3,
                          bases, w2c, cam_pos, dfx, dfy, dcx, dcy, static_cast<double>(fbw), static_cast<double>(fbh), dil,
                          aa != 0);
    std::vector<GpsLaw> laws(gps ? n : 0);
    // the render's point cap: width x height / (2 ss^2) framebuffer pixels unless given; < 0: none
    const uint32_t cap = cap_arg < 0 ? 0u
                         : cap_arg > 0 ? static_cast<uint32_t>(cap_arg)
                                       : static_cast<uint32_t>(std::nearbyint(static_cast<float>(fbw) * static_cast<float>(fbh) /
                                                                              (2.0f * ss * ss)));
    for (uint32_t g = 0; g < n && gps; ++g) laws[g] = gps_law(pd[g], cap);
    std::vector<double> qx, qw;
    if (gps) gauss_legendre01(std::max(quad, 1), qx, qw);
    const bool grad = d_means != nullptr;
    std::vector<GradProj> gp(grad ? n : 0);
    for (auto& x : gp) x = GradProj{};
    const double norm = 1.0 / (ss * ss);
    const size_t n_px = static_cast<size_t>(width) * height;
    std::fill(image, image + 3 * n_px, 0.0);
    std::fill(alpha, alpha + n_px, 0.0);
    std::fill(depth, depth + n_px, 0.0);
    double L = 0.0;
    std::vector<double> al;
    std::vector<FragP> fp;
    for (uint32_t py = 0; py < fbh; ++py)
        for (uint32_t px = 0; px < fbw; ++px) {
            auto& f = frags[static_cast<size_t>(py) * fbw + px];
            std::sort(f.begin(), f.end());
            const size_t ip = static_cast<size_t>(py / ss) * width + px / ss;
            const size_t m = f.size();
            al.assign(m, 0.0);
            fp.resize(m);
            std::vector<double> T(m + 1, 1.0);
            for (size_t k = 0; k < m; ++k) {
                const uint32_t g = f[k].second;
                fp[k] = gps ? gps_fragment(pd[g], laws[g], px, py, qx, qw) : st_fragment(pd[g], px, py);
                al[k] = fp[k].p;
                T[k + 1] = T[k] * (1.0 - al[k]);
            }
            double Cc[3] = {0, 0, 0}, Aa = 0, Dd = 0;
            for (size_t k = 0; k < m; ++k) {
                const ProjD& p = pd[f[k].second];
                const double wgt = al[k] * T[k];
                for (int ch = 0; ch < 3; ++ch) Cc[ch] += p.color[ch] * wgt;
                Aa += wgt;
                Dd += p.t[2] * wgt;
            }
            for (int ch = 0; ch < 3; ++ch) image[3 * ip + ch] += Cc[ch] * norm;
            alpha[ip] += Aa * norm;
            depth[ip] += Dd * norm;
            if (g_image == nullptr) continue;
            const double gi[3] = {g_image[3 * ip] * norm, g_image[3 * ip + 1] * norm, g_image[3 * ip + 2] * norm};
            const double ga = g_alpha ? g_alpha[ip] * norm : 0.0, gdp = g_depth ? g_depth[ip] * norm : 0.0;
            L += gi[0] * Cc[0] + gi[1] * Cc[1] + gi[2] * Cc[2] + ga * Aa + gdp * Dd;
            if (!grad) continue;
            // suffix sums over the fragments behind k
            double sc = 0.0, sz = 0.0;
            for (size_t kk = m; kk-- > 0;) {
                const uint32_t g = f[kk].second;
                const ProjD& p = pd[g];
                const double a = al[kk];
                double gc = 0.0;
                for (int ch = 0; ch < 3; ++ch) gc += gi[ch] * p.color[ch];
                const double inv = 1.0 / std::max(1.0 - a, 1e-12);
                const double dA = gc * T[kk] - sc * inv + ga * T[m] * inv + gdp * (p.t[2] * T[kk] - sz * inv);
                double gcol = 0.0;
                for (int ch = 0; ch < 3; ++ch) gcol += gi[ch] * p.color[ch];
                sc += gcol * a * T[kk];
                sz += p.t[2] * a * T[kk];
                GradProj& G = gp[g];
                for (int ch = 0; ch < 3; ++ch) G.color[ch] += gi[ch] * a * T[kk];
                G.depth += gdp * a * T[kk];
                // the fragment's probability through its partial derivatives
                const FragP& q = fp[kk];
                G.op += dA * q.d_op;
                for (int c = 0; c < 3; ++c) G.conic[c] += dA * q.d_conic[c];
                G.m2[0] += dA * q.d_m2[0];
                G.m2[1] += dA * q.d_m2[1];
            }
        }
    if (loss) *loss = L;
    if (!grad) return 0;
    for (uint32_t g = 0; g < n; ++g)
        project_d_backward(pd[g], gp[g], sh + static_cast<size_t>(g) * bases * 3, bases, w2c, dfx, dfy, d_means + 3 * g,
                           d_scales + 3 * g, d_rotations + 4 * g, d_opacities + g, d_sh + static_cast<size_t>(g) * bases * 3);
    return 0;
}

}  // namespace

extern "C" {

int oracle_expected_image(const double* means, const double* scales, const double* rotations, const double* opacities,
                          const double* sh, uint32_t n, uint32_t bases, const double* w2c, const double* cam_pos,
                          uint32_t width, uint32_t height, double fx, double fy, double cx, double cy, double near_plane,
                          double far_plane, int ss_raw, int aa, const float* base_means, const float* base_scales,
                          const float* base_rotations, const float* base_opacities, const double* g_image,
                          const double* g_alpha, const double* g_depth, double* image, double* alpha, double* depth,
                          double* loss, double* d_means, double* d_scales, double* d_rotations, double* d_opacities,
                          double* d_sh) {
    return expected_image_impl(means, scales, rotations, opacities, sh, n, bases, w2c, cam_pos, width, height, fx, fy,
                               cx, cy, near_plane, far_plane, ss_raw, aa, base_means, base_scales, base_rotations,
                               base_opacities, g_image, g_alpha, g_depth, image, alpha, depth, loss, d_means, d_scales,
                               d_rotations, d_opacities, d_sh, false, 0, 0);
}

int oracle_expected_image_gps(const double* means, const double* scales, const double* rotations,
                              const double* opacities, const double* sh, uint32_t n, uint32_t bases, const double* w2c,
                              const double* cam_pos, uint32_t width, uint32_t height, double fx, double fy, double cx,
                              double cy, double near_plane, double far_plane, int ss_raw, int aa,
                              const float* base_means, const float* base_scales, const float* base_rotations,
                              const float* base_opacities, const double* g_image, const double* g_alpha,
                              const double* g_depth, double* image, double* alpha, double* depth, double* loss,
                              double* d_means, double* d_scales, double* d_rotations, double* d_opacities,
                              double* d_sh, int quad, int max_fragments) {
    return expected_image_impl(means, scales, rotations, opacities, sh, n, bases, w2c, cam_pos, width, height, fx, fy,
                               cx, cy, near_plane, far_plane, ss_raw, aa, base_means, base_scales, base_rotations,
                               base_opacities, g_image, g_alpha, g_depth, image, alpha, depth, loss, d_means, d_scales,
                               d_rotations, d_opacities, d_sh, true, quad, max_fragments);
}

}  // extern "C"
