// Backward pass of stochastic transparency: an unbiased one-sample estimator of the gradient of the
// expected image, computed from the sample's own winners (the reference has no backward).
//
// For a (sub)pixel with fragments in key order, one sample's colour, alpha and depth have the
// expectations C = sum c_i a_i T_i, A = sum a_i T_i, D = sum z_i a_i T_i (T_i = prod over the
// fragments before i of (1 - a_j)). With w the sample's winner (the closest accepted fragment):
//   E[1(w = k)]            = a_k T_k                  -> dC/dc_k, dD/dz_k
//   E[1(key_w >= key_k)]   = T_k                      (nothing before k was accepted)
//   E[1(key_w >  key_k) c_w] = sum_{i after k} c_i a_i T_i
//   E[1(w = none)]         = 1 - A
// so that, per sample, with upstream gradients g (colour), g_a, g_d of the pixel,
//   dL/da_k ~ g.(1(key_w >= key_k) c_k - 1(key_w > key_k) c_w / (1 - a_k))
//           + g_a 1(w = none) / (1 - a_k) + g_d (1(key_w >= key_k) z_k - 1(key_w > key_k) z_w / (1 - a_k))
// is unbiased for dE[L]/da_k of a linear loss. Fragment gradients are accumulated per Gaussian in
// its projected quantities (opacity, conic, 2-D mean, depth, colour) and a projection backward
// chains them to means, log-scales, quaternions, opacity logits and SH coefficients. The winners
// come from re-rendering the sample (same frame index) or from its stored framebuffer.
#include <cstdint>
#include <cuda_runtime.h>
#include "sgs_backward_gps.h"
#include "sgs_internal.h"
#include "sgs_rows.cuh"

namespace sgs {
namespace {

constexpr uint32_t kBlock = 256;
constexpr uint32_t kWarpsPerBlock = kBlock / 32;
constexpr uint32_t kFullMask = 0xffffffffu;
constexpr uint32_t kCoopFragments = 64;  // larger AABBs are processed by the whole warp
constexpr uint32_t kBigFragments = 2048;  // fused walk: larger AABBs go to the row-chunk queue
constexpr uint32_t kChunkPixels = 2048;   // pixels per stolen chunk (whole rows, at most 32)
constexpr uint32_t kQueueBlocksPerSM = 8;
constexpr int kAccum = 10;               // op, conic x/y/z, mean2d x/y, depth, colour r/g/b

// ---- Gaussian point splatting: the probability that a Gaussian puts a point into a pixel ----------
// A GPS Gaussian (projected opacity o, dilated 2-D covariance with conic C, mean m) draws
// N = rint(max(kf(w), 0)) points, w standard normal and kf the Cornish-Fisher expansion of a Poisson
// quantile at lambda = 2 pi sqrt(det) Li2(o) (math_utils.h:98-111, accumulate_scatter.cu:104-112),
// each independently with density -ln(1 - o G(x)) / lambda, G(x) = exp(-(x - m)^T C (x - m) / 2)
// (truncated_box_muller). A point in the square of a (sub)pixel whose centre passes the power test
// registers there, so the Gaussian reaches the pixel with probability h = 1 - Q,
//   Q = E[(1 - q)^N] = sum_n P(N = n) (1 - q)^n,  q = Lambda_p / lambda,
//   Lambda_p = integral over the pixel square of -ln(1 - o G),
// independently of the other Gaussians: the stochastic-transparency estimator holds with alpha
// replaced by h. Lambda_p and its derivatives come from a 3 x 3 Gauss-Legendre rule over the pixel.
// P(N = n) and dP/dlambda come from a table over log2(lambda) in [-10, 3] (32 terms, the rest of
// the law folded into the last), built per call by gps_count_law_kernel (sgs_backward_gps.h) in the
// caller's scratch; from lambda = 8 up the
// count is taken as Poisson (Q = exp(-Lambda_p)), which the draw matches there to within 3e-4.
constexpr int kLawRows = 1025;
constexpr int kLawTerms = 32;
constexpr float kLawLog2Min = -10.0f;
constexpr float kLawLog2Span = 13.0f;
static_assert(kLawTerms == 32, "one lane of the table kernel per term");

// kf(w) at lambda and its partial derivatives in w and lambda
__device__ __forceinline__ double law_kf(const double w, const double lam) {
    const double s = sqrt(lam), w2 = w * w;
    return lam + s * w + (w2 - 1.0) / 6.0 + (-(w / 36.0) - w2 * w / 72.0) / s +
           (-(8.0 / 405.0) + (7.0 / 810.0) * w2 + w2 * w2 / 270.0) / lam;
}
__device__ __forceinline__ double law_kf_w(const double w, const double lam) {
    const double s = sqrt(lam), w2 = w * w;
    return s + w / 3.0 + (-(1.0 / 36.0) - w2 / 24.0) / s + ((14.0 / 810.0) * w + (4.0 / 270.0) * w2 * w) / lam;
}
__device__ __forceinline__ double law_kf_lam(const double w, const double lam) {
    const double s = sqrt(lam), w2 = w * w;
    return 1.0 + w / (2.0 * s) - 0.5 * (-(w / 36.0) - w2 * w / 72.0) / (lam * s) -
           (-(8.0 / 405.0) + (7.0 / 810.0) * w2 + w2 * w2 / 270.0) / (lam * lam);
}

// One warp per table row (lambda = 2^(kLawLog2Min + kLawLog2Span r / (kLawRows - 1))). The quartic kf
// is monotone between the roots of kf' on [-12, 12] (outside, kf exceeds every threshold used); lane n
// computes F(n + 1/2) = P(kf(w) < n + 1/2) over those pieces and its lambda-derivative
// -sum over the roots r of kf = t of phi(r) (dkf/dlambda)(r) / |dkf/dw(r)|; then P(N = n) =
// F(n + 1/2) - F(n - 1/2), and the last term takes all of N >= kLawTerms - 1. Stored as (P, dP).
__global__ void __launch_bounds__(32) gps_count_law_kernel(float2* __restrict__ law) {
    constexpr double kW = 12.0;
    constexpr int kPerLane = 150;  // 32 x 150 grid intervals of kf' over [-kW, kW]
    constexpr int kMaxCuts = 16;
    __shared__ double s_cut[kMaxCuts + 2];
    __shared__ int s_n;
    const uint32_t lane = threadIdx.x;
    const double lam = exp2(static_cast<double>(kLawLog2Min) +
                            static_cast<double>(kLawLog2Span) * blockIdx.x / static_cast<double>(kLawRows - 1));
    if (lane == 0) s_n = 0;
    __syncwarp();
    const double step = 2.0 * kW / (32.0 * kPerLane);
    double w_prev = -kW + step * kPerLane * lane;
    double d_prev = law_kf_w(w_prev, lam);
    for (int i = 1; i <= kPerLane; ++i) {
        const double w = -kW + step * (kPerLane * lane + i);
        const double d = law_kf_w(w, lam);
        if ((d_prev < 0.0) != (d < 0.0)) {
            double lo = w_prev, hi = w;
            const bool lo_neg = d_prev < 0.0;
            for (int it = 0; it < 64 && hi - lo > 1e-15; ++it) {
                const double mid = 0.5 * (lo + hi);
                if ((law_kf_w(mid, lam) < 0.0) == lo_neg) lo = mid;
                else hi = mid;
            }
            const int slot = atomicAdd(&s_n, 1);
            if (slot < kMaxCuts) s_cut[slot + 1] = 0.5 * (lo + hi);
        }
        w_prev = w;
        d_prev = d;
    }
    __syncwarp();
    const int n_cut = min(s_n, kMaxCuts);
    if (lane == 0) {
        // insertion sort of the interior cuts, framed by the ends of the interval
        for (int i = 2; i <= n_cut; ++i) {
            const double v = s_cut[i];
            int j = i - 1;
            while (j >= 1 && s_cut[j] > v) {
                s_cut[j + 1] = s_cut[j];
                --j;
            }
            s_cut[j + 1] = v;
        }
        s_cut[0] = -kW;
        s_cut[n_cut + 1] = kW;
    }
    __syncwarp();
    const double t = lane + 0.5;
    double F = 0.0, dF = 0.0;
    for (int i = 0; i <= n_cut; ++i) {
        const double a = s_cut[i], bnd = s_cut[i + 1];
        const double fa = law_kf(a, lam), fb = law_kf(bnd, lam);
        const bool up = fb >= fa;
        const double lo_v = up ? fa : fb, hi_v = up ? fb : fa;
        if (t <= lo_v) continue;
        const double ca = 0.5 * erfc(-a * 0.70710678118654752), cb = 0.5 * erfc(-bnd * 0.70710678118654752);
        if (t >= hi_v) {
            F += cb - ca;
            continue;
        }
        double lo = a, hi = bnd;
        for (int it = 0; it < 64 && hi - lo > 1e-15; ++it) {
            const double mid = 0.5 * (lo + hi);
            if ((law_kf(mid, lam) < t) == up) lo = mid;
            else hi = mid;
        }
        const double r = 0.5 * (lo + hi);
        const double cr = 0.5 * erfc(-r * 0.70710678118654752);
        F += up ? cr - ca : cb - cr;
        const double slope = fabs(law_kf_w(r, lam));
        if (slope > 0.0) dF -= exp(-0.5 * r * r) * 0.39894228040143268 * law_kf_lam(r, lam) / slope;
    }
    double F_below = __shfl_up_sync(0xffffffffu, F, 1);
    double dF_below = __shfl_up_sync(0xffffffffu, dF, 1);
    if (lane == 0) {
        F_below = 0.0;
        dF_below = 0.0;
    }
    double P = F - F_below, dP = dF - dF_below;
    if (lane == kLawTerms - 1) {  // N >= kLawTerms - 1
        P = 1.0 - F_below;
        dP = -dF_below;
    }
    law[static_cast<size_t>(blockIdx.x) * kLawTerms + lane] = make_float2(static_cast<float>(P), static_cast<float>(dP));
}

// Per-Gaussian constants of the GPS hit probability.
struct GpsConstants {
    float lambda;      // expected point count
    float d_lambda[4]; // d lambda / d (opacity, conic x, y, z)
    float law_pos;     // row position of lambda in the count table; kLawRows - 1: Poisson
    float pad[2];
};

__device__ __forceinline__ GpsConstants gps_constants(const Projected& p) {
    GpsConstants c;
    const float sd = sqrtf(p.determinant);
    const float lam = kTwoPi * sd * gps_dilog(p.opacity);
    const float D = p.conic.x * p.conic.z - p.conic.y * p.conic.y;  // 1 / det
    c.lambda = lam;
    c.d_lambda[0] = kTwoPi * sd * (-logf(fmaxf(1.0f - p.opacity, 1.0e-7f)) / p.opacity);  // Li2'(o) = -ln(1 - o) / o
    c.d_lambda[1] = -0.5f * lam * p.conic.z / D;
    c.d_lambda[2] = lam * p.conic.y / D;
    c.d_lambda[3] = -0.5f * lam * p.conic.x / D;
    const float pos = (log2f(lam) - kLawLog2Min) * (static_cast<float>(kLawRows - 1) / kLawLog2Span);
    c.law_pos = fminf(fmaxf(pos, 0.0f), static_cast<float>(kLawRows - 1));
    c.pad[0] = c.pad[1] = 0.0f;
    return c;
}

// Q (no point of the Gaussian in the pixel) and its derivatives in the projected opacity, the conic
// and the 2-D mean, for the pixel whose centre lies at (dx0, dy0) from the mean.
struct GpsFragment {
    float Q, dQ_op, dQ_conic[3], dQ_m[2];
};

__device__ __forceinline__ GpsFragment gps_fragment(const float cx, const float cy, const float cz, const float op,
                                                    const float3 conic, const GpsConstants& c, const float dx0,
                                                    const float dy0, const float2* __restrict__ law) {
    constexpr float kOff = 0.38729833462074170f;  // Gauss-Legendre nodes of [0, 1]: 1/2 +- sqrt(3/5) / 2
    constexpr float kWe = 5.0f / 18.0f, kWm = 8.0f / 18.0f;
    float L = 0.0f, s_o = 0.0f, s_xx = 0.0f, s_xy = 0.0f, s_yy = 0.0f, s_x = 0.0f, s_y = 0.0f;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        const float dx = dx0 + static_cast<float>(i - 1) * kOff;
        const float wi = i == 1 ? kWm : kWe;
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            const float dy = dy0 + static_cast<float>(j - 1) * kOff;
            const float W = wi * (j == 1 ? kWm : kWe);
            const float e = dx * (cx * dx + cy * dy) + cz * dy * dy;  // log2 G
            const float oG = op * exp2f(fminf(e, 0.0f));
            const float rest = 1.0f - oG;
            L -= W * logf(rest);
            const float w = W * oG / rest;
            s_o += w;
            s_xx += w * dx * dx;
            s_xy += w * dx * dy;
            s_yy += w * dy * dy;
            s_x += w * dx;
            s_y += w * dy;
        }
    }
    float Q, dQ_dL, dQ_dlam;
    if (c.law_pos >= static_cast<float>(kLawRows - 1)) {
        Q = expf(-L);
        dQ_dL = -Q;
        dQ_dlam = 0.0f;
    } else {
        const int row = static_cast<int>(c.law_pos);
        const float t = c.law_pos - static_cast<float>(row);
        const float2* r0 = law + static_cast<size_t>(row) * kLawTerms;
        const float2* r1 = r0 + kLawTerms;
        const float Z = fmaxf(1.0f - L / c.lambda, 0.0f);
        float dZ = 0.0f, dl = 0.0f;
        Q = 0.0f;
        for (int n = kLawTerms - 1; n >= 0; --n) {
            const float2 a = r0[n], b = r1[n];
            dZ = dZ * Z + Q;
            Q = Q * Z + (a.x + t * (b.x - a.x));
            dl = dl * Z + (a.y + t * (b.y - a.y));
        }
        dQ_dL = -dZ / c.lambda;
        dQ_dlam = dZ * L / (c.lambda * c.lambda) + dl;
    }
    GpsFragment f;
    f.Q = Q;
    f.dQ_op = dQ_dL * (s_o / op) + dQ_dlam * c.d_lambda[0];
    f.dQ_conic[0] = dQ_dL * (-0.5f * s_xx) + dQ_dlam * c.d_lambda[1];
    f.dQ_conic[1] = dQ_dL * (-s_xy) + dQ_dlam * c.d_lambda[2];
    f.dQ_conic[2] = dQ_dL * (-0.5f * s_yy) + dQ_dlam * c.d_lambda[3];
    f.dQ_m[0] = dQ_dL * (conic.x * s_x + conic.y * s_y);
    f.dQ_m[1] = dQ_dL * (conic.y * s_x + conic.z * s_y);
    return f;
}

// View-dependent colour of every Gaussian (the colour its fragments would give a pixel).
__global__ void __launch_bounds__(kBlock) colors_kernel(const BackwardParams b) {
    const uint32_t g = blockIdx.x * kBlock + threadIdx.x;
    if (g >= b.n) return;
    const float vx = b.means[3 * g + 0] - b.cam_position[0];
    const float vy = b.means[3 * g + 1] - b.cam_position[1];
    const float vz = b.means[3 * g + 2] - b.cam_position[2];
    const float inv_len = rsqrtf(vx * vx + vy * vy + vz * vz);
    const float3 c = eval_sh(b.sh + static_cast<size_t>(g) * b.sh_bases * 3, vx * inv_len, vy * inv_len, vz * inv_len,
                             b.sh_bases);
    b.colors[3 * g + 0] = c.x;
    b.colors[3 * g + 1] = c.y;
    b.colors[3 * g + 2] = c.z;
}

struct FragAccum {
    float v[kAccum];
};

// Contribution of one fragment of Gaussian k at framebuffer pixel (px, py) to k's accumulators.
__device__ __forceinline__ void fragment_grad(const BackwardParams& b, const Projected& p, const float3 ce,
                                             const unsigned long long key_k, const float3 ck, const uint32_t px,
                                             const uint32_t py, FragAccum& acc) {
    const float mx = p.mean2d.x - 0.5f, my = p.mean2d.y - 0.5f;
    const float dx = static_cast<float>(px) - mx;
    const float dy = static_cast<float>(py) - my;
    const float alpha = fragment_alpha(ce, p.opacity, dx, dy);
    if (alpha < kMinAlpha) return;
    const uint32_t pix = py * b.cam.width_int + px;
    const unsigned long long key_w = b.framebuffer[pix];
    const float4 sw = b.samples[pix];  // winner colour and depth (0 for background)
    // upstream gradients of the image pixel, spread over its subpixels and the averaged samples
    const uint32_t ip = (py / b.ss) * b.width + px / b.ss;
    const float gs = b.grad_scale;
    const float g0 = b.grad_image[3 * ip + 0] * gs, g1 = b.grad_image[3 * ip + 1] * gs, g2 = b.grad_image[3 * ip + 2] * gs;
    const float ga = b.grad_alpha != nullptr ? b.grad_alpha[ip] * gs : 0.0f;
    const float gd = b.grad_depth != nullptr ? b.grad_depth[ip] * gs : 0.0f;
    const bool ge = key_w >= key_k;
    const bool gt = key_w > key_k;
    const bool none = key_w == kEmptyFragment;
    const float inv = 1.0f / fmaxf(1.0f - alpha, 1e-12f);
    const float gck = g0 * ck.x + g1 * ck.y + g2 * ck.z;
    const float gcw = g0 * sw.x + g1 * sw.y + g2 * sw.z;
    float dA = (ge ? gck : 0.0f) - (gt ? gcw * inv : 0.0f) + (none ? ga * inv : 0.0f);
    dA += gd * ((ge ? p.depth : 0.0f) - (gt ? sw.w * inv : 0.0f));
    if (key_w == key_k) {  // this Gaussian won the pixel
        acc.v[6] += gd;
        acc.v[7] += g0;
        acc.v[8] += g1;
        acc.v[9] += g2;
    }
    // alpha = opacity exp(-0.5 (cX dx^2 + cZ dy^2) - cY dx dy)
    const float dAe = dA * alpha;
    acc.v[0] += dA * (alpha / p.opacity);
    acc.v[1] += dAe * (-0.5f * dx * dx);
    acc.v[2] += dAe * (-dx * dy);
    acc.v[3] += dAe * (-0.5f * dy * dy);
    acc.v[4] += dAe * (p.conic.x * dx + p.conic.y * dy);
    acc.v[5] += dAe * (p.conic.y * dx + p.conic.z * dy);
}

// One thread per Gaussian; AABBs above kCoopFragments pixels are processed by the whole warp.
__global__ void __launch_bounds__(kBlock) fragments_backward_kernel(const BackwardParams b) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t idx = blockIdx.x * kBlock + threadIdx.x;
    bool active = idx < b.n;
    const uint32_t g = active ? idx : b.n - 1;
    Projected p;
    if (!project_gaussian(active, g, b.means, b.scales, b.rotations, b.opacities, b.w2c, b.cam, p)) return;
    const PixelRect rect = pixel_rect(p.bounds, b.cam);
    const uint32_t count = active ? rect.width * rect.height : 0u;
    const float3 ce = conic_for_exp2(p.conic);
    const unsigned long long key = pack_fragment(p.depth, g);
    const float3 ck = make_float3(b.colors[3 * g + 0], b.colors[3 * g + 1], b.colors[3 * g + 2]);
    FragAccum acc;
#pragma unroll
    for (int i = 0; i < kAccum; ++i) acc.v[i] = 0.0f;
    if (count <= kCoopFragments) {
        for (uint32_t f = 0; f < count; ++f)
            fragment_grad(b, p, ce, key, ck, rect.x_min + f % rect.width, rect.y_min + f / rect.width, acc);
    }
    uint32_t pending = __ballot_sync(kFullMask, count > kCoopFragments);
    while (pending) {
        const uint32_t src = __ffs(pending) - 1;
        pending &= pending - 1;
        Projected q;
        q.depth = __shfl_sync(kFullMask, p.depth, src);
        q.opacity = __shfl_sync(kFullMask, p.opacity, src);
        q.mean2d = make_float2(__shfl_sync(kFullMask, p.mean2d.x, src), __shfl_sync(kFullMask, p.mean2d.y, src));
        q.conic = make_float3(__shfl_sync(kFullMask, p.conic.x, src), __shfl_sync(kFullMask, p.conic.y, src),
                              __shfl_sync(kFullMask, p.conic.z, src));
        const float3 qce = conic_for_exp2(q.conic);
        const unsigned long long qkey = __shfl_sync(kFullMask, key, src);
        const float3 qck = make_float3(__shfl_sync(kFullMask, ck.x, src), __shfl_sync(kFullMask, ck.y, src),
                                       __shfl_sync(kFullMask, ck.z, src));
        const uint32_t x0 = __shfl_sync(kFullMask, rect.x_min, src), y0 = __shfl_sync(kFullMask, rect.y_min, src);
        const uint32_t w = __shfl_sync(kFullMask, rect.width, src), n = __shfl_sync(kFullMask, count, src);
        FragAccum part;
#pragma unroll
        for (int i = 0; i < kAccum; ++i) part.v[i] = 0.0f;
        for (uint32_t f = lane; f < n; f += 32) fragment_grad(b, q, qce, qkey, qck, x0 + f % w, y0 + f / w, part);
#pragma unroll
        for (int i = 0; i < kAccum; ++i) {
            float v = part.v[i];
            for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFullMask, v, o);
            if (lane == src) acc.v[i] += v;
        }
    }
    if (!active) return;
    float* out = b.accum + static_cast<size_t>(g) * kAccum;
#pragma unroll
    for (int i = 0; i < kAccum; ++i)
        if (acc.v[i] != 0.0f) out[i] += acc.v[i];
}


// ---- Fused form over S samples ------------------------------------------------------------------
// The estimator is a sum over samples of terms that depend on the sample only through the pixel's
// winner. sample_terms_kernel stores, per framebuffer pixel and sample, the winner key and
// T = s (g . c_w + g_d z_w); one walk over every Gaussian's fragments then evaluates alpha and the
// geometric factors once and sums the S samples' contributions:
//   dL/da_k = ge (g . c_k + g_d z_k) - sum_{key_w > key_k} T / (1 - a_k) + g_a n_none / (1 - a_k)
// with ge = #samples whose winner is not in front of k and n_none = #samples with no winner.
// A fragment behind every sample's winner (key_k > the pixel's largest winner key, an empty pixel
// counting as the largest key) contributes exactly zero; the walk tests that first, so the per-sample
// table is read only for the fragments in front of some winner.

__global__ void __launch_bounds__(kBlock) sample_terms_kernel(const BackwardParams b) {
    const uint32_t pix = blockIdx.x * kBlock + threadIdx.x;
    if (pix >= b.n_fb) return;
    const unsigned long long key = b.framebuffer[pix];
    const float4 sw = b.samples[pix];  // winner colour and depth (0 for background)
    const uint32_t px = pix % b.cam.width_int, py = pix / b.cam.width_int;
    const uint32_t ip = (py / b.ss) * b.width + px / b.ss;
    float t = b.grad_image[3 * ip + 0] * sw.x + b.grad_image[3 * ip + 1] * sw.y + b.grad_image[3 * ip + 2] * sw.z;
    if (b.grad_depth != nullptr) t += b.grad_depth[ip] * sw.w;
    const size_t slot = static_cast<size_t>(pix) * b.n_samples + b.sample;
    b.pix_keys[slot] = key;
    b.pix_terms[slot] = t * b.grad_scale;
    // the farthest winner of the samples so far (launches are ordered: sample 0 starts the maximum)
    b.pix_max_key[pix] = b.sample == 0 ? key : max(b.pix_max_key[pix], key);
}

// The same table from the framebuffers of all S samples at once (consecutive, b.n_fb apart): the
// winner's colour is its Gaussian's view-dependent colour (colors_kernel, the function the sample
// pass evaluates) and its depth the key's high word.
__global__ void __launch_bounds__(kBlock) framebuffer_terms_kernel(const BackwardParams b) {
    const uint32_t pix = blockIdx.x * kBlock + threadIdx.x;
    if (pix >= b.n_fb) return;
    const uint32_t px = pix % b.cam.width_int, py = pix / b.cam.width_int;
    const uint32_t ip = (py / b.ss) * b.width + px / b.ss;
    const float g0 = b.grad_image[3 * ip + 0], g1 = b.grad_image[3 * ip + 1], g2 = b.grad_image[3 * ip + 2];
    const float gd = b.grad_depth != nullptr ? b.grad_depth[ip] : 0.0f;
    unsigned long long max_key = 0;
    const size_t row = static_cast<size_t>(pix) * b.n_samples;
    for (uint32_t s = 0; s < b.n_samples; ++s) {
        const unsigned long long key = b.framebuffer[static_cast<size_t>(s) * b.n_fb + pix];
        float t = 0.0f;
        if (key != kEmptyFragment) {
            const uint32_t w = static_cast<uint32_t>(key);
            t = g0 * b.colors[3 * w + 0] + g1 * b.colors[3 * w + 1] + g2 * b.colors[3 * w + 2] +
                gd * __uint_as_float(static_cast<uint32_t>(key >> 32));
        }
        b.pix_keys[row + s] = key;
        b.pix_terms[row + s] = t * b.grad_scale;
        max_key = max(max_key, key);
    }
    b.pix_max_key[pix] = max_key;
}

// Rows per chunk of a queued Gaussian of AABB width w (log2): about kChunkPixels pixels, a power of
// two between 1 and 32; each row of a chunk is walked in 32 / rows segments.
__device__ __forceinline__ uint32_t log_chunk_rows(const uint32_t w) {
    const uint32_t rows = max(1u, min(32u, kChunkPixels / max(w, 1u)));
    return 31u - __clz(rows);
}

// Per-Gaussian constants of the fused walk (96 bytes).
struct WalkGaussian {
    float mx, my;             // mean2d - 0.5
    float cx, cy, cz;         // exp2-scaled conic
    float opacity;
    SpanConstants span;
    float conic_x, conic_y, conic_z;
    float depth;
    float ckx, cky, ckz;      // view-dependent colour
    uint32_t key_lo, key_hi;
    uint32_t x_min, y_min, w;
    uint32_t row_first;       // first row position in the warp's row list
    uint32_t pad[2];
};
static_assert(sizeof(WalkGaussian) == 96, "WalkEntry pairs it with 32 bytes of GPS constants");


// A queue entry of the fused walk: the walk constants and, for GPS, the hit-probability constants.
struct WalkEntry {
    WalkGaussian g;
    GpsConstants c;
};
static_assert(sizeof(WalkEntry) == 128, "the backward workspace reserves 128 bytes per queue entry");

// Lane walks the span of row y of Gaussian q (when valid), one pixel per step, and adds the S
// samples' fragment gradients to acc. kGps: the fragment probability is the GPS hit probability
// (constants gc) instead of alpha.
template <bool kGps>
__device__ __forceinline__ void walk_row_gradients(const BackwardParams& b, const WalkGaussian& q,
                                                   const GpsConstants& gc, const float2* __restrict__ law,
                                                   const bool valid, const uint32_t y, FragAccum& acc,
                                                   const uint32_t seg = 0, const uint32_t log_segs = 0) {
    uint32_t xs = 0, len = 0;
    float dy = 0.0f;
    if (valid) {
        dy = static_cast<float>(y) - q.my;
        row_span(q.x_min, q.w, q.mx, q.span, dy, xs, len);
        if (log_segs > 0) {
            const uint32_t part = (len + (1u << log_segs) - 1u) >> log_segs;
            const uint32_t skip = min(seg * part, len);
            xs += skip;
            len = min(len - skip, part);
        }
    }
    const uint32_t steps = __reduce_max_sync(kFullMask, len);
    if (steps == 0) return;
    const uint32_t S = b.n_samples;
    const float gs = b.grad_scale;
    const float cydy = q.cy * dy, czdy = q.cz * dy;
    const uint32_t iy = y / b.ss;
    const float* g_row = b.grad_image + 3 * static_cast<size_t>(iy) * b.width;
    const float* ga_row = b.grad_alpha != nullptr ? b.grad_alpha + static_cast<size_t>(iy) * b.width : nullptr;
    const float* gd_row = b.grad_depth != nullptr ? b.grad_depth + static_cast<size_t>(iy) * b.width : nullptr;
    const unsigned long long key_k = (static_cast<unsigned long long>(q.key_hi) << 32) | q.key_lo;
    const size_t pix0 = static_cast<size_t>(y) * b.cam.width_int + xs;
    uint32_t ix = xs / b.ss, sub = xs - ix * b.ss;
    float fx = static_cast<float>(xs);
    for (uint32_t i = 0; i < steps; ++i) {
        if (i < len && key_k <= b.pix_max_key[pix0 + i]) {
            const float dx = fx - q.mx;
            const float e = dx * (q.cx * dx + cydy) + czdy * dy;
            const float alpha = q.opacity * exp2f(fminf(e, 0.0f));
            if (alpha >= kMinAlpha) {
                const float g0 = g_row[3 * ix + 0] * gs, g1 = g_row[3 * ix + 1] * gs, g2 = g_row[3 * ix + 2] * gs;
                const float ga = ga_row != nullptr ? ga_row[ix] * gs : 0.0f;
                const float gd = gd_row != nullptr ? gd_row[ix] * gs : 0.0f;
                const unsigned long long* keys = b.pix_keys + (pix0 + i) * S;
                const float* terms = b.pix_terms + (pix0 + i) * S;
                uint32_t ge = 0, won = 0, none = 0;
                float behind = 0.0f;
                uint32_t s = 0;
                if ((S & 1u) == 0) {
                    for (; s < S; s += 2) {
                        const ulonglong2 kk = *reinterpret_cast<const ulonglong2*>(keys + s);
                        const float2 tt = *reinterpret_cast<const float2*>(terms + s);
                        ge += (kk.x >= key_k) + (kk.y >= key_k);
                        won += (kk.x == key_k) + (kk.y == key_k);
                        none += (kk.x == kEmptyFragment) + (kk.y == kEmptyFragment);
                        behind += (kk.x > key_k ? tt.x : 0.0f) + (kk.y > key_k ? tt.y : 0.0f);
                    }
                }
                for (; s < S; ++s) {
                    const unsigned long long kk = keys[s];
                    ge += kk >= key_k;
                    won += kk == key_k;
                    none += kk == kEmptyFragment;
                    if (kk > key_k) behind += terms[s];
                }
                const float gck = g0 * q.ckx + g1 * q.cky + g2 * q.ckz + gd * q.depth;
                if (won != 0) {
                    const float wf = static_cast<float>(won);
                    acc.v[6] += gd * wf;
                    acc.v[7] += g0 * wf;
                    acc.v[8] += g1 * wf;
                    acc.v[9] += g2 * wf;
                }
                if (kGps) {
                    // h = 1 - Q: dL/dh from the samples, then through Q's partial derivatives
                    const GpsFragment f = gps_fragment(q.cx, q.cy, q.cz, q.opacity,
                                                       make_float3(q.conic_x, q.conic_y, q.conic_z), gc, dx, dy,
                                                       law);
                    const float inv = 1.0f / fmaxf(f.Q, 1e-12f);
                    const float dH = static_cast<float>(ge) * gck - inv * behind + inv * ga * static_cast<float>(none);
                    acc.v[0] -= dH * f.dQ_op;
                    acc.v[1] -= dH * f.dQ_conic[0];
                    acc.v[2] -= dH * f.dQ_conic[1];
                    acc.v[3] -= dH * f.dQ_conic[2];
                    acc.v[4] -= dH * f.dQ_m[0];
                    acc.v[5] -= dH * f.dQ_m[1];
                } else {
                    const float inv = 1.0f / fmaxf(1.0f - alpha, 1e-12f);
                    const float dA = static_cast<float>(ge) * gck - inv * behind + inv * ga * static_cast<float>(none);
                    // alpha = opacity exp(-0.5 (cX dx^2 + cZ dy^2) - cY dx dy)
                    const float dAe = dA * alpha;
                    acc.v[0] += dA * (alpha / q.opacity);
                    acc.v[1] += dAe * (-0.5f * dx * dx);
                    acc.v[2] += dAe * (-dx * dy);
                    acc.v[3] += dAe * (-0.5f * dy * dy);
                    acc.v[4] += dAe * (q.conic_x * dx + q.conic_y * dy);
                    acc.v[5] += dAe * (q.conic_y * dx + q.conic_z * dy);
                }
            }
        }
        fx += 1.0f;
        if (++sub == b.ss) {
            sub = 0;
            ++ix;
        }
    }
}

// One thread per Gaussian: the rows of a warp's 32 Gaussians are laid end to end, 32 per step, and
// each lane walks one row; the row sums go to per-Gaussian accumulators in shared memory.
template <bool kGps>
__global__ void __launch_bounds__(kBlock) fragments_samples_kernel(const BackwardParams b, const float2* __restrict__ law) {
    __shared__ WalkGaussian s_g[kWarpsPerBlock][32];
    __shared__ GpsConstants s_c[kGps ? kWarpsPerBlock : 1][32];
    __shared__ float s_acc[kWarpsPerBlock][32][kAccum];
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t wib = threadIdx.x >> 5;
    const uint32_t lt_mask = (1u << lane) - 1u;
    const uint32_t upto_mask = kFullMask >> (31u - lane);
    const uint32_t idx = blockIdx.x * kBlock + threadIdx.x;
    bool active = idx < b.n;
    const uint32_t g = active ? idx : b.n - 1;
#pragma unroll
    for (int i = 0; i < kAccum; ++i) s_acc[wib][lane][i] = 0.0f;
    Projected p;
    if (!project_gaussian(active, g, b.means, b.scales, b.rotations, b.opacities, b.w2c, b.cam, p)) return;
    const PixelRect rect = pixel_rect(p.bounds, b.cam);
    bool has_rows = active && rect.width > 0 && rect.height > 0;
    WalkGaussian q;
    GpsConstants c{};
    if (kGps && has_rows) c = gps_constants(p);
    if (has_rows) {
        q.mx = p.mean2d.x - 0.5f;
        q.my = p.mean2d.y - 0.5f;
        const float3 ce = conic_for_exp2(p.conic);
        q.cx = ce.x;
        q.cy = ce.y;
        q.cz = ce.z;
        q.opacity = p.opacity;
        q.span = span_constants(ce.x, ce.y, ce.z, p.opacity);
        q.conic_x = p.conic.x;
        q.conic_y = p.conic.y;
        q.conic_z = p.conic.z;
        q.depth = p.depth;
        q.ckx = b.colors[3 * g + 0];
        q.cky = b.colors[3 * g + 1];
        q.ckz = b.colors[3 * g + 2];
        const unsigned long long key = pack_fragment(p.depth, g);
        q.key_lo = static_cast<uint32_t>(key);
        q.key_hi = static_cast<uint32_t>(key >> 32);
        q.x_min = rect.x_min;
        q.y_min = rect.y_min;
        q.w = rect.width;
        q.row_first = 0;
        // large footprints go to the queue (walked in row chunks across all SMs) unless it is full
        if (rect.width * rect.height > kBigFragments) {
            const uint32_t log_rpc = log_chunk_rows(rect.width);
            const uint32_t chunks = (rect.height + (1u << log_rpc) - 1u) >> log_rpc;
            const unsigned long long old = atomicAdd(&b.bw_queue->packed, (1ull << kQueueEntryShift) | chunks);
            const uint32_t e = static_cast<uint32_t>(old >> kQueueEntryShift);
            const unsigned long long first_chunk = old & kQueueChunkMask;
            if (e < b.bw_capacity && first_chunk + chunks <= kMaxQueueChunks) {
                WalkEntry* entry = static_cast<WalkEntry*>(b.bw_entries) + e;
                entry->g = q;
                if (kGps) entry->c = c;
                b.bw_meta[e] = make_uint4(rect.y_min, rect.height, log_rpc, static_cast<uint32_t>(first_chunk));
                b.bw_index[e] = g;
                has_rows = false;
            } else if (e < b.bw_capacity) {
                // past 32-bit chunk indices: marked unused (the marked entries are the last ones), walked here
                b.bw_meta[e] = make_uint4(0u, 0u, 0u, kUnusedQueueEntry);
            }
        }
    }
    const uint32_t gmask = __ballot_sync(kFullMask, has_rows);
    const uint32_t h = has_rows ? rect.height : 0u;
    const uint32_t row_incl = warp_inclusive_sum(h, lane);
    const uint32_t total_rows = __shfl_sync(kFullMask, row_incl, 31);
    const uint32_t slot = __popc(gmask & lt_mask);
    if (has_rows) {
        q.row_first = row_incl - h;
        s_g[wib][slot] = q;
        if (kGps) s_c[wib][slot] = c;
    }
    __syncwarp();
    int prev = -1;
    for (uint32_t base = 0; base < total_rows; base += 32) {
        const uint32_t rel = (row_incl - h) - base;
        const uint32_t bits = __reduce_or_sync(kFullMask, (has_rows && rel < 32u) ? (1u << rel) : 0u);
        const int owner = prev + __popc(bits & upto_mask);
        prev += __popc(bits);
        const uint32_t r = base + lane;
        const bool valid = r < total_rows;
        const WalkGaussian rq = s_g[wib][valid ? owner : 0];
        const GpsConstants rc = kGps ? s_c[wib][valid ? owner : 0] : GpsConstants{};
        FragAccum acc;
#pragma unroll
        for (int i = 0; i < kAccum; ++i) acc.v[i] = 0.0f;
        walk_row_gradients<kGps>(b, rq, rc, law, valid, rq.y_min + (r - rq.row_first), acc);
        if (valid) {
#pragma unroll
            for (int i = 0; i < kAccum; ++i)
                if (acc.v[i] != 0.0f) atomicAdd(&s_acc[wib][owner][i], acc.v[i]);
        }
    }
    __syncwarp();
    if (!has_rows) return;
    float* out = b.accum + static_cast<size_t>(g) * kAccum;
#pragma unroll
    for (int i = 0; i < kAccum; ++i) {
        const float v = s_acc[wib][slot][i];
        if (v != 0.0f) out[i] += v;
    }
}

// Persistent consumer of the fused walk's large-Gaussian queue: each warp steals one chunk of rows
// (R rows, each split into 32 / R lane segments), sums the lanes' gradients and adds them to the
// Gaussian's accumulators.
template <bool kGps>
__global__ void __launch_bounds__(kBlock) fragments_samples_queue_kernel(const BackwardParams b,
                                                                         const float2* __restrict__ law) {
    const uint32_t lane = threadIdx.x & 31u;
    const unsigned long long packed = b.bw_queue->packed;
    const uint32_t n_entries =
        static_cast<uint32_t>(min(packed >> kQueueEntryShift, static_cast<unsigned long long>(b.bw_capacity)));
    if (n_entries == 0) return;
    uint32_t last_entry = n_entries - 1;  // the last used entry; entry 0 starts at chunk 0 and always is
    if (b.bw_meta[last_entry].w == kUnusedQueueEntry)
        last_entry = queue_entry_of_chunk(b.bw_meta, n_entries, kUnusedQueueEntry - 1u, lane);
    const uint4 last = b.bw_meta[last_entry];
    const uint32_t n_chunks = last.w + ((last.y + (1u << last.z) - 1u) >> last.z);
    const WalkEntry* entries = static_cast<const WalkEntry*>(b.bw_entries);
    for (;;) {
        uint32_t c = 0;
        if (lane == 0) c = atomicAdd(&b.bw_queue->next_chunk, 1u);
        c = __shfl_sync(kFullMask, c, 0);
        if (c >= n_chunks) break;
        uint32_t lo = 0, hi = n_entries - 1;
        while (lo < hi) {
            const uint32_t mid = (lo + hi + 1) >> 1;
            if (b.bw_meta[mid].w <= c) lo = mid;
            else hi = mid - 1;
        }
        const uint4 m = b.bw_meta[lo];
        const uint32_t log_rows = m.z;
        const uint32_t r0 = (c - m.w) << log_rows;
        if (r0 >= m.y || log_rows > 5u) {
            if (lane == 0) atomicOr(&b.bw_queue->error, 1u);
            continue;
        }
        const WalkGaussian q = entries[lo].g;
        const GpsConstants gc = kGps ? entries[lo].c : GpsConstants{};
        const uint32_t r = r0 + (lane & ((1u << log_rows) - 1u));
        FragAccum acc;
#pragma unroll
        for (int i = 0; i < kAccum; ++i) acc.v[i] = 0.0f;
        walk_row_gradients<kGps>(b, q, gc, law, r < m.y, q.y_min + r, acc, lane >> log_rows, 5u - log_rows);
        float* out = b.accum + static_cast<size_t>(b.bw_index[lo]) * kAccum;
#pragma unroll
        for (int i = 0; i < kAccum; ++i) {
            float v = acc.v[i];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFullMask, v, o);
            if (lane == 0 && v != 0.0f) atomicAdd(out + i, v);
        }
    }
}

// Signed SH basis of eval_sh (gs_utils.h:212-243) and its gradient w.r.t. the direction.
__device__ __forceinline__ void sh_basis(const float x, const float y, const float z, float Y[16], float dY[16][3]) {
    const float xx = x * x, yy = y * y, zz = z * z;
    Y[0] = kSH0; dY[0][0] = 0; dY[0][1] = 0; dY[0][2] = 0;
    Y[1] = -kSH1 * y; dY[1][0] = 0; dY[1][1] = -kSH1; dY[1][2] = 0;
    Y[2] = kSH1 * z; dY[2][0] = 0; dY[2][1] = 0; dY[2][2] = kSH1;
    Y[3] = -kSH1 * x; dY[3][0] = -kSH1; dY[3][1] = 0; dY[3][2] = 0;
    Y[4] = kSH2a * x * y; dY[4][0] = kSH2a * y; dY[4][1] = kSH2a * x; dY[4][2] = 0;
    Y[5] = -kSH2a * y * z; dY[5][0] = 0; dY[5][1] = -kSH2a * z; dY[5][2] = -kSH2a * y;
    Y[6] = kSH2b * zz - kSH2c; dY[6][0] = 0; dY[6][1] = 0; dY[6][2] = 2.0f * kSH2b * z;
    Y[7] = -kSH2a * x * z; dY[7][0] = -kSH2a * z; dY[7][1] = 0; dY[7][2] = -kSH2a * x;
    Y[8] = kSH2d * (xx - yy); dY[8][0] = 2.0f * kSH2d * x; dY[8][1] = -2.0f * kSH2d * y; dY[8][2] = 0;
    Y[9] = y * (kSH3a * yy - kSH3b * xx); dY[9][0] = -2.0f * kSH3b * x * y; dY[9][1] = 3.0f * kSH3a * yy - kSH3b * xx; dY[9][2] = 0;
    Y[10] = kSH3c * x * y * z; dY[10][0] = kSH3c * y * z; dY[10][1] = kSH3c * x * z; dY[10][2] = kSH3c * x * y;
    Y[11] = y * (kSH3d - kSH3e * zz); dY[11][0] = 0; dY[11][1] = kSH3d - kSH3e * zz; dY[11][2] = -2.0f * kSH3e * y * z;
    Y[12] = z * (kSH3f * zz - kSH3g); dY[12][0] = 0; dY[12][1] = 0; dY[12][2] = 3.0f * kSH3f * zz - kSH3g;
    Y[13] = x * (kSH3d - kSH3e * zz); dY[13][0] = kSH3d - kSH3e * zz; dY[13][1] = 0; dY[13][2] = -2.0f * kSH3e * x * z;
    Y[14] = kSH3h * z * (xx - yy); dY[14][0] = 2.0f * kSH3h * x * z; dY[14][1] = -2.0f * kSH3h * y * z; dY[14][2] = kSH3h * (xx - yy);
    Y[15] = x * (kSH3b * yy - kSH3a * xx); dY[15][0] = kSH3b * yy - 3.0f * kSH3a * xx; dY[15][1] = 2.0f * kSH3b * x * y; dY[15][2] = 0;
}

// Projection backward (gs_utils.h:38-193 differentiated): accumulated projected-quantity gradients to
// the parameters. Culled Gaussians receive zero gradients.
__global__ void __launch_bounds__(kBlock) projection_backward_kernel(const BackwardParams b) {
    const uint32_t g = blockIdx.x * kBlock + threadIdx.x;
    if (g >= b.n) return;
    const float* acc = b.accum + static_cast<size_t>(g) * kAccum;
    float* dm = b.d_means + 3 * g;
    float* ds = b.d_scales + 3 * g;
    float* dq = b.d_rotations + 4 * g;
    float* dsh = b.d_sh + static_cast<size_t>(g) * b.sh_bases * 3;
    dm[0] = dm[1] = dm[2] = 0.0f;
    ds[0] = ds[1] = ds[2] = 0.0f;
    dq[0] = dq[1] = dq[2] = dq[3] = 0.0f;
    b.d_opacities[g] = 0.0f;
    for (uint32_t i = 0; i < b.sh_bases * 3; ++i) dsh[i] = 0.0f;
    bool any = false;
    for (int i = 0; i < kAccum; ++i) any |= acc[i] != 0.0f;
    if (!any) return;

    const float mx = b.means[3 * g], my = b.means[3 * g + 1], mz = b.means[3 * g + 2];
    const float4 r1 = b.w2c[0], r2 = b.w2c[1], r3 = b.w2c[2];
    const float tx = r1.x * mx + r1.y * my + r1.z * mz + r1.w;
    const float ty = r2.x * mx + r2.y * my + r2.z * mz + r2.w;
    const float tz = r3.x * mx + r3.y * my + r3.z * mz + r3.w;
    const float x = tx / tz, y = ty / tz;
    const PassCamera& cam = b.cam;
    const float cl = (-0.15f * cam.width - cam.center_x) / cam.focal_x, cr = (1.15f * cam.width - cam.center_x) / cam.focal_x;
    const float ct = (-0.15f * cam.height - cam.center_y) / cam.focal_y, cb = (1.15f * cam.height - cam.center_y) / cam.focal_y;
    const float xc = fminf(fmaxf(x, cl), cr), yc = fminf(fmaxf(y, ct), cb);
    const bool free_x = x > cl && x < cr, free_y = y > ct && y < cb;
    // rotation of the normalised quaternion
    const float4 q = b.rotations[g];
    const float qnorm = sqrtf(q.x * q.x + q.y * q.y + q.z * q.z + q.w * q.w);
    const float w = q.x / qnorm, X = q.y / qnorm, Yq = q.z / qnorm, Z = q.w / qnorm;
    const float R[3][3] = {{1 - 2 * (Yq * Yq + Z * Z), 2 * (X * Yq - w * Z), 2 * (X * Z + w * Yq)},
                           {2 * (X * Yq + w * Z), 1 - 2 * (X * X + Z * Z), 2 * (Yq * Z - w * X)},
                           {2 * (X * Z - w * Yq), 2 * (Yq * Z + w * X), 1 - 2 * (X * X + Yq * Yq)}};
    const float v[3] = {expf(2.0f * b.scales[3 * g]), expf(2.0f * b.scales[3 * g + 1]), expf(2.0f * b.scales[3 * g + 2])};
    float S[3][3];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) S[i][j] = R[i][0] * v[0] * R[j][0] + R[i][1] * v[1] * R[j][1] + R[i][2] * v[2] * R[j][2];
    const float W3[3][3] = {{r1.x, r1.y, r1.z}, {r2.x, r2.y, r2.z}, {r3.x, r3.y, r3.z}};
    const float J[2][3] = {{cam.focal_x / tz, 0.0f, -cam.focal_x * xc / tz}, {0.0f, cam.focal_y / tz, -cam.focal_y * yc / tz}};
    float T[2][3];
    for (int i = 0; i < 2; ++i)
        for (int j = 0; j < 3; ++j) T[i][j] = J[i][0] * W3[0][j] + J[i][1] * W3[1][j] + J[i][2] * W3[2][j];
    float cov[2][2];
    for (int i = 0; i < 2; ++i)
        for (int j = 0; j < 2; ++j) {
            float s = 0.0f;
            for (int k = 0; k < 3; ++k)
                for (int l = 0; l < 3; ++l) s += T[i][k] * S[k][l] * T[j][l];
            cov[i][j] = s;
        }
    const float dil = (cam.proper_aa ? kDilationProperAA : kDilation) * cam.ss * cam.ss;
    const float a = cov[0][0] + dil, bb = cov[0][1], c = cov[1][1] + dil;
    const float det = a * c - bb * bb;
    const float C[2][2] = {{c / det, -bb / det}, {-bb / det, a / det}};
    const float op = 1.0f / (1.0f + expf(-b.opacities[g]));
    // proper antialiasing scales the opacity by f = sqrt(det_raw / det), det_raw of the undilated
    // covariance (gs_utils.h:165-166); acc[0] is the gradient w.r.t. that scaled opacity
    const float det_raw = cov[0][0] * cov[1][1] - cov[0][1] * cov[0][1];
    const float ratio = det_raw / det;
    const float f = cam.proper_aa ? sqrtf(fmaxf(ratio, 0.0f)) : 1.0f;

    // opacity logit
    b.d_opacities[g] = acc[0] * f * op * (1.0f - op);
    // conic = inverse(cov2d + dilation)
    const float G[2][2] = {{acc[1], 0.5f * acc[2]}, {0.5f * acc[2], acc[3]}};
    float CG[2][2], GA[2][2];
    for (int i = 0; i < 2; ++i)
        for (int j = 0; j < 2; ++j) CG[i][j] = C[i][0] * G[0][j] + C[i][1] * G[1][j];
    for (int i = 0; i < 2; ++i)
        for (int j = 0; j < 2; ++j) GA[i][j] = -(CG[i][0] * C[0][j] + CG[i][1] * C[1][j]);
    if (cam.proper_aa && ratio > 0.0f) {
        // f through the covariance: dr/dxx = (yy det - det_raw (yy + d)) / det^2 (likewise yy) and
        // dr/dxy = 2 xy (det_raw - det) / det^2, split over the two off-diagonal entries
        const float k = acc[0] * op / (2.0f * f) / (det * det);
        GA[0][0] += k * (cov[1][1] * det - det_raw * c);
        GA[1][1] += k * (cov[0][0] * det - det_raw * a);
        GA[0][1] += k * (bb * (det_raw - det));
        GA[1][0] += k * (bb * (det_raw - det));
    }
    float dS[3][3], dT[2][3];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            float s = 0.0f;
            for (int k = 0; k < 2; ++k)
                for (int l = 0; l < 2; ++l) s += T[k][i] * GA[k][l] * T[l][j];
            dS[i][j] = s;
        }
    for (int i = 0; i < 2; ++i)
        for (int j = 0; j < 3; ++j) {
            float s = 0.0f;
            for (int k = 0; k < 2; ++k)
                for (int l = 0; l < 3; ++l) s += GA[i][k] * T[k][l] * S[l][j];
            dT[i][j] = 2.0f * s;
        }
    float dJ[2][3];
    for (int i = 0; i < 2; ++i)
        for (int j = 0; j < 3; ++j) dJ[i][j] = dT[i][0] * W3[j][0] + dT[i][1] * W3[j][1] + dT[i][2] * W3[j][2];
    float dtz = acc[6];
    dtz += dJ[0][0] * (-cam.focal_x / (tz * tz)) + dJ[0][2] * (cam.focal_x * xc / (tz * tz)) +
           dJ[1][1] * (-cam.focal_y / (tz * tz)) + dJ[1][2] * (cam.focal_y * yc / (tz * tz));
    float dxv = acc[4] * cam.focal_x, dyv = acc[5] * cam.focal_y;
    if (free_x) dxv += dJ[0][2] * (-cam.focal_x / tz);
    if (free_y) dyv += dJ[1][2] * (-cam.focal_y / tz);
    const float dtx = dxv / tz, dty = dyv / tz;
    dtz -= dxv * tx / (tz * tz) + dyv * ty / (tz * tz);
    float gm[3];
    for (int i = 0; i < 3; ++i) gm[i] = W3[0][i] * dtx + W3[1][i] * dty + W3[2][i] * dtz;
    // covariance = R V R^T
    for (int i = 0; i < 3; ++i) {
        float s = 0.0f;
        for (int k = 0; k < 3; ++k)
            for (int l = 0; l < 3; ++l) s += R[k][i] * dS[k][l] * R[l][i];
        ds[i] = s * 2.0f * v[i];
    }
    float dR[3][3];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            float s = 0.0f;
            for (int k = 0; k < 3; ++k) s += (dS[i][k] + dS[k][i]) * R[k][j];
            dR[i][j] = s * v[j];
        }
    float dqn[4];
    dqn[0] = 2 * (-Z * dR[0][1] + Yq * dR[0][2] + Z * dR[1][0] - X * dR[1][2] - Yq * dR[2][0] + X * dR[2][1]);
    dqn[1] = 2 * (Yq * dR[0][1] + Z * dR[0][2] + Yq * dR[1][0] - 2 * X * dR[1][1] - w * dR[1][2] + Z * dR[2][0] +
                  w * dR[2][1] - 2 * X * dR[2][2]);
    dqn[2] = 2 * (-2 * Yq * dR[0][0] + X * dR[0][1] + w * dR[0][2] + X * dR[1][0] + Z * dR[1][2] - w * dR[2][0] +
                  Z * dR[2][1] - 2 * Yq * dR[2][2]);
    dqn[3] = 2 * (-2 * Z * dR[0][0] - w * dR[0][1] + X * dR[0][2] + w * dR[1][0] - 2 * Z * dR[1][1] + Yq * dR[1][2] +
                  X * dR[2][0] + Yq * dR[2][1]);
    const float dot = dqn[0] * w + dqn[1] * X + dqn[2] * Yq + dqn[3] * Z;
    dq[0] = (dqn[0] - w * dot) / qnorm;
    dq[1] = (dqn[1] - X * dot) / qnorm;
    dq[2] = (dqn[2] - Yq * dot) / qnorm;
    dq[3] = (dqn[3] - Z * dot) / qnorm;
    // colour = max(0.5 + sum Y_b sh_b, 0); direction = normalize(mean - camera)
    const float dvx = mx - b.cam_position[0], dvy = my - b.cam_position[1], dvz = mz - b.cam_position[2];
    const float len = sqrtf(dvx * dvx + dvy * dvy + dvz * dvz);
    const float dir[3] = {dvx / len, dvy / len, dvz / len};
    float Y[16], dY[16][3];
    sh_basis(dir[0], dir[1], dir[2], Y, dY);
    const float* shg = b.sh + static_cast<size_t>(g) * b.sh_bases * 3;
    const float* col = b.colors + 3 * g;
    float ddir[3] = {0.0f, 0.0f, 0.0f};
    for (int ch = 0; ch < 3; ++ch) {
        const float gc = col[ch] > 0.0f ? acc[7 + ch] : 0.0f;
        for (uint32_t k = 0; k < b.sh_bases; ++k) {
            dsh[3 * k + ch] = gc * Y[k];
            ddir[0] += gc * shg[3 * k + ch] * dY[k][0];
            ddir[1] += gc * shg[3 * k + ch] * dY[k][1];
            ddir[2] += gc * shg[3 * k + ch] * dY[k][2];
        }
    }
    const float dd = ddir[0] * dir[0] + ddir[1] * dir[1] + ddir[2] * dir[2];
    for (int k = 0; k < 3; ++k) dm[k] = gm[k] + (ddir[k] - dir[k] * dd) / len;
}

}  // namespace

cudaError_t launch_backward_colors(const BackwardParams& p, cudaStream_t stream) {
    if (p.n == 0) return cudaSuccess;
    colors_kernel<<<(p.n + kBlock - 1) / kBlock, kBlock, 0, stream>>>(p);
    return cudaGetLastError();
}

cudaError_t launch_backward_fragments(const BackwardParams& p, cudaStream_t stream) {
    if (p.n == 0) return cudaSuccess;
    fragments_backward_kernel<<<(p.n + kBlock - 1) / kBlock, kBlock, 0, stream>>>(p);
    return cudaGetLastError();
}

cudaError_t launch_backward_framebuffer_terms(const BackwardParams& p, cudaStream_t stream) {
    if (p.n_fb == 0) return cudaSuccess;
    framebuffer_terms_kernel<<<(p.n_fb + kBlock - 1) / kBlock, kBlock, 0, stream>>>(p);
    return cudaGetLastError();
}

cudaError_t launch_backward_sample_terms(const BackwardParams& p, cudaStream_t stream) {
    if (p.n_fb == 0) return cudaSuccess;
    sample_terms_kernel<<<(p.n_fb + kBlock - 1) / kBlock, kBlock, 0, stream>>>(p);
    return cudaGetLastError();
}

cudaError_t launch_backward_fragments_samples(const BackwardParams& p, cudaStream_t stream) {
    if (p.n == 0) return cudaSuccess;
    const unsigned grid = (p.n + kBlock - 1) / kBlock;
    const unsigned queue_grid = static_cast<unsigned>(max(p.num_sms, 1)) * kQueueBlocksPerSM;
    fragments_samples_kernel<false><<<grid, kBlock, 0, stream>>>(p, nullptr);
    fragments_samples_queue_kernel<false><<<queue_grid, kBlock, 0, stream>>>(p, nullptr);
    return cudaGetLastError();
}

cudaError_t launch_backward_fragments_samples_gps(const BackwardParams& p, float2* law, cudaStream_t stream) {
    if (p.n == 0) return cudaSuccess;
    if (law == nullptr) return cudaErrorInvalidValue;
    const unsigned grid = (p.n + kBlock - 1) / kBlock;
    const unsigned queue_grid = static_cast<unsigned>(max(p.num_sms, 1)) * kQueueBlocksPerSM;
    gps_count_law_kernel<<<kLawRows, 32, 0, stream>>>(law);
    fragments_samples_kernel<true><<<grid, kBlock, 0, stream>>>(p, law);
    fragments_samples_queue_kernel<true><<<queue_grid, kBlock, 0, stream>>>(p, law);
    return cudaGetLastError();
}

size_t gps_count_law_bytes() { return sizeof(float2) * static_cast<size_t>(kLawRows) * kLawTerms; }

cudaError_t launch_gps_count_law(float2* law, cudaStream_t stream) {
    gps_count_law_kernel<<<kLawRows, 32, 0, stream>>>(law);
    return cudaGetLastError();
}

cudaError_t launch_backward_projection(const BackwardParams& p, cudaStream_t stream) {
    if (p.n == 0) return cudaSuccess;
    projection_backward_kernel<<<(p.n + kBlock - 1) / kBlock, kBlock, 0, stream>>>(p);
    return cudaGetLastError();
}

}  // namespace sgs
