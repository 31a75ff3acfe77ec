// Test-only harness around the reference CUDA backend (StochasticGSCudaBackend).
//
// This file is ORACLE infrastructure: it is compiled by oracle/build_ref.py together with the
// reference's own, unmodified kernel sources (accumulate_scatter.cu, accumulate_hybrid.cu,
// accumulate_hybrid_gps.cu, resolve.cu) into oracle/_ref/. It never ships with the product.
// The reference's `_C.render` (render.cu:16-158) returns only the resolved image, so this harness
// calls the reference's own host launchers directly to expose the intermediate buffers that the
// parity tests compare bit for bit:
//   accumulate()       -> the packed (depth_bits << 32 | index) winner framebuffer
//                         (render.cu:65-67 allocation/clear, render.cu:85-125 dispatch)
//   sample_resolve()   -> samples, reuse weights and the four outputs (resolve.cu:355-444)
//   project()          -> per-Gaussian projection results of gs_utils.h:38-193
// Frame indices are explicit arguments here instead of render.cu:56-57's process-global counter.
#include <cstdint>
#include <ATen/cuda/CUDAContext.h>
#include <c10/cuda/CUDAGuard.h>
#include <torch/extension.h>
#include <cooperative_groups.h>
#include "helper_math.h"
#include "math_utils.h"
#include "gs_utils.h"
#include "render_utils.h"
#include "accumulate_scatter.h"
#include "accumulate_hybrid.h"
#include "accumulate_hybrid_gps.h"
#include "resolve.h"

namespace cg = cooperative_groups;

namespace {

CameraSettings make_camera(uint32_t width, uint32_t height, float fx, float fy, float cx, float cy, float near_plane,
                           float far_plane, bool proper_antialiasing, int ss) {
    return CameraSettings{width, height, fx, fy, cx, cy, near_plane, far_plane, proper_antialiasing,
                          static_cast<uint32_t>(std::max(1, ss))};
}

torch::Tensor accumulate(const torch::Tensor& means, const torch::Tensor& scales, const torch::Tensor& rotations,
                         const torch::Tensor& opacities, const torch::Tensor& w2c, uint32_t width, uint32_t height,
                         float fx, float fy, float cx, float cy, float near_plane, float far_plane,
                         bool proper_antialiasing, int ss, bool use_gps, bool hybrid_scheduling,
                         const torch::Tensor& blue_noise, uint32_t frame_idx) {
    const at::cuda::CUDAGuard guard(means.device());
    auto stream = at::cuda::getCurrentCUDAStream();
    const CameraSettings camera = make_camera(width, height, fx, fy, cx, cy, near_plane, far_plane, proper_antialiasing, ss);
    const uint32_t n = means.size(0);
    const int64_t n_fb = static_cast<int64_t>(width) * height * camera.supersampling_factor * camera.supersampling_factor;
    auto fb = torch::empty({n_fb}, torch::TensorOptions().dtype(torch::kLong).device(means.device()));
    auto* fb_ptr = reinterpret_cast<unsigned long long*>(fb.data_ptr<int64_t>());
    cudaMemsetAsync(fb_ptr, 0xff, sizeof(unsigned long long) * n_fb, stream);
    auto m = means.contiguous(), s = scales.contiguous(), r = rotations.contiguous(), o = opacities.contiguous(),
         w = w2c.contiguous(), bn = blue_noise.contiguous();
    const bool use_bn = bn.numel() > 0;
    const uint8_t* slice = use_bn ? bn.data_ptr<uint8_t>() + (frame_idx % blue_noise_depth) * blue_noise_width * blue_noise_height : nullptr;
    const uint32_t rotation = (frame_idx / blue_noise_depth) * 0x9E3779B9u;
    auto* mp = reinterpret_cast<const float3*>(m.data_ptr<float>());
    auto* sp = reinterpret_cast<const float3*>(s.data_ptr<float>());
    auto* rp = reinterpret_cast<const float4*>(r.data_ptr<float>());
    auto* op = o.data_ptr<float>();
    auto* wp = reinterpret_cast<const float4*>(w.data_ptr<float>());
    if (hybrid_scheduling && use_gps) accumulate_hybrid_gps(mp, sp, rp, op, wp, fb_ptr, n, frame_idx, camera, stream);
    else if (hybrid_scheduling) accumulate_hybrid(mp, sp, rp, op, wp, fb_ptr, n, frame_idx, camera, slice, rotation, stream);
    else accumulate_scatter(mp, sp, rp, op, wp, fb_ptr, n, frame_idx, camera, use_gps, slice, rotation, stream);
    return fb;
}

std::vector<torch::Tensor> sample_resolve(
    const torch::Tensor& means, const torch::Tensor& scales, const torch::Tensor& rotations,
    const torch::Tensor& opacities, const torch::Tensor& sh, const torch::Tensor& w2c, const torch::Tensor& cam_position,
    uint32_t width, uint32_t height, float fx, float fy, float cx, float cy, float near_plane, float far_plane,
    bool proper_antialiasing, int ss, bool spatial_reuse, const torch::Tensor& framebuffer,
    const torch::Tensor& k_buffer_primitives, const torch::Tensor& k_buffer_occlusion,
    const torch::Tensor& history_image, const torch::Tensor& history_depth, const torch::Tensor& history_alpha,
    const torch::Tensor& history_weight_mass, const torch::Tensor& view_to_previous_view, int temporal_mode) {
    const at::cuda::CUDAGuard guard(means.device());
    auto stream = at::cuda::getCurrentCUDAStream();
    const CameraSettings camera = make_camera(width, height, fx, fy, cx, cy, near_plane, far_plane, proper_antialiasing, ss);
    const int64_t n_fb = static_cast<int64_t>(width) * height * camera.supersampling_factor * camera.supersampling_factor;
    auto opts = torch::TensorOptions().dtype(torch::kFloat).device(means.device());
    auto image = torch::empty({height, width, 3}, opts);
    auto depth = torch::empty({height, width, 1}, opts);
    auto alpha = torch::empty({height, width, 1}, opts);
    auto weight_mass = torch::empty({height, width, 1}, opts);
    auto samples = torch::empty({n_fb, 4}, opts);
    auto reuse = torch::empty({spatial_reuse ? n_fb : 0, 4}, opts);
    auto m = means.contiguous(), s = scales.contiguous(), r = rotations.contiguous(), o = opacities.contiguous(),
         shc = sh.contiguous(), w = w2c.contiguous(), cp = cam_position.contiguous(), v = view_to_previous_view.contiguous();
    sample_and_resolve(
        reinterpret_cast<const float3*>(m.data_ptr<float>()), reinterpret_cast<const float3*>(s.data_ptr<float>()),
        reinterpret_cast<const float4*>(r.data_ptr<float>()), o.data_ptr<float>(),
        reinterpret_cast<const float3*>(shc.data_ptr<float>()), reinterpret_cast<const float4*>(w.data_ptr<float>()),
        reinterpret_cast<const float3*>(cp.data_ptr<float>()),
        reinterpret_cast<const unsigned long long*>(framebuffer.data_ptr<int64_t>()),
        reinterpret_cast<float4*>(samples.data_ptr<float>()), reinterpret_cast<float4*>(reuse.data_ptr<float>()),
        reinterpret_cast<uint2*>(k_buffer_primitives.data_ptr<int>()),
        reinterpret_cast<float4*>(k_buffer_occlusion.data_ptr<float>()),
        reinterpret_cast<const float3*>(history_image.data_ptr<float>()), history_depth.data_ptr<float>(),
        history_alpha.data_ptr<float>(), history_weight_mass.data_ptr<float>(),
        reinterpret_cast<const float4*>(v.data_ptr<float>()),
        reinterpret_cast<float3*>(image.data_ptr<float>()), depth.data_ptr<float>(), alpha.data_ptr<float>(),
        weight_mass.data_ptr<float>(), static_cast<uint32_t>(sh.size(1)), camera, spatial_reuse,
        static_cast<TemporalMode>(temporal_mode), stream);
    return {samples, reuse, image, depth, alpha, weight_mass};
}

// one thread per Gaussian, runs the reference's project_gaussian and stores every output
__global__ void project_cu(const float3* means, const float3* scales, const float4* rotations, const float* opacities,
                           const float4* w2c, float* out, uint32_t n, float width, float height, float fx, float fy,
                           float cx, float cy, float near_plane, float far_plane, bool proper_antialiasing, float ss) {
    auto block = cg::this_thread_block();
    auto warp = cg::tiled_partition<32>(block);
    const uint32_t idx = cg::this_grid().thread_rank();
    bool active = idx < n;
    const uint32_t g = active ? idx : n - 1;
    float depth = 0, opacity = 0, determinant = 0, power_threshold = 0;
    float2 mean2d = make_float2(0.0f);
    float3 conic = make_float3(0.0f), cov2d = make_float3(0.0f);
    float4 bounds = make_float4(0.0f);
    const bool any = project_gaussian(warp, active, g, means, scales, rotations, opacities, w2c, width, height, fx, fy, cx,
                                      cy, near_plane, far_plane, proper_antialiasing, ss, depth, opacity, determinant,
                                      power_threshold, mean2d, conic, cov2d, bounds);
    if (idx >= n) return;
    float* o = out + static_cast<size_t>(idx) * 18;
    o[0] = (any && active) ? 1.0f : 0.0f;
    o[1] = depth; o[2] = opacity; o[3] = determinant; o[4] = power_threshold;
    o[5] = mean2d.x; o[6] = mean2d.y; o[7] = conic.x; o[8] = conic.y; o[9] = conic.z;
    o[10] = cov2d.x; o[11] = cov2d.y; o[12] = cov2d.z;
    o[13] = bounds.x; o[14] = bounds.y; o[15] = bounds.z; o[16] = bounds.w; o[17] = any ? 1.0f : 0.0f;
}

torch::Tensor project(const torch::Tensor& means, const torch::Tensor& scales, const torch::Tensor& rotations,
                      const torch::Tensor& opacities, const torch::Tensor& w2c, uint32_t width, uint32_t height,
                      float fx, float fy, float cx, float cy, float near_plane, float far_plane,
                      bool proper_antialiasing, int ss) {
    const at::cuda::CUDAGuard guard(means.device());
    auto stream = at::cuda::getCurrentCUDAStream();
    const uint32_t n = means.size(0);
    const float s = static_cast<float>(std::max(1, ss));
    auto out = torch::zeros({static_cast<int64_t>(n), 18}, torch::TensorOptions().dtype(torch::kFloat).device(means.device()));
    auto m = means.contiguous(), sc = scales.contiguous(), r = rotations.contiguous(), o = opacities.contiguous(), w = w2c.contiguous();
    project_cu<<<(n + 255) / 256, 256, 0, stream>>>(
        reinterpret_cast<const float3*>(m.data_ptr<float>()), reinterpret_cast<const float3*>(sc.data_ptr<float>()),
        reinterpret_cast<const float4*>(r.data_ptr<float>()), o.data_ptr<float>(),
        reinterpret_cast<const float4*>(w.data_ptr<float>()), out.data_ptr<float>(), n,
        static_cast<float>(width * std::max(1, ss)), static_cast<float>(height * std::max(1, ss)), fx * s, fy * s, cx * s,
        cy * s, near_plane, far_plane, proper_antialiasing, s);
    return out;
}

}  // namespace

PYBIND11_MODULE(TORCH_EXTENSION_NAME, m) {
    m.def("accumulate", &accumulate);
    m.def("sample_resolve", &sample_resolve);
    m.def("project", &project);
}
