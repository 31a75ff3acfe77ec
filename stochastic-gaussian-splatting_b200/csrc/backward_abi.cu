// C ABI of the backward pass (include/sgs_b200.h): validation, the render workspace's buffers, and the
// launch sequence (colours once, one fragment pass per sample, projection backward at the end).
#include <cstdint>
#include <cuda_runtime.h>
#include "../../include/sgs_b200.h"
#include "sgs_internal.h"

namespace {

using namespace sgs;

constexpr size_t kAccumFloats = 10;

struct BackwardSetup {
    BackwardParams p;
    sgs_workspace_layout layout;
};

int setup(const sgs_gaussians* g, const sgs_camera* c, const sgs_settings* s, BackwardSetup& out) {
    if (g == nullptr || c == nullptr || s == nullptr) return record_error(SGS_ERROR_INVALID_ARGUMENT, "null argument");
    if (s->use_gps || s->spatial_reuse || s->proper_antialiasing)
        return record_error(SGS_ERROR_INVALID_ARGUMENT,
                            "the backward pass supports stochastic transparency without spatial reuse or proper "
                            "antialiasing");
    if (g->sh_bases != 1 && g->sh_bases != 4 && g->sh_bases != 9 && g->sh_bases != 16)
        return record_error(SGS_ERROR_INVALID_ARGUMENT, "sh_bases must be 1, 4, 9 or 16");
    if (g->n_gaussians > 0 && (!g->means || !g->scales || !g->rotations || !g->opacities || !g->sh_coefficients))
        return record_error(SGS_ERROR_INVALID_ARGUMENT, "null Gaussian array");
    if (!c->w2c || !c->cam_position) return record_error(SGS_ERROR_INVALID_ARGUMENT, "null camera array");
    const int st = sgs_get_workspace_layout(g, c, s, &out.layout);
    if (st != SGS_OK) return st;
    const uint32_t ss = s->supersampling_factor < 1 ? 1u : static_cast<uint32_t>(s->supersampling_factor);
    const float ssf = static_cast<float>(ss);
    BackwardParams& p = out.p;
    p = BackwardParams{};
    p.means = g->means;
    p.scales = g->scales;
    p.rotations = reinterpret_cast<const float4*>(g->rotations);
    p.opacities = g->opacities;
    p.sh = g->sh_coefficients;
    p.w2c = reinterpret_cast<const float4*>(c->w2c);
    p.cam_position = c->cam_position;
    p.n = g->n_gaussians;
    p.sh_bases = g->sh_bases;
    p.cam.width = static_cast<float>(c->width * ss);
    p.cam.height = static_cast<float>(c->height * ss);
    p.cam.focal_x = c->focal_x * ssf;
    p.cam.focal_y = c->focal_y * ssf;
    p.cam.center_x = c->center_x * ssf;
    p.cam.center_y = c->center_y * ssf;
    p.cam.near_plane = c->near_plane;
    p.cam.far_plane = c->far_plane;
    p.cam.ss = ssf;
    p.cam.width_int = c->width * ss;
    p.cam.proper_aa = false;
    p.width = c->width;
    p.ss = ss;
    return SGS_OK;
}

void set_backward_buffers(BackwardParams& p, void* backward_workspace) {
    float* base = static_cast<float*>(backward_workspace);
    p.colors = base;
    p.accum = base + ((3 * static_cast<size_t>(p.n) + 3) & ~size_t(3));
}

}  // namespace

extern "C" {

size_t sgs_backward_workspace_size(uint32_t n_gaussians) {
    const size_t colors = (3 * static_cast<size_t>(n_gaussians) + 3) & ~size_t(3);
    return (colors + kAccumFloats * n_gaussians) * sizeof(float);
}

int sgs_backward_accumulate(const sgs_gaussians* gaussians, const sgs_camera* camera, const sgs_settings* settings,
                            const void* render_workspace, const float* grad_image, const float* grad_alpha,
                            const float* grad_depth, float weight, int first, void* backward_workspace,
                            void* stream_ptr) {
    BackwardSetup S;
    int st = setup(gaussians, camera, settings, S);
    if (st != SGS_OK) return st;
    if (render_workspace == nullptr || grad_image == nullptr || backward_workspace == nullptr ||
        (reinterpret_cast<uintptr_t>(backward_workspace) & 15u) != 0)
        return record_error(SGS_ERROR_INVALID_ARGUMENT, "null render workspace, image gradient or backward workspace");
    cudaStream_t stream = static_cast<cudaStream_t>(stream_ptr);
    BackwardParams& p = S.p;
    const char* ws = static_cast<const char*>(render_workspace);
    p.framebuffer = reinterpret_cast<const unsigned long long*>(ws + S.layout.framebuffer);
    p.samples = reinterpret_cast<const float4*>(ws + S.layout.samples);
    p.grad_image = grad_image;
    p.grad_alpha = grad_alpha;
    p.grad_depth = grad_depth;
    p.grad_scale = weight / static_cast<float>(p.ss * p.ss);
    set_backward_buffers(p, backward_workspace);
    cudaError_t err = cudaSuccess;
    if (first) {
        err = cudaMemsetAsync(p.accum, 0, kAccumFloats * p.n * sizeof(float), stream);
        if (err == cudaSuccess) err = launch_backward_colors(p, stream);
    }
    if (err == cudaSuccess) err = launch_backward_fragments(p, stream);
    if (err != cudaSuccess) return record_error(SGS_ERROR_CUDA, "backward: %s", cudaGetErrorString(err));
    return SGS_OK;
}

int sgs_backward_finish(const sgs_gaussians* gaussians, const sgs_camera* camera, const sgs_settings* settings,
                        void* backward_workspace, float* d_means, float* d_scales, float* d_rotations,
                        float* d_opacities, float* d_sh, void* stream_ptr) {
    BackwardSetup S;
    int st = setup(gaussians, camera, settings, S);
    if (st != SGS_OK) return st;
    if (backward_workspace == nullptr || !d_means || !d_scales || !d_rotations || !d_opacities || !d_sh)
        return record_error(SGS_ERROR_INVALID_ARGUMENT, "null gradient output or backward workspace");
    BackwardParams& p = S.p;
    set_backward_buffers(p, backward_workspace);
    p.d_means = d_means;
    p.d_scales = d_scales;
    p.d_rotations = d_rotations;
    p.d_opacities = d_opacities;
    p.d_sh = d_sh;
    const cudaError_t err = launch_backward_projection(p, static_cast<cudaStream_t>(stream_ptr));
    if (err != cudaSuccess) return record_error(SGS_ERROR_CUDA, "backward: %s", cudaGetErrorString(err));
    return SGS_OK;
}

}  // extern "C"
