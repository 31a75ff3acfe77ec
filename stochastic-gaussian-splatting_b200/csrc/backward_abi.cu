// C ABI of the backward pass (include/sgs_b200.h): validation, the render workspace's buffers, and the
// launch sequence (colours once, one fragment pass per sample, projection backward at the end).
#include <cstdint>
#include <cuda_runtime.h>
#include "../../include/sgs_b200.h"
#include "sgs_backward_gps.h"
#include "sgs_internal.h"

namespace {

using namespace sgs;

constexpr size_t kAccumFloats = 10;

struct BackwardSetup {
    BackwardParams p;
    sgs_workspace_layout layout;
    bool gps;
    float2* gps_law;  // GPS: the count-law table in the sample scratch
};

int setup(const sgs_gaussians* g, const sgs_camera* c, const sgs_settings* s, BackwardSetup& out) {
    if (g == nullptr || c == nullptr || s == nullptr) return record_error(SGS_ERROR_INVALID_ARGUMENT, "null argument");
    if (s->spatial_reuse)
        return record_error(SGS_ERROR_INVALID_ARGUMENT, "the backward pass does not support spatial reuse");
    if (g->sh_bases != 1 && g->sh_bases != 4 && g->sh_bases != 9 && g->sh_bases != 16)
        return record_error(SGS_ERROR_INVALID_ARGUMENT, "sh_bases must be 1, 4, 9 or 16");
    if (g->quantized != nullptr)
        return record_error(SGS_ERROR_INVALID_ARGUMENT,
                            "the backward pass differentiates the float32 parameters, not the quantised layout");
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
    p.cam.proper_aa = s->proper_antialiasing;
    p.width = c->width;
    p.ss = ss;
    p.n_fb = c->width * ss * c->height * ss;
    out.gps = s->use_gps != 0;
    out.gps_law = nullptr;
    return SGS_OK;
}

constexpr uint32_t kMaxFusedSamples = 1024;

size_t align256(const size_t v) { return (v + 255) & ~size_t(255); }

// Interleaved per-pixel sample table of the fused backward: keys, then terms, the per-pixel largest
// key, and for GPS the count-law table (returned; null without GPS).
float2* set_sample_table(BackwardParams& p, void* scratch, const uint32_t n_samples, const bool gps) {
    p.n_samples = n_samples;
    p.pix_keys = static_cast<unsigned long long*>(scratch);
    const size_t keys = align256(sizeof(unsigned long long) * p.n_fb * static_cast<size_t>(n_samples));
    const size_t terms = align256(sizeof(float) * p.n_fb * static_cast<size_t>(n_samples));
    const size_t max_keys = align256(sizeof(unsigned long long) * p.n_fb);
    p.pix_terms = reinterpret_cast<float*>(static_cast<char*>(scratch) + keys);
    p.pix_max_key = reinterpret_cast<unsigned long long*>(static_cast<char*>(scratch) + keys + terms);
    return gps ? reinterpret_cast<float2*>(static_cast<char*>(scratch) + keys + terms + max_keys) : nullptr;
}

cudaError_t launch_walk(const BackwardSetup& S, cudaStream_t stream) {
    return S.gps ? launch_backward_fragments_samples_gps(S.p, S.gps_law, stream)
                 : launch_backward_fragments_samples(S.p, stream);
}

// Entries of the large-Gaussian queue of the fused walk (at most 2^18).
uint32_t queue_capacity(const uint32_t n) { return n < (1u << 18) ? n : (1u << 18); }
constexpr size_t kWalkGaussianBytes = 128;  // walk constants (96) and GPS constants (32)

// Backward workspace: colours (3 per Gaussian, padded to 4), accumulators (10 per Gaussian), then
// the fused walk's queue (header, entries, meta, indices), each section 256-byte aligned.
struct BackwardLayout {
    size_t colors, accum, queue, entries, meta, index, total;
};

BackwardLayout backward_layout(const uint32_t n) {
    BackwardLayout L{};
    const size_t cap = queue_capacity(n);
    L.colors = 0;
    L.accum = align256(sizeof(float) * ((3 * static_cast<size_t>(n) + 3) & ~size_t(3)));
    L.queue = L.accum + align256(sizeof(float) * kAccumFloats * n);
    L.entries = L.queue + align256(sizeof(WorkQueue));
    L.meta = L.entries + align256(kWalkGaussianBytes * cap);
    L.index = L.meta + align256(sizeof(uint4) * cap);
    L.total = L.index + align256(sizeof(uint32_t) * cap);
    return L;
}

void set_backward_buffers(BackwardParams& p, void* backward_workspace) {
    char* base = static_cast<char*>(backward_workspace);
    const BackwardLayout L = backward_layout(p.n);
    p.colors = reinterpret_cast<float*>(base + L.colors);
    p.accum = reinterpret_cast<float*>(base + L.accum);
    p.bw_queue = reinterpret_cast<WorkQueue*>(base + L.queue);
    p.bw_entries = base + L.entries;
    p.bw_meta = reinterpret_cast<uint4*>(base + L.meta);
    p.bw_index = reinterpret_cast<uint32_t*>(base + L.index);
    p.bw_capacity = queue_capacity(p.n);
}

}  // namespace

extern "C" {

size_t sgs_backward_workspace_size(uint32_t n_gaussians) { return backward_layout(n_gaussians).total; }

int sgs_backward_accumulate(const sgs_gaussians* gaussians, const sgs_camera* camera, const sgs_settings* settings,
                            const void* render_workspace, const float* grad_image, const float* grad_alpha,
                            const float* grad_depth, float weight, int first, void* backward_workspace,
                            void* stream_ptr) {
    BackwardSetup S;
    int st = setup(gaussians, camera, settings, S);
    if (st != SGS_OK) return st;
    if (S.gps)
        return record_error(SGS_ERROR_INVALID_ARGUMENT,
                            "GPS gradients use the fused walk (sgs_backward_accumulate_samples or "
                            "sgs_backward_accumulate_framebuffers)");
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

size_t sgs_backward_samples_scratch_size(const sgs_camera* camera, const sgs_settings* settings,
                                         uint32_t n_samples) {
    if (camera == nullptr || settings == nullptr || n_samples == 0 || n_samples > kMaxFusedSamples) return 0;
    const uint32_t ss = settings->supersampling_factor < 1 ? 1u : static_cast<uint32_t>(settings->supersampling_factor);
    const size_t n_fb = static_cast<size_t>(camera->width) * ss * camera->height * ss;
    return align256(sizeof(unsigned long long) * n_fb * n_samples) + align256(sizeof(float) * n_fb * n_samples) +
           align256(sizeof(unsigned long long) * n_fb) + (settings->use_gps ? align256(gps_count_law_bytes()) : 0);
}

size_t sgs_gps_count_law_size(void) { return gps_count_law_bytes(); }

int sgs_gps_count_law(void* out, void* stream_ptr) {
    if (out == nullptr || (reinterpret_cast<uintptr_t>(out) & 7u) != 0)
        return record_error(SGS_ERROR_INVALID_ARGUMENT, "the count-law table needs an 8-byte aligned device buffer");
    const cudaError_t err = launch_gps_count_law(static_cast<float2*>(out), static_cast<cudaStream_t>(stream_ptr));
    if (err != cudaSuccess) return record_error(SGS_ERROR_CUDA, "count law: %s", cudaGetErrorString(err));
    return SGS_OK;
}

int sgs_backward_sample_terms(const sgs_gaussians* gaussians, const sgs_camera* camera, const sgs_settings* settings,
                              const void* render_workspace, const float* grad_image, const float* grad_alpha,
                              const float* grad_depth, float weight, uint32_t sample, uint32_t n_samples,
                              void* scratch, void* stream_ptr) {
    BackwardSetup S;
    int st = setup(gaussians, camera, settings, S);
    if (st != SGS_OK) return st;
    if (render_workspace == nullptr || grad_image == nullptr || scratch == nullptr ||
        (reinterpret_cast<uintptr_t>(scratch) & 255u) != 0)
        return record_error(SGS_ERROR_INVALID_ARGUMENT,
                            "null render workspace or image gradient, or scratch not 256-byte aligned");
    if (n_samples == 0 || n_samples > kMaxFusedSamples || sample >= n_samples)
        return record_error(SGS_ERROR_INVALID_ARGUMENT, "sample %u of %u (at most %u samples)", sample, n_samples,
                            kMaxFusedSamples);
    BackwardParams& p = S.p;
    const char* ws = static_cast<const char*>(render_workspace);
    p.framebuffer = reinterpret_cast<const unsigned long long*>(ws + S.layout.framebuffer);
    p.samples = reinterpret_cast<const float4*>(ws + S.layout.samples);
    p.grad_image = grad_image;
    p.grad_alpha = grad_alpha;
    p.grad_depth = grad_depth;
    p.grad_scale = weight / static_cast<float>(p.ss * p.ss);
    S.gps_law = set_sample_table(p, scratch, n_samples, S.gps);
    p.sample = sample;
    const cudaError_t err = launch_backward_sample_terms(p, static_cast<cudaStream_t>(stream_ptr));
    if (err != cudaSuccess) return record_error(SGS_ERROR_CUDA, "backward: %s", cudaGetErrorString(err));
    return SGS_OK;
}

int sgs_backward_accumulate_samples(const sgs_gaussians* gaussians, const sgs_camera* camera,
                                    const sgs_settings* settings, const float* grad_image, const float* grad_alpha,
                                    const float* grad_depth, float weight, uint32_t n_samples, int first,
                                    void* scratch, void* backward_workspace, void* stream_ptr) {
    BackwardSetup S;
    int st = setup(gaussians, camera, settings, S);
    if (st != SGS_OK) return st;
    if (grad_image == nullptr || scratch == nullptr || backward_workspace == nullptr ||
        (reinterpret_cast<uintptr_t>(scratch) & 255u) != 0 || (reinterpret_cast<uintptr_t>(backward_workspace) & 15u) != 0)
        return record_error(SGS_ERROR_INVALID_ARGUMENT,
                            "null image gradient, scratch or backward workspace, or misaligned buffers");
    if (n_samples == 0 || n_samples > kMaxFusedSamples)
        return record_error(SGS_ERROR_INVALID_ARGUMENT, "%u samples (1 to %u)", n_samples, kMaxFusedSamples);
    cudaStream_t stream = static_cast<cudaStream_t>(stream_ptr);
    BackwardParams& p = S.p;
    p.grad_image = grad_image;
    p.grad_alpha = grad_alpha;
    p.grad_depth = grad_depth;
    p.grad_scale = weight / static_cast<float>(p.ss * p.ss);
    S.gps_law = set_sample_table(p, scratch, n_samples, S.gps);
    set_backward_buffers(p, backward_workspace);
    cudaError_t err = cudaSuccess;
    if (first) {
        err = cudaMemsetAsync(p.accum, 0, kAccumFloats * p.n * sizeof(float), stream);
        if (err == cudaSuccess) err = launch_backward_colors(p, stream);
    }
    if (err == cudaSuccess) err = cudaMemsetAsync(p.bw_queue, 0, sizeof(WorkQueue), stream);
    if (err == cudaSuccess) {
        int device = 0;
        err = cudaGetDevice(&device);
        if (err == cudaSuccess) err = cudaDeviceGetAttribute(&p.num_sms, cudaDevAttrMultiProcessorCount, device);
    }
    if (err == cudaSuccess) err = launch_walk(S, stream);
    if (err != cudaSuccess) return record_error(SGS_ERROR_CUDA, "backward: %s", cudaGetErrorString(err));
    return SGS_OK;
}

int sgs_backward_accumulate_framebuffers(const sgs_gaussians* gaussians, const sgs_camera* camera,
                                         const sgs_settings* settings, const void* framebuffers, uint32_t n_samples,
                                         const float* grad_image, const float* grad_alpha, const float* grad_depth,
                                         float weight, int first, void* scratch, void* backward_workspace,
                                         void* stream_ptr) {
    BackwardSetup S;
    int st = setup(gaussians, camera, settings, S);
    if (st != SGS_OK) return st;
    if (framebuffers == nullptr || grad_image == nullptr || scratch == nullptr || backward_workspace == nullptr ||
        (reinterpret_cast<uintptr_t>(framebuffers) & 7u) != 0 || (reinterpret_cast<uintptr_t>(scratch) & 255u) != 0 ||
        (reinterpret_cast<uintptr_t>(backward_workspace) & 15u) != 0)
        return record_error(SGS_ERROR_INVALID_ARGUMENT,
                            "null framebuffers, image gradient, scratch or backward workspace, or misaligned buffers");
    if (n_samples == 0 || n_samples > kMaxFusedSamples)
        return record_error(SGS_ERROR_INVALID_ARGUMENT, "%u samples (1 to %u)", n_samples, kMaxFusedSamples);
    cudaStream_t stream = static_cast<cudaStream_t>(stream_ptr);
    BackwardParams& p = S.p;
    p.framebuffer = static_cast<const unsigned long long*>(framebuffers);
    p.grad_image = grad_image;
    p.grad_alpha = grad_alpha;
    p.grad_depth = grad_depth;
    p.grad_scale = weight / static_cast<float>(p.ss * p.ss);
    S.gps_law = set_sample_table(p, scratch, n_samples, S.gps);
    set_backward_buffers(p, backward_workspace);
    cudaError_t err = cudaSuccess;
    if (first) err = cudaMemsetAsync(p.accum, 0, kAccumFloats * p.n * sizeof(float), stream);
    if (err == cudaSuccess) err = launch_backward_colors(p, stream);
    if (err == cudaSuccess) err = launch_backward_framebuffer_terms(p, stream);
    if (err == cudaSuccess) err = cudaMemsetAsync(p.bw_queue, 0, sizeof(WorkQueue), stream);
    if (err == cudaSuccess) {
        int device = 0;
        err = cudaGetDevice(&device);
        if (err == cudaSuccess) err = cudaDeviceGetAttribute(&p.num_sms, cudaDevAttrMultiProcessorCount, device);
    }
    if (err == cudaSuccess) err = launch_walk(S, stream);
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
