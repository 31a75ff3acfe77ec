// C ABI of the render path (include/sgs_b200.h): argument validation, workspace layout, the
// process-wide frame index and the launch sequence of one sample-frame.
//
// Host orchestration follows render.cu:16-158 of the reference: clear the framebuffer, pick the
// accumulate variant (GPS or ST, scatter or hybrid), then sample and resolve. Differences by
// design: outputs and scratch come from the caller (no allocation inside), the frame counter is
// atomic and settable, all inputs are validated, and no path synchronises with the host (the
// reference's hybrid paths read device counts back twice per call).
#include <atomic>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <cuda_runtime.h>
#include "../../include/sgs_b200.h"
#include "sgs_internal.h"

namespace {

using namespace sgs;

std::atomic<uint32_t> g_frame_index{0};
thread_local std::string t_last_error;
// optional accumulate-stage events (sgs_set_stage_events)
thread_local cudaEvent_t t_stage_start = nullptr;
thread_local cudaEvent_t t_stage_end = nullptr;
// optional cap on the stochastic-transparency large-Gaussian queue (sgs_set_queue_limit), 0 = none
std::atomic<uint32_t> g_queue_limit{0};

constexpr size_t kAlign = 256;
constexpr uint32_t kDefaultMaxBinned = 1u << 20;     // accumulate_hybrid_gps.cu:22
constexpr uint32_t kStQueueCapacity = 1u << 18;       // large ST Gaussians held by the queue
constexpr uint32_t kMaxSamplesPerCall = 1024;         // sgs_render_samples
constexpr int kMaxDevices = 64;
std::atomic<int> g_sm_count[kMaxDevices];

int fail(const int status, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    t_last_error = buf;
    return status;
}

size_t align_up(const size_t v) { return (v + kAlign - 1) / kAlign * kAlign; }

bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

uint32_t clamp_ss(const int32_t ss) { return ss < 1 ? 1u : static_cast<uint32_t>(ss); }

struct Derived {
    uint32_t ss;
    uint64_t n_fb;
    uint64_t n_pixels;
    uint32_t queue_capacity;
    uint32_t max_binned;
};

// Validates the arguments that determine sizes; fills the derived sizes.
int derive(const sgs_gaussians* g, const sgs_camera* c, const sgs_settings* s, Derived& d) {
    if (g == nullptr || c == nullptr || s == nullptr) return fail(SGS_ERROR_INVALID_ARGUMENT, "null argument struct");
    if (c->width == 0 || c->height == 0) return fail(SGS_ERROR_INVALID_ARGUMENT, "image size must be positive");
    d.ss = clamp_ss(s->supersampling_factor);
    const uint64_t fbw = static_cast<uint64_t>(c->width) * d.ss;
    const uint64_t fbh = static_cast<uint64_t>(c->height) * d.ss;
    if (fbw >= (1u << 24) || fbh >= (1u << 24))
        return fail(SGS_ERROR_INVALID_ARGUMENT, "framebuffer side must be below 2^24 (exact float coordinates)");
    d.n_fb = fbw * fbh;
    if (d.n_fb > 0xffffffffull) return fail(SGS_ERROR_INVALID_ARGUMENT, "framebuffer must have fewer than 2^32 pixels");
    d.n_pixels = static_cast<uint64_t>(c->width) * c->height;
    d.queue_capacity = 0;
    d.max_binned = 0;
    if (g->n_gaussians > 0) {
        if (s->use_gps) {
            if (s->hybrid_scheduling) {
                d.max_binned = s->max_binned != 0 ? s->max_binned : std::min(g->n_gaussians, kDefaultMaxBinned);
                d.max_binned = std::min(d.max_binned, g->n_gaussians);
                // an entry whose chunks would pass 32-bit chunk indices is not binned (the producer
                // marks it and scatters its Gaussian), so the queue holds max_binned entries like the
                // reference's bin
                d.queue_capacity = d.max_binned;
            }
        } else {
            // the Gaussians the reference's hybrid pass gathers (accumulate_hybrid.cu:27,345)
            if (s->hybrid_scheduling)
                d.max_binned = std::min(s->max_binned != 0 ? s->max_binned : kDefaultMaxBinned, g->n_gaussians);
            d.queue_capacity = std::min(g->n_gaussians, kStQueueCapacity);
            const uint32_t cap = g_queue_limit.load(std::memory_order_relaxed);
            if (cap != 0) d.queue_capacity = std::min(d.queue_capacity, cap);
            const uint64_t limit = 0xffffffffull / std::max<uint64_t>(fbh, 1);
            if (d.queue_capacity > limit) d.queue_capacity = static_cast<uint32_t>(limit);
        }
    }
    return SGS_OK;
}

struct FullLayout {
    sgs_workspace_layout pub;
    size_t q_key, q_geom, q_geom2, q_meta, q_count;
};

FullLayout make_layout(const Derived& d, const sgs_settings* s, const uint32_t n_samples = 1) {
    FullLayout F{};
    sgs_workspace_layout& L = F.pub;
    size_t off = 0;
    L.queue = off;
    off = align_up(off + sizeof(WorkQueue));
    L.framebuffer = off;  // n_samples framebuffers of n_fb keys, back to back
    off = align_up(off + d.n_fb * n_samples * sizeof(unsigned long long));
    L.samples = off;
    off = align_up(off + d.n_fb * sizeof(float4));
    L.reuse_weights = off;
    if (s->spatial_reuse) off = align_up(off + d.n_fb * sizeof(float4));
    const size_t q = d.queue_capacity;
    F.q_key = off;
    off = align_up(off + q * sizeof(unsigned long long));
    F.q_geom = off;
    off = align_up(off + q * sizeof(float4));
    F.q_geom2 = off;
    off = align_up(off + q * sizeof(float4));
    F.q_meta = off;
    off = align_up(off + q * sizeof(uint4));
    F.q_count = off;
    off = align_up(off + q * sizeof(uint32_t));
    L.total = off;
    return F;
}

int sm_count() {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0) return 148;
    if (dev >= kMaxDevices) {
        int n = 0;
        cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
        return n > 0 ? n : 148;
    }
    int n = g_sm_count[dev].load(std::memory_order_relaxed);
    if (n == 0) {
        cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
        if (n <= 0) n = 148;
        g_sm_count[dev].store(n, std::memory_order_relaxed);
    }
    return n;
}

PassCamera pass_camera(const sgs_camera* c, const sgs_settings* s, const uint32_t ss) {
    const float ssf = static_cast<float>(ss);
    PassCamera cam;
    cam.width = static_cast<float>(c->width * ss);
    cam.height = static_cast<float>(c->height * ss);
    cam.focal_x = c->focal_x * ssf;
    cam.focal_y = c->focal_y * ssf;
    cam.center_x = c->center_x * ssf;
    cam.center_y = c->center_y * ssf;
    cam.near_plane = c->near_plane;
    cam.far_plane = c->far_plane;
    cam.ss = ssf;
    cam.width_int = c->width * ss;
    cam.proper_aa = s->proper_antialiasing != 0;
    return cam;
}

}  // namespace

int sgs::record_error(const int status, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    t_last_error = buf;
    return status;
}

extern "C" {

size_t sgs_workspace_size(const sgs_gaussians* gaussians, const sgs_camera* camera, const sgs_settings* settings) {
    Derived d;
    if (derive(gaussians, camera, settings, d) != SGS_OK) return 0;
    return make_layout(d, settings).pub.total;
}

int sgs_get_workspace_layout(const sgs_gaussians* gaussians, const sgs_camera* camera, const sgs_settings* settings,
                             sgs_workspace_layout* layout) {
    Derived d;
    const int st = derive(gaussians, camera, settings, d);
    if (st != SGS_OK) return st;
    if (layout == nullptr) return fail(SGS_ERROR_INVALID_ARGUMENT, "null layout");
    *layout = make_layout(d, settings).pub;
    return SGS_OK;
}

}  // extern "C"

namespace {

// Event between the accumulate and the resolve stream of split renders (one per host thread).
thread_local cudaEvent_t t_split_event = nullptr;

__global__ void advance_frame_kernel(uint32_t* frame_counter, const uint32_t n) { *frame_counter += n; }

// The render of sgs_render / sgs_render_split: clear and accumulate on `acc_stream`, sample and
// resolve on `res_stream` (the same stream for sgs_render).
int render_on_streams(const sgs_gaussians* g, const sgs_camera* c, const sgs_settings* s, const sgs_history* h,
                      const sgs_outputs* o, void* workspace, size_t workspace_bytes, cudaStream_t acc_stream,
                      cudaStream_t res_stream, const uint32_t n_samples = 1) {
    t_last_error.clear();
    Derived d;
    int st = derive(g, c, s, d);
    if (st != SGS_OK) return st;
    if (n_samples == 0 || n_samples > kMaxSamplesPerCall)
        return fail(SGS_ERROR_INVALID_ARGUMENT, "%u samples per call (1 to %u)", n_samples, kMaxSamplesPerCall);
    if (n_samples > 1 && acc_stream != res_stream)
        return fail(SGS_ERROR_INVALID_ARGUMENT, "several samples per call run on one stream");
    if (static_cast<uint64_t>(d.n_fb) * n_samples > 0xffffffffull)
        return fail(SGS_ERROR_INVALID_ARGUMENT, "the samples' framebuffers exceed 2^32 pixels");
    if (h == nullptr || o == nullptr) return fail(SGS_ERROR_INVALID_ARGUMENT, "null history or outputs");
    if (s->temporal_mode < SGS_TEMPORAL_RESET || s->temporal_mode > SGS_TEMPORAL_REPROJECT)
        return fail(SGS_ERROR_INVALID_ARGUMENT, "invalid temporal mode %d", s->temporal_mode);
    if (g->n_gaussians > 0) {
        if (g->quantized != nullptr) {
            if (!g->quantized_chunks || !g->sh_half || !aligned16(g->quantized) || !aligned16(g->quantized_chunks))
                return fail(SGS_ERROR_INVALID_ARGUMENT,
                            "the quantised layout needs 16-byte aligned records and chunk table, and half SH");
            if (g->preactivated != nullptr)
                return fail(SGS_ERROR_INVALID_ARGUMENT, "the preactivated and quantised layouts exclude each other");
        } else {
            if (!g->means || !g->scales || !g->rotations || !g->opacities || !g->sh_coefficients)
                return fail(SGS_ERROR_INVALID_ARGUMENT, "null Gaussian array");
            if (!aligned16(g->rotations)) return fail(SGS_ERROR_INVALID_ARGUMENT, "rotations must be 16-byte aligned");
        }
        if (!aligned16(g->preactivated))
            return fail(SGS_ERROR_INVALID_ARGUMENT, "the preactivated layout must be 16-byte aligned");
    }
    if (g->sh_bases != 1 && g->sh_bases != 4 && g->sh_bases != 9 && g->sh_bases != 16)
        return fail(SGS_ERROR_INVALID_ARGUMENT, "sh_bases must be 1, 4, 9 or 16 (got %u)", g->sh_bases);
    if (!c->w2c || !aligned16(c->w2c)) return fail(SGS_ERROR_INVALID_ARGUMENT, "w2c must be a 16-byte aligned pointer");
    if (!c->cam_position) return fail(SGS_ERROR_INVALID_ARGUMENT, "null cam_position");
    if (!o->image || !o->depth || !o->alpha || !o->weight_mass) return fail(SGS_ERROR_INVALID_ARGUMENT, "null output");
    if (s->temporal_mode != SGS_TEMPORAL_RESET && (!h->image || !h->depth || !h->alpha || !h->weight_mass))
        return fail(SGS_ERROR_INVALID_ARGUMENT, "temporal mode %d needs the history", s->temporal_mode);
    if (s->temporal_mode == SGS_TEMPORAL_REPROJECT &&
        (!s->view_to_previous_view || !aligned16(s->view_to_previous_view)))
        return fail(SGS_ERROR_INVALID_ARGUMENT, "REPROJECT needs a 16-byte aligned view_to_previous_view");
    if (s->spatial_reuse && (!h->k_buffer_primitives || !h->k_buffer_occlusion || !aligned16(h->k_buffer_occlusion) ||
                             (reinterpret_cast<uintptr_t>(h->k_buffer_primitives) & 7u) != 0))
        return fail(SGS_ERROR_INVALID_ARGUMENT, "spatial reuse needs aligned k-buffer arrays");
    const FullLayout F = make_layout(d, s, n_samples);
    const sgs_workspace_layout& L = F.pub;
    if (workspace == nullptr || (reinterpret_cast<uintptr_t>(workspace) & (kAlign - 1)) != 0)
        return fail(SGS_ERROR_WORKSPACE, "workspace must be a 256-byte aligned device pointer");
    if (workspace_bytes < L.total)
        return fail(SGS_ERROR_WORKSPACE, "workspace has %zu bytes, needs %zu", workspace_bytes, L.total);

    const bool split = acc_stream != res_stream;
    if (split && t_split_event == nullptr &&
        cudaEventCreateWithFlags(&t_split_event, cudaEventDisableTiming) != cudaSuccess) {
        t_split_event = nullptr;
        return fail(SGS_ERROR_CUDA, "could not create the event between the accumulate and resolve streams");
    }
    char* ws = static_cast<char*>(workspace);
    // the host counter serves calls that keep no frame index in device memory
    const uint32_t frame =
        s->frame_index_device != nullptr ? 0u : g_frame_index.fetch_add(n_samples, std::memory_order_relaxed);
    const int sms = sm_count();

    Workspace w{};
    w.queue = reinterpret_cast<WorkQueue*>(ws + L.queue);
    w.framebuffer = reinterpret_cast<unsigned long long*>(ws + L.framebuffer);
    w.samples = reinterpret_cast<float4*>(ws + L.samples);
    w.reuse_weights = reinterpret_cast<float4*>(ws + L.reuse_weights);
    w.q.key = reinterpret_cast<unsigned long long*>(ws + F.q_key);
    w.q.geom = reinterpret_cast<float4*>(ws + F.q_geom);
    w.q.geom2 = reinterpret_cast<float4*>(ws + F.q_geom2);
    w.q.meta = reinterpret_cast<uint4*>(ws + F.q_meta);
    w.q.count = reinterpret_cast<uint32_t*>(ws + F.q_count);
    w.q.capacity = d.queue_capacity;

    const PassCamera cam = pass_camera(c, s, d.ss);
    AccumulateParams ap{};
    ap.means = g->means;
    ap.scales = g->scales;
    ap.rotations = reinterpret_cast<const float4*>(g->rotations);
    ap.opacities = g->opacities;
    ap.w2c = reinterpret_cast<const float4*>(c->w2c);
    ap.framebuffer = w.framebuffer;
    ap.n = g->n_gaussians;
    ap.frame_idx = frame;
    ap.frame_ptr = s->frame_index_device;
    ap.cam = cam;
    // the kernels pick one blue-noise slice per frame, rotated by the golden ratio per pass
    ap.blue_noise = s->use_gps ? nullptr : s->blue_noise;
    ap.max_fragments = s->max_fragments;
    ap.max_binned = d.max_binned;
    ap.hybrid = s->hybrid_scheduling != 0;
    ap.queue = w.queue;
    ap.q = w.q;
    ap.n_samples = n_samples;
    ap.fb_stride = d.n_fb;
    ap.pre = reinterpret_cast<const float4*>(g->preactivated);
    const QuantizedModel qm{static_cast<const uint4*>(g->quantized), reinterpret_cast<const float4*>(g->quantized_chunks),
                            static_cast<const __half*>(g->sh_half)};
    ap.quant = qm;

    ResolveParams rp{};
    rp.means = g->means;
    rp.scales = g->scales;
    rp.rotations = reinterpret_cast<const float4*>(g->rotations);
    rp.opacities = g->opacities;
    rp.sh = g->sh_coefficients;
    rp.w2c = reinterpret_cast<const float4*>(c->w2c);
    rp.cam_position = c->cam_position;
    rp.framebuffer = w.framebuffer;
    rp.samples = w.samples;
    rp.reuse_weights = w.reuse_weights;
    rp.k_prims = reinterpret_cast<uint2*>(h->k_buffer_primitives);
    rp.k_occl = reinterpret_cast<float4*>(h->k_buffer_occlusion);
    rp.hist_image = h->image;
    rp.hist_depth = h->depth;
    rp.hist_alpha = h->alpha;
    rp.hist_weight_mass = h->weight_mass;
    rp.v2pv = reinterpret_cast<const float4*>(s->view_to_previous_view);
    rp.image = o->image;
    rp.depth = o->depth;
    rp.alpha = o->alpha;
    rp.weight_mass = o->weight_mass;
    rp.n_fb = static_cast<uint32_t>(d.n_fb);
    rp.n_pixels = static_cast<uint32_t>(d.n_pixels);
    rp.sh_bases = g->sh_bases;
    rp.width = c->width;
    rp.height = c->height;
    rp.ss = d.ss;
    rp.focal_x = c->focal_x;
    rp.focal_y = c->focal_y;
    rp.center_x = c->center_x;
    rp.center_y = c->center_y;
    rp.far_plane = c->far_plane;
    rp.cam = cam;
    rp.spatial_reuse = s->spatial_reuse != 0;
    rp.sh_vec4 = g->sh_bases == 16 && aligned16(g->sh_coefficients);
    rp.frame_counter = s->frame_index_device;
    rp.temporal_mode = s->temporal_mode;
    rp.n_samples = n_samples;
    rp.fb_stride = d.n_fb;
    rp.quant = qm;

    // the clear and accumulate passes of one framebuffer (or, with p.n_samples > 1, of all of them)
    auto accumulate = [&](const AccumulateParams& p, const size_t n_clear) -> int {
        cudaError_t err = launch_clear(p.framebuffer, n_clear, w.queue, sms, acc_stream);
        if (err != cudaSuccess) return fail(SGS_ERROR_CUDA, "clear: %s", cudaGetErrorString(err));
        if (g->n_gaussians == 0) return SGS_OK;
        if (t_stage_start != nullptr) cudaEventRecord(t_stage_start, acc_stream);
        err = s->use_gps ? launch_accumulate_gps(p, sms, acc_stream) : launch_accumulate_st(p, sms, acc_stream);
        if (t_stage_end != nullptr && err == cudaSuccess) err = cudaEventRecord(t_stage_end, acc_stream);
        if (err != cudaSuccess) return fail(SGS_ERROR_CUDA, "accumulate: %s", cudaGetErrorString(err));
        return SGS_OK;
    };
    auto resolve = [&](const ResolveParams& r) -> int {
        const cudaError_t err = launch_sample_resolve(r, res_stream);
        if (err != cudaSuccess) return fail(SGS_ERROR_CUDA, "sample/resolve: %s", cudaGetErrorString(err));
        return SGS_OK;
    };

    if (n_samples > 1 && (s->spatial_reuse || s->temporal_mode == SGS_TEMPORAL_REPROJECT)) {
        // The k-buffer and the Reproject history are updated sample by sample: the whole pipeline runs
        // once per sample, the first in the call's temporal mode and the rest Static, each merging into
        // the outputs in place (a Static resolve reads a pixel's history only in the thread that writes
        // the pixel). The same passes as n_samples single calls.
        for (uint32_t sm = 0; sm < n_samples; ++sm) {
            AccumulateParams pa = ap;
            pa.n_samples = 1;
            pa.frame_idx = frame + sm;
            ResolveParams pr = rp;
            pr.n_samples = 1;
            if (sm > 0) {
                pr.temporal_mode = SGS_TEMPORAL_STATIC;
                pr.hist_image = o->image;
                pr.hist_depth = o->depth;
                pr.hist_alpha = o->alpha;
                pr.hist_weight_mass = o->weight_mass;
            }
            st = accumulate(pa, d.n_fb);
            if (st == SGS_OK) st = resolve(pr);
            if (st != SGS_OK) return st;
        }
        return SGS_OK;
    }
    if (n_samples > 1 && s->use_gps && s->hybrid_scheduling) {
        // Several GPS samples with hybrid scheduling: each frame's points are drawn by its own scatter
        // and queue passes into its own framebuffer (the work queue is reused in stream order), then one
        // resolve pass merges the n framebuffers in frame order.
        cudaError_t err = launch_clear(w.framebuffer, d.n_fb * n_samples, w.queue, sms, acc_stream);
        if (err != cudaSuccess) return fail(SGS_ERROR_CUDA, "clear: %s", cudaGetErrorString(err));
        if (t_stage_start != nullptr) cudaEventRecord(t_stage_start, acc_stream);
        for (uint32_t sm = 0; sm < n_samples && g->n_gaussians > 0; ++sm) {
            AccumulateParams pa = ap;
            pa.n_samples = 1;
            pa.framebuffer = w.framebuffer + static_cast<size_t>(sm) * d.n_fb;
            pa.frame_offset = sm;
            if (sm > 0) {
                err = launch_clear(pa.framebuffer, 0, w.queue, sms, acc_stream);  // the queue header only
                if (err != cudaSuccess) return fail(SGS_ERROR_CUDA, "clear: %s", cudaGetErrorString(err));
            }
            err = launch_accumulate_gps(pa, sms, acc_stream);
            if (err != cudaSuccess) return fail(SGS_ERROR_CUDA, "accumulate: %s", cudaGetErrorString(err));
        }
        if (t_stage_end != nullptr) cudaEventRecord(t_stage_end, acc_stream);
        return resolve(rp);
    }

    st = accumulate(ap, d.n_fb * n_samples);
    if (st != SGS_OK) return st;
    if (split) {
        // the next call's accumulate pass may start before this resolve: advance the device-resident
        // frame index behind this accumulate pass instead
        if (s->frame_index_device != nullptr) {
            advance_frame_kernel<<<1, 1, 0, acc_stream>>>(s->frame_index_device, n_samples);
            rp.frame_counter = nullptr;
        }
        cudaError_t err = cudaEventRecord(t_split_event, acc_stream);
        if (err == cudaSuccess) err = cudaStreamWaitEvent(res_stream, t_split_event, 0);
        if (err == cudaSuccess) err = cudaGetLastError();
        if (err != cudaSuccess) return fail(SGS_ERROR_CUDA, "stream split: %s", cudaGetErrorString(err));
    }
    return resolve(rp);
}

}  // namespace

extern "C" {

int sgs_render(const sgs_gaussians* g, const sgs_camera* c, const sgs_settings* s, const sgs_history* h,
               const sgs_outputs* o, void* workspace, size_t workspace_bytes, void* stream) {
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    return render_on_streams(g, c, s, h, o, workspace, workspace_bytes, st, st);
}

int sgs_render_split(const sgs_gaussians* g, const sgs_camera* c, const sgs_settings* s, const sgs_history* h,
                     const sgs_outputs* o, void* workspace, size_t workspace_bytes, void* accumulate_stream,
                     void* resolve_stream) {
    return render_on_streams(g, c, s, h, o, workspace, workspace_bytes, static_cast<cudaStream_t>(accumulate_stream),
                             static_cast<cudaStream_t>(resolve_stream));
}

size_t sgs_samples_workspace_size(const sgs_gaussians* g, const sgs_camera* c, const sgs_settings* s,
                                  uint32_t n_samples) {
    Derived d;
    if (derive(g, c, s, d) != SGS_OK || n_samples == 0 || n_samples > kMaxSamplesPerCall) return 0;
    return make_layout(d, s, n_samples).pub.total;
}

int sgs_render_samples(const sgs_gaussians* g, const sgs_camera* c, const sgs_settings* s, const sgs_history* h,
                       const sgs_outputs* o, uint32_t n_samples, void* workspace, size_t workspace_bytes,
                       void* stream) {
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    return render_on_streams(g, c, s, h, o, workspace, workspace_bytes, st, st, n_samples);
}

void sgs_set_queue_limit(uint32_t max_entries) { g_queue_limit.store(max_entries, std::memory_order_relaxed); }

int sgs_preactivate(const sgs_gaussians* g, float* out, void* stream) {
    if (g == nullptr) return fail(SGS_ERROR_INVALID_ARGUMENT, "null argument");
    if (g->n_gaussians == 0) return SGS_OK;
    if (out == nullptr) return fail(SGS_ERROR_INVALID_ARGUMENT, "null output");
    if (!g->scales || !g->rotations || !g->opacities) return fail(SGS_ERROR_INVALID_ARGUMENT, "null Gaussian array");
    if (!aligned16(g->rotations) || !aligned16(out))
        return fail(SGS_ERROR_INVALID_ARGUMENT, "rotations and the output must be 16-byte aligned");
    const cudaError_t err = launch_preactivate(g->scales, reinterpret_cast<const float4*>(g->rotations), g->opacities,
                                               g->n_gaussians, reinterpret_cast<float4*>(out),
                                               static_cast<cudaStream_t>(stream));
    if (err != cudaSuccess) return fail(SGS_ERROR_CUDA, "preactivate launch: %s", cudaGetErrorString(err));
    return SGS_OK;
}

int sgs_probe_atomic_min(void* slots, uint64_t n_slots, uint32_t ops_per_thread, uint32_t blocks, uint32_t pattern,
                         uint32_t seed, void* stream) {
    if (slots == nullptr || (reinterpret_cast<uintptr_t>(slots) & 7u) != 0)
        return fail(SGS_ERROR_INVALID_ARGUMENT, "slots must be an 8-byte aligned device pointer");
    if (n_slots == 0 || (n_slots & (n_slots - 1)) != 0)
        return fail(SGS_ERROR_INVALID_ARGUMENT, "n_slots must be a power of two");
    if (blocks == 0 || blocks > (1u << 20) || ops_per_thread == 0 || ops_per_thread > (1u << 16) || pattern > 1)
        return fail(SGS_ERROR_INVALID_ARGUMENT, "blocks 1..2^20, ops_per_thread 1..2^16, pattern 0 or 1");
    const cudaError_t err = launch_atomic_min_probe(static_cast<unsigned long long*>(slots), n_slots, ops_per_thread,
                                                    blocks, pattern, seed, static_cast<cudaStream_t>(stream));
    if (err != cudaSuccess) return fail(SGS_ERROR_CUDA, "atomic probe launch: %s", cudaGetErrorString(err));
    return SGS_OK;
}

void sgs_set_stage_events(void* accumulate_start, void* accumulate_end) {
    t_stage_start = static_cast<cudaEvent_t>(accumulate_start);
    t_stage_end = static_cast<cudaEvent_t>(accumulate_end);
}

uint32_t sgs_get_frame_index(void) { return g_frame_index.load(std::memory_order_relaxed); }

void sgs_set_frame_index(uint32_t frame_index) { g_frame_index.store(frame_index, std::memory_order_relaxed); }

uint32_t sgs_k_buffer_size(void) { return kKBufferSize; }

int sgs_abi_version(void) { return SGS_ABI_VERSION; }

const char* sgs_last_error(void) { return t_last_error.c_str(); }

}  // extern "C"
