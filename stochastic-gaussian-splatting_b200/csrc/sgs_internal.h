// Internal host-side interface between the C ABI (render_abi.cu) and the kernel files.
#pragma once

#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>
#include "sgs_project.cuh"

namespace sgs {

// Large-Gaussian work queue shared by the ST and GPS accumulate passes. Entries are appended
// with one 64-bit atomicAdd on `packed` = (entry count << 40) | chunk count, so every entry's
// first chunk index is known at insertion and increases with the entry index.
struct WorkQueue {
    unsigned long long packed;   // (entries << 40) | chunks, reserved by producers
    unsigned int next_chunk;     // work-stealing cursor of the consumer kernel
    unsigned int overflow;       // producers that found the queue full (processed in place)
    unsigned int error;          // nonzero when a consumer met an inconsistent entry
    unsigned int binned;         // hybrid ST: Gaussians the reference would gather, in arrival order
    unsigned int pad[2];
};
constexpr unsigned long long kQueueEntryShift = 40;
constexpr unsigned long long kQueueChunkMask = (1ull << kQueueEntryShift) - 1;
// Producers queue chunk indices below this, so the consumers' cursor (which overshoots the last chunk
// by at most one claim per warp) cannot wrap around.
constexpr unsigned long long kMaxQueueChunks = 0xffffffffull - (1ull << 24);
// First-chunk value of a queue entry left unused because its chunks would pass
// kMaxQueueChunks (above every chunk index, so the entry search never returns it).
constexpr uint32_t kUnusedQueueEntry = 0xffffffffu;

// Per-entry arrays of the large-Gaussian queue (structure of arrays, 16-byte aligned).
struct QueueArrays {
    unsigned long long* key;  // packed fragment key
    float4* geom;             // ST: mean2d - 0.5 (x, y), exp2-scaled conic (x, y); GPS: mean2d, L.x, L.y
    float4* geom2;            // ST: conic z, opacity, x_min, width (bit casts); GPS: L.z, power threshold, opacity_rcp, dilog
    uint4* meta;              // ST: y_min, height, rows per chunk, first chunk; GPS: conic x/y/z bits, first chunk
    uint32_t* count;          // GPS: number of points
    uint32_t capacity;
};

// Queue entry owning chunk c: the last e in [0, n) with meta[e].w (the entry's first chunk,
// nondecreasing in e, meta[0].w = 0) <= c. A 32-ary search by the whole warp (every lane calls it
// with the same arguments): each step the lanes read 32 evenly spaced first chunks at once and a
// ballot keeps the segment that holds the answer, so 2^20 entries take 4 rounds of loads instead
// of 20 dependent ones.
__device__ __forceinline__ uint32_t queue_entry_of_chunk(const uint4* __restrict__ meta, const uint32_t n,
                                                         const uint32_t c, const uint32_t lane) {
    uint32_t lo = 0, hi = n;  // the answer lies in [lo, hi)
    while (hi - lo > 1u) {
        const uint32_t step = (hi - lo + 31u) >> 5;
        const uint32_t idx = lo + lane * step;
        const bool le = lane == 0u || (idx < hi && meta[idx].w <= c);
        const uint32_t k = 31u - __clz(__ballot_sync(0xffffffffu, le));
        lo += k * step;
        hi = min(hi, lo + step);
    }
    return lo;
}

// Scratch carved out of the caller's workspace by layout_workspace().
struct Workspace {
    unsigned long long* framebuffer;  // P_fb packed keys
    float4* samples;                  // P_fb (rgb, depth)
    float4* reuse_weights;            // P_fb when spatial reuse is on
    WorkQueue* queue;
    QueueArrays q;
    size_t bytes;
};

struct AccumulateParams {
    const float* means;
    const float* scales;
    const float4* rotations;
    const float* opacities;
    const float4* w2c;
    unsigned long long* framebuffer;
    uint32_t n;
    uint32_t frame_idx;               // used when frame_ptr is null
    const uint32_t* frame_ptr;        // device-resident frame index, or null
    uint32_t frame_offset;            // added to either: sample s of a call whose passes run per sample
    PassCamera cam;
    const uint8_t* blue_noise;        // (64, 128, 128) volume; null: white noise
    uint32_t max_fragments;           // GPS point cap per Gaussian
    uint32_t max_binned;              // hybrid: binned Gaussian capacity (accumulate_hybrid*.cu max_binned)
    bool hybrid;                      // hybrid scheduling
    WorkQueue* queue;
    QueueArrays q;
    uint32_t n_samples;               // samples of one call (frames frame .. frame + n_samples - 1)
    size_t fb_stride;                 // framebuffer elements between consecutive samples' framebuffers
    const float4* pre;                // preactivated layout (2 float4 per Gaussian) or null
    QuantizedModel quant;             // quantised layout (records == null: the float32 arrays)
};

// Frame-dependent random-number state of one call: the frame index (from device memory when the
// caller keeps it there) and the blue-noise slice and rotation it selects (render.cu:77-82).
struct FrameRng {
    uint32_t frame;
    const uint8_t* slice;
    uint32_t rotation;
};

// The random-number state of frame `frame`.
__device__ __forceinline__ FrameRng frame_rng_at(const AccumulateParams& a, const uint32_t frame) {
    FrameRng r;
    r.frame = frame;
    r.slice = a.blue_noise != nullptr
                  ? a.blue_noise + static_cast<size_t>(frame % kBlueNoiseDepth) * kBlueNoiseWidth * kBlueNoiseHeight
                  : nullptr;
    r.rotation = (frame / kBlueNoiseDepth) * 0x9E3779B9u;
    return r;
}

__device__ __forceinline__ FrameRng frame_rng(const AccumulateParams& a) {
    return frame_rng_at(a, (a.frame_ptr != nullptr ? *a.frame_ptr : a.frame_idx) + a.frame_offset);
}

cudaError_t launch_clear(unsigned long long* framebuffer, size_t n_fb, WorkQueue* queue, int num_sms,
                         cudaStream_t stream);
cudaError_t launch_accumulate_st(const AccumulateParams& p, int num_sms, cudaStream_t stream);
cudaError_t launch_accumulate_gps(const AccumulateParams& p, int num_sms, cudaStream_t stream);
cudaError_t launch_quantize(const float* means, const float* scales, const float4* rotations, const float* opacities,
                            const float* sh, uint32_t sh_floats, uint32_t n, uint4* records, float4* chunks,
                            __half* sh_half, cudaStream_t stream);
cudaError_t launch_composite(const float* image, const float* depth, const float* alpha, const float* background,
                             uint32_t n, float* rgb, float* depth_out, float* alpha_out, cudaStream_t stream);
cudaError_t launch_preactivate(const float* scales, const float4* rotations, const float* opacities, uint32_t n,
                              float4* out, cudaStream_t stream);
cudaError_t launch_atomic_min_probe(unsigned long long* slots, uint64_t n_slots, uint32_t ops, uint32_t blocks,
                                    uint32_t pattern, uint32_t seed, cudaStream_t stream);

struct ResolveParams {
    const float* means;
    const float* scales;
    const float4* rotations;
    const float* opacities;
    const float* sh;
    const float4* w2c;
    const float* cam_position;
    const unsigned long long* framebuffer;
    float4* samples;
    float4* reuse_weights;
    uint2* k_prims;
    float4* k_occl;
    const float* hist_image;
    const float* hist_depth;
    const float* hist_alpha;
    const float* hist_weight_mass;
    const float4* v2pv;
    float* image;
    float* depth;
    float* alpha;
    float* weight_mass;
    uint32_t n_fb;
    uint32_t n_pixels;
    uint32_t sh_bases;
    uint32_t width, height, ss;
    float focal_x, focal_y, center_x, center_y, far_plane;  // image pixels (resolve)
    PassCamera cam;                                          // framebuffer (sample)
    bool spatial_reuse;
    bool sh_vec4;    // degree-3 SH at a 16-byte aligned base: winners load their coefficients as float4
    uint32_t* frame_counter;  // device-resident frame index advanced by the last pass, or null
    int temporal_mode;
    uint32_t n_samples;       // samples merged by one call (the first in temporal_mode, the rest Static)
    size_t fb_stride;         // framebuffer elements between consecutive samples' framebuffers
    QuantizedModel quant;     // quantised layout (records == null: the float32 arrays)
};

cudaError_t launch_sample_resolve(const ResolveParams& p, cudaStream_t stream);

// Backward pass of stochastic transparency (backward_st.cu).
struct BackwardParams {
    const float* means;
    const float* scales;
    const float4* rotations;
    const float* opacities;
    const float* sh;
    const float4* w2c;
    const float* cam_position;
    uint32_t n;
    uint32_t sh_bases;
    PassCamera cam;                          // framebuffer camera
    uint32_t width;                          // image width (pixels)
    uint32_t ss;
    const unsigned long long* framebuffer;   // the sample's winners
    const float4* samples;                   // the sample's winner colour and depth
    const float* grad_image;                 // (H, W, 3) upstream gradient of the image
    const float* grad_alpha;                 // (H, W) or null
    const float* grad_depth;                 // (H, W) or null
    float grad_scale;                        // weight of this sample in the output / ss^2
    float* colors;                           // (N, 3) per-Gaussian colour
    float* accum;                            // (N, 10) projected-quantity gradients
    float* d_means;
    float* d_scales;
    float* d_rotations;
    float* d_opacities;
    float* d_sh;
    // fused form over S samples: per framebuffer pixel and sample, the winner key and
    // T = grad_scale (g . c_w + g_d z_w), interleaved [pixel][sample]
    unsigned long long* pix_keys;
    float* pix_terms;
    unsigned long long* pix_max_key;         // per pixel, the largest winner key of the samples
    // queue of Gaussians with large footprints, walked in row chunks by a persistent kernel
    WorkQueue* bw_queue;
    void* bw_entries;                        // WalkGaussian per entry (backward_st.cu)
    uint4* bw_meta;                          // y_min, height, log2 rows per chunk, first chunk
    uint32_t* bw_index;                      // Gaussian index per entry
    uint32_t bw_capacity;
    int num_sms;
    uint32_t n_samples;                      // S
    uint32_t sample;                         // the sample whose terms sample_terms writes
    uint32_t n_fb;                           // framebuffer pixels
};

cudaError_t launch_backward_colors(const BackwardParams& p, cudaStream_t stream);
cudaError_t launch_backward_fragments(const BackwardParams& p, cudaStream_t stream);
cudaError_t launch_backward_projection(const BackwardParams& p, cudaStream_t stream);
cudaError_t launch_backward_sample_terms(const BackwardParams& p, cudaStream_t stream);
cudaError_t launch_backward_framebuffer_terms(const BackwardParams& p, cudaStream_t stream);
cudaError_t launch_backward_fragments_samples(const BackwardParams& p, cudaStream_t stream);

// Sets the calling thread's sgs_last_error() message (printf format) and returns `status`.
int record_error(int status, const char* fmt, ...);

}  // namespace sgs
