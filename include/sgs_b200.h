/*
 * sgs_b200.h - C ABI of the B200 stochastic Gaussian splatting render path.
 *
 * One call renders one stochastic sample ("sample-frame") of a 3D Gaussian splatting scene and
 * merges it into the caller's progressive history, exactly like one `_C.render(...)` call of the
 * reference extension StochasticGSCudaBackend (StochasticGSCudaBackend/render.cu:16-158, bound by
 * PYBIND11_MODULE at render.cu:162-165 and wrapped by StochasticGSCudaBackend/render.py:72-96).
 * Plain pointers and sizes only: every array pointer is a device pointer of the current CUDA
 * device, row-major and contiguous, and `stream` is a cudaStream_t (NULL = legacy default stream).
 * Calls are asynchronous with respect to the host; the functions never synchronise the device.
 *
 * Status codes: 0 success, negative on error; sgs_last_error() describes the last error of the
 * calling thread. Invalid arguments are rejected before any launch (the reference does not
 * validate and traps on an invalid temporal mode, resolve.cu:342).
 */
#ifndef SGS_B200_H
#define SGS_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SGS_ABI_VERSION 4
#define SGS_K_BUFFER_SIZE 4 /* k-buffer entries per (sub)pixel, resolve.h:9 / render.cu:164 */

enum sgs_status {
    SGS_OK = 0,
    SGS_ERROR_INVALID_ARGUMENT = -1,
    SGS_ERROR_WORKSPACE = -2, /* workspace missing, misaligned or smaller than sgs_workspace_size() */
    SGS_ERROR_CUDA = -3       /* a CUDA runtime call or launch failed */
};

enum sgs_temporal_mode { /* StochasticGSCudaBackend/render.py:44-47, resolve.h:11-15 */
    SGS_TEMPORAL_RESET = 0,
    SGS_TEMPORAL_STATIC = 1,
    SGS_TEMPORAL_REPROJECT = 2
};

/* Gaussian model in the layout of Model.py:22-79 (render.cu:17-21). */
typedef struct sgs_gaussians {
    const float* means;           /* (N, 3) world positions */
    const float* scales;          /* (N, 3) log scales */
    const float* rotations;       /* (N, 4) quaternions (r, i, j, k), any norm; 16-byte aligned */
    const float* opacities;       /* (N) opacity logits */
    const float* sh_coefficients; /* (N, B, 3) SH coefficients */
    uint32_t n_gaussians;         /* N (0 renders background) */
    uint32_t sh_bases;            /* B: 1, 4, 9 or 16 (degree 0..3) */
    const float* preactivated;    /* optional (N, 8) from sgs_preactivate, 16-byte aligned, or NULL; when
                                   * set, the accumulate pass reads covariance and opacity from it (the
                                   * same bits) instead of rebuilding them from scales, rotations and
                                   * opacities. It must match those arrays; nothing checks that. */
    const void* quantized;        /* optional (N, 4) uint32 records of sgs_quantize, 16-byte aligned, or NULL;
                                   * when set, every pass reads positions, rotations, scales and opacities
                                   * from them (the float32 arrays above may then be NULL) */
    const float* quantized_chunks; /* with `quantized`: the (sgs_quantized_chunks(N), 8) chunk table */
    const void* sh_half;          /* with `quantized`: the (N, B, 3) IEEE half SH coefficients of sgs_quantize,
                                   * read by the sample pass instead of sh_coefficients */
} sgs_gaussians;

/* Pinhole camera in image pixels (render.cu:22-31, render_utils.h:19-30). */
typedef struct sgs_camera {
    const float* w2c;          /* world-to-view, >= 3 rows of 4 floats; 16-byte aligned */
    const float* cam_position; /* (3) camera position in world space */
    uint32_t width;            /* image width in pixels */
    uint32_t height;           /* image height in pixels */
    float focal_x, focal_y;    /* focal lengths in pixels */
    float center_x, center_y;  /* principal point in pixels (x right, y down) */
    float near_plane, far_plane;
} sgs_camera;

/* Switches of one call (render.cu:32-37,44-45). */
typedef struct sgs_settings {
    int32_t proper_antialiasing;
    int32_t supersampling_factor;            /* values < 1 act as 1 (render.cu:52) */
    int32_t use_gps;                         /* Gaussian point splatting instead of stochastic transparency */
    int32_t hybrid_scheduling;               /* load-balanced pass for large Gaussians */
    int32_t spatial_reuse;                   /* resample the four neighbours through the k-buffer */
    int32_t temporal_mode;                   /* enum sgs_temporal_mode */
    const uint8_t* blue_noise;               /* (64, 128, 128) u8 volume, or NULL for white noise */
    const float* view_to_previous_view;      /* 4x4 row-major, read in REPROJECT mode; 16-byte aligned */
    uint32_t max_fragments;                  /* GPS points per Gaussian cap; 0 = W*H/2 as the reference */
    uint32_t max_binned;                     /* hybrid bin capacity; 0 = min(N, 2^20) as the reference */
    uint32_t* frame_index_device;            /* NULL: the process-wide frame index (render.cu:56-57); else a
                                                device word the call reads as its frame index and advances
                                                by one on the GPU, so that calls captured in a CUDA graph
                                                draw new random numbers on every replay */
} sgs_settings;

/* Caller-owned state carried between calls (render.cu:38-43). */
typedef struct sgs_history {
    const float* image;        /* (H, W, 3) previous premultiplied colour; read in STATIC / REPROJECT */
    const float* depth;        /* (H, W, 1) */
    const float* alpha;        /* (H, W, 1) */
    const float* weight_mass;  /* (H, W, 1) */
    int32_t* k_buffer_primitives; /* (K, P_fb, 2) (index, depth bits); updated in place with spatial reuse */
    float* k_buffer_occlusion;    /* (K, P_fb, 4); updated in place with spatial reuse */
} sgs_history;

/* Freshly written outputs (render.cu:59-62), the next call's history. May not alias the history. */
typedef struct sgs_outputs {
    float* image;       /* (H, W, 3) colour premultiplied by alpha */
    float* depth;       /* (H, W, 1) depth premultiplied by alpha */
    float* alpha;       /* (H, W, 1) */
    float* weight_mass; /* (H, W, 1) accumulated resampling weight */
} sgs_outputs;

/* Offsets (bytes, from the workspace start) of the intermediate buffers of sgs_render. */
typedef struct sgs_workspace_layout {
    size_t framebuffer;   /* uint64 (P_fb): packed (depth_bits << 32 | index) winners, ~0 = empty */
    size_t samples;       /* float (P_fb, 4): winner colour and depth (0 = background) */
    size_t reuse_weights; /* float (P_fb, 4) with spatial reuse, else unused */
    size_t queue;         /* large-Gaussian work queue */
    size_t total;         /* == sgs_workspace_size() */
} sgs_workspace_layout;

/* Scratch bytes sgs_render needs for these arguments (replaces the per-call allocations of
 * render.cu:63-65, accumulate_hybrid.cu:356-366 and accumulate_hybrid_gps.cu:212-219). The
 * workspace must be 256-byte aligned; it need not be initialised. */
size_t sgs_workspace_size(const sgs_gaussians* gaussians, const sgs_camera* camera, const sgs_settings* settings);

/* Fills `layout` for these arguments; returns SGS_OK or an error status. */
int sgs_get_workspace_layout(const sgs_gaussians* gaussians, const sgs_camera* camera, const sgs_settings* settings,
                             sgs_workspace_layout* layout);

/* One sample-frame (replaces `_C.render`, render.cu:16-158): clears the framebuffer, accumulates
 * the closest accepted fragment per (sub)pixel, evaluates the winners' colours, resolves and
 * merges with the history. Uses and then increments the process-wide frame index, which seeds
 * every random number (render.cu:56-57). Enqueued on `stream`; no host synchronisation. */
int sgs_render(const sgs_gaussians* gaussians, const sgs_camera* camera, const sgs_settings* settings,
               const sgs_history* history, const sgs_outputs* outputs, void* workspace, size_t workspace_bytes,
               void* stream);

/* sgs_render split over two streams (no counterpart in the reference): the framebuffer clear and
 * the accumulate pass are enqueued on `accumulate_stream`, the sample and resolve passes on
 * `resolve_stream` behind an event recorded after the accumulate pass. The accumulate pass reads
 * only the Gaussians, the camera and the workspace, so a following call with another workspace can
 * accumulate while this one resolves (many views in one CUDA graph, a progressive loop). The caller
 * orders `accumulate_stream` after its writes of the Gaussians and the camera, and `resolve_stream`
 * after its writes of the history and k-buffer and before its reads of the outputs; the workspace
 * must stay untouched until the resolve pass is done. A device-resident frame index is advanced on
 * `accumulate_stream`. The first call on a host thread creates the event between the streams: make
 * it before any stream capture. With both streams equal this is sgs_render. */
int sgs_render_split(const sgs_gaussians* gaussians, const sgs_camera* camera, const sgs_settings* settings,
                     const sgs_history* history, const sgs_outputs* outputs, void* workspace, size_t workspace_bytes,
                     void* accumulate_stream, void* resolve_stream);

/* Several samples in one call (no counterpart in the reference; it is the sample loop of
 * Renderer.py:85-87 moved onto the device): renders n_samples samples with frame indices f .. f + n - 1
 * (f = the current frame index, which advances by n) and merges them into the history in order, the
 * first in settings->temporal_mode and the rest Static. The outputs (and, with spatial reuse, the
 * k-buffer) equal those of n_samples sgs_render calls bit for bit. Stochastic transparency: one walk
 * over the Gaussians' fragments evaluates each fragment's alpha once and every sample's threshold;
 * GPS with scatter scheduling: one projection, then each frame's point draws; GPS with hybrid
 * scheduling: each frame's scatter and queue passes into its own framebuffer; in these three cases one
 * resolve pass reads the history once and merges the n framebuffers. With spatial reuse or a first
 * sample in Reproject, the k-buffer and the reprojected history change sample by sample, so the
 * whole pipeline runs once per sample inside the call. n_samples from 1 to 1024. The workspace holds
 * sgs_samples_workspace_size(..., n_samples) bytes (n_samples framebuffers). */
size_t sgs_samples_workspace_size(const sgs_gaussians* gaussians, const sgs_camera* camera,
                                  const sgs_settings* settings, uint32_t n_samples);
int sgs_render_samples(const sgs_gaussians* gaussians, const sgs_camera* camera, const sgs_settings* settings,
                       const sgs_history* history, const sgs_outputs* outputs, uint32_t n_samples, void* workspace,
                       size_t workspace_bytes, void* stream);

/* The frame compositing of the reference's renderer plugin (Renderer.py:91-97), on the device: for
 * each of n_pixels pixels of a history (image (n, 3) premultiplied, depth and alpha (n)), alpha_out =
 * clamp(alpha, 0, 1), rgb = clamp(image + (1 - alpha_out) * background_rgb, 0, 1) and depth_out =
 * depth / max(alpha_out, 1e-8), each operation rounded like the separate elementwise tensor operations
 * of the plugin (so the results equal them bit for bit). background_rgb is a device pointer to 3
 * floats, so a captured CUDA graph reads the current background on every replay; depth_out and
 * alpha_out may be NULL (depth may then be NULL too). */
int sgs_composite(const float* image, const float* depth, const float* alpha, const float* background_rgb,
                  uint32_t n_pixels, float* rgb, float* depth_out, float* alpha_out, void* stream);

/* sgs_render for callers that cannot allocate device memory while rendering (a plugin inside a
 * host application under a fixed memory budget, a C caller without a caching allocator). It has no
 * counterpart in the reference. The caller passes inputs, history and outputs as for sgs_render;
 * the scratch lives in a fixed 64 MiB device array of the library instead of a caller workspace,
 * so nothing is allocated per call. That array is held by every CUDA context that loads it, until
 * the process exits. Every call looks up the array's device address in the context current on the
 * calling thread, so the address is valid for that context (also after cudaDeviceReset, or under a
 * caller's own driver context); the first call in a context may load the module: make it before
 * any stream capture. All calls on a device share the array: the render clears what must start
 * empty, but calls that can overlap on the GPU race and must be ordered by the caller. Renders
 * needing more than 64 MiB of scratch (sgs_workspace_size) are rejected with SGS_ERROR_WORKSPACE
 * before any launch. Stochastic transparency at 1920x1080 without supersampling or spatial reuse
 * fits for any scene size; hybrid GPS at 1920x1080 fits up to about 289,000 queue entries
 * (max_binned, by default min(N, 2^20)), so larger scenes need settings->max_binned at or below
 * that. */
int sgs_render_no_alloc(const sgs_gaussians* gaussians, const sgs_camera* camera, const sgs_settings* settings,
                        const sgs_history* history, const sgs_outputs* outputs, void* stream);

/* Backward pass of stochastic transparency (no counterpart in the reference, which renders only).
 * Gradients of a loss of the averaged image of S samples w.r.t. means, log-scales, quaternions,
 * opacity logits and SH coefficients, by an unbiased one-sample estimator of the gradient of the
 * expected image computed from each sample's winners:
 *   1. for each sample s, after the sgs_render call that produced it (or a re-render with the same
 *      frame index and settings), call sgs_backward_accumulate with that call's workspace, the
 *      upstream gradients of the output image (H, W, 3), alpha and depth (H, W; may be NULL) and
 *      `weight` = the sample's weight in the averaged output (1/S for a plain progressive average);
 *      `first` = 1 for the first sample (clears the accumulators);
 *   2. sgs_backward_finish writes the parameter gradients (overwriting them).
 * Supported: stochastic transparency (white or blue noise, scatter or hybrid), any supersampling, with
 * or without proper antialiasing, Reset/Static; not spatial reuse (SGS_ERROR_INVALID_ARGUMENT). GPS
 * gradients are computed by the fused form below only (this call rejects GPS settings).
 * `backward_workspace` holds sgs_backward_workspace_size(n) bytes, 16-byte aligned. */
size_t sgs_backward_workspace_size(uint32_t n_gaussians);
int sgs_backward_accumulate(const sgs_gaussians* gaussians, const sgs_camera* camera, const sgs_settings* settings,
                            const void* render_workspace, const float* grad_image, const float* grad_alpha,
                            const float* grad_depth, float weight, int first, void* backward_workspace, void* stream);
int sgs_backward_finish(const sgs_gaussians* gaussians, const sgs_camera* camera, const sgs_settings* settings,
                        void* backward_workspace, float* d_means, float* d_scales, float* d_rotations,
                        float* d_opacities, float* d_sh, void* stream);

/* Fused form of step 1 for S samples that share the upstream gradients and the weight (a plain
 * progressive average: weight = 1/S): one walk over every Gaussian's fragments evaluates alpha and
 * the geometric factors once and sums the S samples' contributions, instead of S walks.
 *   a. for each sample s < S: sgs_backward_sample_terms with the workspace of the sgs_render call
 *      that produced it (or of a re-render with the same frame index), which stores that sample's
 *      winner and colour term per framebuffer pixel in `scratch`; the workspace may be reused for
 *      the next sample once this call is enqueued;
 *   b. sgs_backward_accumulate_samples: the walk; `first` = 1 clears the accumulators.
 * `scratch` holds sgs_backward_samples_scratch_size(camera, settings, S) bytes (12 bytes per
 * framebuffer pixel and sample, plus 8 per pixel, plus sgs_gps_count_law_size() with GPS), 256-byte
 * aligned; S is at most 1024. The samples' terms must be written in order s = 0, 1, ..., S - 1. Same
 * estimator and sgs_backward_finish as above; also Gaussian point splatting (scatter or hybrid
 * scheduling), where each fragment's alpha is replaced by the probability that the Gaussian puts a
 * point into the (sub)pixel: 1 - E[(1 - q)^N], q the share of the Gaussian's point density over the
 * pixel (a 3 x 3 Gauss-Legendre rule), N the point count the render draws (its law tabulated per
 * call in the scratch). */
size_t sgs_backward_samples_scratch_size(const sgs_camera* camera, const sgs_settings* settings, uint32_t n_samples);
int sgs_backward_sample_terms(const sgs_gaussians* gaussians, const sgs_camera* camera, const sgs_settings* settings,
                              const void* render_workspace, const float* grad_image, const float* grad_alpha,
                              const float* grad_depth, float weight, uint32_t sample, uint32_t n_samples,
                              void* scratch, void* stream);
int sgs_backward_accumulate_samples(const sgs_gaussians* gaussians, const sgs_camera* camera,
                                    const sgs_settings* settings, const float* grad_image, const float* grad_alpha,
                                    const float* grad_depth, float weight, uint32_t n_samples, int first,
                                    void* scratch, void* backward_workspace, void* stream);

/* Steps a and b in one call for S samples rendered by one sgs_render_samples call: `framebuffers`
 * points at that call's S framebuffers (the workspace's framebuffer section, consecutive, one key per
 * framebuffer pixel each); the winners' colours are recomputed per Gaussian (the same function the
 * sample pass evaluates) instead of read from a render workspace. Same scratch, weight, `first` and
 * sgs_backward_finish as above. */
int sgs_backward_accumulate_framebuffers(const sgs_gaussians* gaussians, const sgs_camera* camera,
                                         const sgs_settings* settings, const void* framebuffers, uint32_t n_samples,
                                         const float* grad_image, const float* grad_alpha, const float* grad_depth,
                                         float weight, int first, void* scratch, void* backward_workspace,
                                         void* stream);

/* The GPS backward's table of the point count's law (for inspection; the fused walk builds its own):
 * 1025 rows for lambda = 2^(-10 + 13 r / 1024), 32 (P(N = n), dP/dlambda) float pairs each, the last
 * term holding N >= 31. `out` holds sgs_gps_count_law_size() bytes, 8-byte aligned. */
size_t sgs_gps_count_law_size(void);
int sgs_gps_count_law(void* out, void* stream);

/* ---- Learned resolve (no counterpart in the reference) ------------------------------------------
 * A 6-layer 3x3 convolutional denoiser (8 -> 32 -> 32 -> 32 -> 32 -> 32 -> 3, ReLU between layers,
 * the last layer adds the mean colour back) that maps a few samples' features to the converged
 * image; plain progressive averaging (SGS_TEMPORAL_STATIC) stays the fallback. BF16 operands on the
 * sm_100a tensor cores (tcgen05), FP32 accumulation.
 *
 * Image arrays are NHWC: [batch][height][width][channels], 16-byte aligned. Features are FP16 with
 * 8 channels (sgs_denoise_features_finalize); activations and their gradients are BF16 with 16 or
 * 32 channels; the output is FP32 RGB [batch][height][width][3], premultiplied like `History`.
 *
 * Packed weights of one layer, BF16, [tap = 3 dy + dx][in_channel / 8][out_channel][in_channel % 8]
 * (features count as 16 input channels, 8..15 zero). A forward layer with weights W[co][ci][dy][dx]
 * (cross-correlation, zero padding 1) packs W; its data gradient packs W'[tap][n = ci][k = co] =
 * W[8 - tap][co][ci] and runs with the mask epilogue. */
#define SGS_DENOISE_LAYERS 6
#define SGS_DENOISE_WIDTH 32   /* hidden channels */
#define SGS_DENOISE_FEATURES 8 /* FP16 input channels: mean rgb, mean alpha, mean depth x scale,
                                  standard error of the mean luminance, winner change rate, 0 */

enum sgs_conv_epilogue {
    SGS_CONV_RELU = 0,  /* out = relu(conv + bias), BF16 */
    SGS_CONV_FINAL = 1, /* out[0..2] = conv[0..2] + bias[0..2] + residual features[0..2], FP32 RGB */
    SGS_CONV_MASK = 2   /* out = conv * (mask > 0), BF16: the data gradient through the ReLU below */
};

typedef struct sgs_conv3x3_args {
    const void* input;    /* in_channels 8: FP16 features; 16 or 32: BF16 */
    void* output;
    const void* weights;  /* sgs_conv3x3_weights_size(in, out) bytes, packed as above */
    const float* bias;    /* (out_channels); unused by SGS_CONV_MASK */
    const void* mask;     /* SGS_CONV_MASK: BF16 [..][out_channels] activation of the layer below */
    const void* residual; /* SGS_CONV_FINAL: the FP16 features */
    int32_t batch, height, width;
    int32_t in_channels;  /* 8 (features), 16 or 32 */
    int32_t out_channels; /* 16 or 32 */
    int32_t epilogue;     /* sgs_conv_epilogue */
} sgs_conv3x3_args;

/* Supported (in, out, epilogue): (8, 32, RELU), (32, 32, RELU), (32, 16, FINAL), (32, 32, MASK),
 * (16, 32, MASK). */
size_t sgs_conv3x3_weights_size(int32_t in_channels, int32_t out_channels);
int sgs_conv3x3(const sgs_conv3x3_args* conv, void* stream);

/* Adds the weight gradient sum_p dZ[p][co] * X[p + tap][ci] to grad_weights, FP32
 * [9][out_channels][16 or 32] (features count as 16 input channels), and sum_p dZ[p][co] to
 * grad_bias (out_channels). X is the layer input (as in sgs_conv3x3), dZ the BF16 gradient of the
 * layer output before its activation, [..][out_channels]. Supported (in, out): (8, 32), (32, 32),
 * (32, 16). Summation order is not fixed (atomic adds). */
int sgs_conv3x3_wgrad(const void* input, int32_t in_channels, const void* grad_output, int32_t out_channels,
                      int32_t batch, int32_t height, int32_t width, float* grad_weights, float* grad_bias,
                      void* stream);

/* Features of a run of samples. For every sample (a Reset-mode render: its image, alpha and depth,
 * and optionally the winner framebuffer of the render workspace, (depth bits << 32 | index) per
 * pixel at supersampling 1), accumulate into `accum` (8 floats per pixel; `first` starts the sums);
 * then finalize into the FP16 features. */
int sgs_denoise_features_accumulate(const float* image, const float* alpha, const float* depth,
                                    const uint64_t* framebuffer, float* accum, uint32_t n_pixels, int32_t first,
                                    void* stream);
int sgs_denoise_features_finalize(const float* accum, uint32_t n_pixels, uint32_t n_samples, float depth_scale,
                                  void* features, void* stream);

/* The whole denoiser: features -> FP32 RGB. `weights` holds the 6 packed layers back to back
 * (sgs_denoise_weights_size() bytes), `biases` 32 x 5 + 16 floats (the last layer's 3 used). */
size_t sgs_denoise_weights_size(void);
size_t sgs_denoise_scratch_size(int32_t batch, int32_t height, int32_t width);
int sgs_denoise(const void* features, int32_t batch, int32_t height, int32_t width, const void* weights,
                const float* biases, void* scratch, size_t scratch_bytes, float* output, void* stream);

/* Synchronises `stream` and reports whether a denoiser kernel gave up a bounded tensor-core wait
 * (SGS_ERROR_CUDA), clearing the flag. */
int sgs_denoise_status(void* stream);

/* Diagnostics (no counterpart in the reference): CUDA events (cudaEvent_t) that the calling
 * thread's next sgs_render calls record on their stream immediately before the first and after the
 * last kernel of the accumulate stage, so that callers can time that stage with cudaEventElapsedTime.
 * NULL, NULL disables the recording. */
void sgs_set_stage_events(void* accumulate_start, void* accumulate_end);

/* Diagnostics (no counterpart in the reference): caps the stochastic-transparency large-Gaussian
 * work queue at `max_entries` entries (0 restores the default, min(N, 2^18)) for the workspace
 * sizes and renders that follow, process-wide. Gaussians that find the queue full are rendered in
 * place by their warp (same framebuffer); tests use a small cap to exercise that path. */
void sgs_set_queue_limit(uint32_t max_entries);

/* Preactivated layout (README.md:139-142 of the reference lists it as a possible improvement): writes,
 * for each Gaussian of `gaussians` (scales, rotations and opacities are read), two float4 into `out`
 * ((N, 8) floats, 16-byte aligned device memory): the upper triangle of the 3-D covariance
 * R diag(exp(2 s)) R^T as (c11, c12, c13, c22), (c23, c33), then the opacity sigmoid and 1 when the
 * quaternion is usable (else 0). Computed once per model and passed as
 * sgs_gaussians.preactivated, it saves the per-sample rebuild; renders stay bit-identical. */
int sgs_preactivate(const sgs_gaussians* gaussians, float* out, void* stream);

/* Quantised layout (README.md:143-147 of the reference lists it as a possible improvement): encodes
 * the Gaussians of `gaussians` (means, scales, rotations, opacities and, when sh_half is not NULL,
 * sh_coefficients are read) into `records` ((N, 4) uint32, 16 bytes per Gaussian instead of 44:
 * position in 11-10-11 bits inside the box of its chunk of 256 consecutive Gaussians, rotation as the
 * three smallest components of the normalised quaternion in 10 bits each, log-scales and opacity
 * logit as IEEE half), `chunks` ((sgs_quantized_chunks(N), 8) floats: each chunk's lower corner and
 * extent) and `sh_half` ((N, B, 3) IEEE half). All three 16-byte aligned device memory. Passed as
 * sgs_gaussians.quantized / quantized_chunks / sh_half, they replace the float32 arrays in every pass;
 * the images then differ from the float32 ones by the quantisation (not bit-identical). Not usable with
 * the backward. Morton-ordered Gaussians (as Model.py loads them) keep the chunks small. */
uint32_t sgs_quantized_chunks(uint32_t n_gaussians);
int sgs_quantize(const sgs_gaussians* gaussians, void* records, float* chunks, void* sh_half, void* stream);

/* Measurement aid without a counterpart in the reference: launches `blocks` blocks of 256 threads,
 * each thread issuing `ops_per_thread` 64-bit atomic minimum reductions (red.min.u64, the merge of
 * every accumulate pass) into `slots` (n_slots u64 entries, a power of two, 8-byte aligned, device
 * memory). Pattern 0 spreads the reductions over unrelated slots; pattern 1 lets each thread walk
 * its own run of consecutive slots, as one lane of the row walker walks a framebuffer row. Time it
 * with events on `stream`: blocks * 256 * ops_per_thread reductions per launch give the ceiling
 * against which a render's atomics per second are read. */
int sgs_probe_atomic_min(void* slots, uint64_t n_slots, uint32_t ops_per_thread, uint32_t blocks, uint32_t pattern,
                         uint32_t seed, void* stream);

/* Process-wide frame index (render.cu:56-57 keeps it in a hidden static counter that starts at 0);
 * exposed so that random streams can be pinned and resumed. */
uint32_t sgs_get_frame_index(void);
void sgs_set_frame_index(uint32_t frame_index);

/* K of the k-buffer (render.cu:164, `_C.k_buffer_size`). */
uint32_t sgs_k_buffer_size(void);

/* ABI version of the loaded library (SGS_ABI_VERSION). */
int sgs_abi_version(void);

/* Human-readable description of the calling thread's last error ("" when none). */
const char* sgs_last_error(void);

#ifdef __cplusplus
}
#endif

#endif /* SGS_B200_H */
