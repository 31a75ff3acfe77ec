// sgs_render_no_alloc: one sample-frame without any allocation, for callers that cannot allocate
// device memory while they render.
//
// Renderers embedded in a host application often run under a fixed device-memory budget owned by
// someone else: a viewer or game-engine plugin that must not touch the allocator in its frame
// callback, a C caller without PyTorch's caching allocator, or a caller that must not allocate
// between frames for latency reasons. They can still pass their own inputs and outputs, but not
// the scratch (winner framebuffer, samples, work queue) that sgs_render takes as a workspace.
//
// This entry point runs the same launch sequence as sgs_render with that scratch in a fixed
// device array of this file, kScratchBytes large:
//  * the array is a file-scope __device__ variable: a CUDA context that loads this file's module
//    holds it until the process exits (with lazy module loading, from the first call on that
//    device);
//  * host code cannot use the array's name as a device address. Every call looks the address up
//    with cudaGetSymbolAddress in the context current on the calling thread and checks the result,
//    so the address is always the one of the context the kernels run in: after cudaDeviceReset, or
//    for a caller that renders under its own driver context, the next call finds the array where
//    that context placed it (an address kept from an earlier context would dangle). The first call
//    in a context may load the module there: make it outside any stream capture;
//  * every call on a device shares the one array and it keeps the previous call's contents; the
//    render clears the parts that must start empty (framebuffer and queue counters) itself, so
//    nothing needs clearing by the caller, but calls that can overlap on the GPU (different
//    streams or threads without ordering) race on the array and must be serialised by the caller;
//  * requests whose scratch exceeds kScratchBytes are rejected with SGS_ERROR_WORKSPACE before any
//    launch. Stochastic transparency at 1920x1080 without supersampling or spatial reuse fits for
//    any scene size: at most 65.5 MB (framebuffer 16.6 MB, samples 33.2 MB, a work queue of at
//    most 2^18 entries of 60 bytes, 15.7 MB). Hybrid GPS sizes its work queue by max_binned
//    instead (by default min(N, 2^20) entries of 60 bytes): at 1920x1080 it fits up to about
//    289,000 entries, so scenes with more Gaussians need settings->max_binned at or below that.
// No cudaMalloc, cudaFree or allocating library routine is called.
#include <cuda_runtime.h>
#include "../../include/sgs_b200.h"
#include "sgs_internal.h"

namespace {

constexpr size_t kScratchBytes = size_t(64) << 20;  // 64 MiB
__device__ __align__(256) unsigned char g_no_alloc_scratch[kScratchBytes];

}  // namespace

extern "C" int sgs_render_no_alloc(const sgs_gaussians* gaussians, const sgs_camera* camera,
                                   const sgs_settings* settings, const sgs_history* history,
                                   const sgs_outputs* outputs, void* stream) {
    const size_t need = sgs_workspace_size(gaussians, camera, settings);
    if (need == 0) return SGS_ERROR_INVALID_ARGUMENT;  // sgs_last_error() names the bad argument
    if (need > kScratchBytes)
        return sgs::record_error(SGS_ERROR_WORKSPACE,
                                 "sgs_render_no_alloc: this render needs %zu bytes of scratch, the fixed "
                                 "array holds %zu (use sgs_render with a workspace)", need, kScratchBytes);
    void* scratch = nullptr;
    const cudaError_t err = cudaGetSymbolAddress(&scratch, g_no_alloc_scratch);
    if (err != cudaSuccess || scratch == nullptr)
        return sgs::record_error(SGS_ERROR_CUDA, "sgs_render_no_alloc: cudaGetSymbolAddress failed: %s",
                                 cudaGetErrorString(err));
    return sgs_render(gaussians, camera, settings, history, outputs, scratch, kScratchBytes, stream);
}
