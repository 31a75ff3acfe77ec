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
//  * host code cannot use the array's name as a device address, so the first call on each device
//    (with that device current) looks the address up with cudaGetSymbolAddress and keeps it; make
//    that first call outside any stream capture, since the lookup may load the module;
//  * every call on a device shares the one array and it keeps the previous call's contents; the
//    render clears the parts that must start empty (framebuffer and queue counters) itself, so
//    nothing needs clearing by the caller, but calls that can overlap on the GPU (different
//    streams or threads without ordering) race on the array and must be serialised by the caller;
//  * requests whose scratch exceeds kScratchBytes are rejected with SGS_ERROR_WORKSPACE before any
//    launch (1920x1080 without supersampling or spatial reuse fits for any scene size).
// No cudaMalloc, cudaFree or allocating library routine is called.
#include <atomic>
#include <cuda_runtime.h>
#include "../../include/sgs_b200.h"
#include "sgs_internal.h"

namespace {

constexpr size_t kScratchBytes = size_t(64) << 20;  // 64 MiB
constexpr int kMaxDevices = 64;

__device__ __align__(256) unsigned char g_no_alloc_scratch[kScratchBytes];

std::atomic<void*> g_scratch_address[kMaxDevices];

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
    int device = 0;
    if (cudaGetDevice(&device) != cudaSuccess || device < 0 || device >= kMaxDevices)
        return sgs::record_error(SGS_ERROR_CUDA, "sgs_render_no_alloc: no usable current device");
    void* scratch = g_scratch_address[device].load(std::memory_order_acquire);
    if (scratch == nullptr) {
        void* address = nullptr;
        const cudaError_t err = cudaGetSymbolAddress(&address, g_no_alloc_scratch);
        if (err != cudaSuccess || address == nullptr)
            return sgs::record_error(SGS_ERROR_CUDA, "sgs_render_no_alloc: cudaGetSymbolAddress failed: %s",
                                     cudaGetErrorString(err));
        g_scratch_address[device].store(address, std::memory_order_release);
        scratch = address;
    }
    return sgs_render(gaussians, camera, settings, history, outputs, scratch, kScratchBytes, stream);
}
