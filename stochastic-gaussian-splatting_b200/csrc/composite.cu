// Frame compositing of the renderer plugin (Renderer.py:91-97 of the reference), on the device:
// alpha clamped to [0, 1], the premultiplied colour composited over the background colour and
// clamped, the premultiplied depth divided by max(alpha, 1e-8). Each operation is rounded like the
// separate elementwise tensor operations a caller would run (IEEE round-to-nearest, no contraction,
// a correctly rounded division), so the results equal those operations bit for bit; as one kernel
// the compositing can sit in the CUDA graph of a progressive frame.
#include <cstdint>
#include <cuda_runtime.h>
#include "../../include/sgs_b200.h"
#include "sgs_internal.h"

namespace sgs {
namespace {

constexpr uint32_t kCompositeBlock = 256;

__global__ void __launch_bounds__(kCompositeBlock) composite_kernel(
    const float* __restrict__ image, const float* __restrict__ depth, const float* __restrict__ alpha,
    const float* __restrict__ background, const uint32_t n, float* __restrict__ rgb_out,
    float* __restrict__ depth_out, float* __restrict__ alpha_out) {
    const uint32_t i = blockIdx.x * kCompositeBlock + threadIdx.x;
    if (i >= n) return;
    const float a = fminf(fmaxf(alpha[i], 0.0f), 1.0f);
    const float t = __fsub_rn(1.0f, a);
#pragma unroll
    for (uint32_t c = 0; c < 3; ++c) {
        const float v = __fadd_rn(image[3 * i + c], __fmul_rn(t, background[c]));
        rgb_out[3 * i + c] = fminf(fmaxf(v, 0.0f), 1.0f);
    }
    if (alpha_out != nullptr) alpha_out[i] = a;
    if (depth_out != nullptr) depth_out[i] = __fdiv_rn(depth[i], fmaxf(a, 1.0e-8f));
}

}  // namespace

cudaError_t launch_composite(const float* image, const float* depth, const float* alpha, const float* background,
                             const uint32_t n, float* rgb, float* depth_out, float* alpha_out, cudaStream_t stream) {
    if (n == 0) return cudaSuccess;
    composite_kernel<<<(n + kCompositeBlock - 1) / kCompositeBlock, kCompositeBlock, 0, stream>>>(
        image, depth, alpha, background, n, rgb, depth_out, alpha_out);
    return cudaGetLastError();
}

}  // namespace sgs

extern "C" int sgs_composite(const float* image, const float* depth, const float* alpha, const float* background_rgb,
                             uint32_t n_pixels, float* rgb, float* depth_out, float* alpha_out, void* stream) {
    if (n_pixels == 0) return SGS_OK;
    if (image == nullptr || alpha == nullptr || background_rgb == nullptr || rgb == nullptr ||
        (depth_out != nullptr && depth == nullptr))
        return sgs::record_error(SGS_ERROR_INVALID_ARGUMENT, "sgs_composite: null image, alpha, background or output");
    const cudaError_t err = sgs::launch_composite(image, depth, alpha, background_rgb, n_pixels, rgb, depth_out,
                                                  alpha_out, static_cast<cudaStream_t>(stream));
    if (err != cudaSuccess)
        return sgs::record_error(SGS_ERROR_CUDA, "sgs_composite launch: %s", cudaGetErrorString(err));
    return SGS_OK;
}
