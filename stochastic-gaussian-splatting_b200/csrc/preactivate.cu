// Preactivated Gaussian layout (the first improvement the reference's README lists at
// README.md:139-142): the 3-D covariance and the opacity sigmoid, computed once per model instead of
// once per Gaussian and sample. Each Gaussian becomes two float4, (c11, c12, c13, c22) and
// (c23, c33, opacity, 1 when the quaternion is usable else 0), 32 B read by the projection in place
// of 12 B of log-scales, 16 B of quaternion and 4 B of logit and their 3 + 1 exponentials. The values
// come from the same device code the projection uses otherwise (cov3d_of, opacity_of), so renders
// with and without the layout produce the same bits.
#include <cstdint>
#include <cuda_runtime.h>
#include "sgs_internal.h"

namespace sgs {
namespace {

constexpr uint32_t kPreBlock = 256;

__global__ void __launch_bounds__(kPreBlock) preactivate_kernel(const float* __restrict__ scales,
                                                               const float4* __restrict__ rotations,
                                                               const float* __restrict__ opacities, const uint32_t n,
                                                               float4* __restrict__ out) {
    const uint32_t g = blockIdx.x * kPreBlock + threadIdx.x;
    if (g >= n) return;
    float4 v0, v1;
    preactivated_of(g, scales, rotations, opacities, v0, v1);
    out[2 * g] = v0;
    out[2 * g + 1] = v1;
}

}  // namespace

cudaError_t launch_preactivate(const float* scales, const float4* rotations, const float* opacities, const uint32_t n,
                               float4* out, cudaStream_t stream) {
    if (n == 0) return cudaSuccess;
    preactivate_kernel<<<(n + kPreBlock - 1) / kPreBlock, kPreBlock, 0, stream>>>(scales, rotations, opacities, n, out);
    return cudaGetLastError();
}

}  // namespace sgs
