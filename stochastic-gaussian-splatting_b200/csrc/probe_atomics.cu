// Throughput probe of 64-bit atomic minimum reductions (red.min.u64), the merge operation of every
// accumulate pass. The measured rate is the ceiling that the fragment and point counts of a render
// are compared against (atomics issued per second of accumulate time).
//
// Thread t of the launch issues `ops` reductions into `slots` (a power of two of u64 entries).
// Pattern 0 (random): op i goes to slot h(t, i) & (slots - 1), with h the lowbias32 integer hash
// (Chris Wellons' hash-prospector constants), so consecutive reductions of a warp hit unrelated
// sectors. Pattern 1 (rows): lane t walks its own run of consecutive slots starting at
// h(t) * 2048, as a lane of the stochastic-transparency row walker walks one framebuffer row. The
// value of op i is (h(t, i) << 32) | t, so some minima change and most do not, as in a render.
//
// Everything is in bounds by construction: slot indices are masked with slots - 1 and the host
// entry point checks that `slots` is a power of two no larger than the buffer.
#include <cstdint>
#include <cuda_runtime.h>
#include "sgs_internal.h"

namespace sgs {
namespace {

constexpr uint32_t kProbeBlock = 256;

__device__ __forceinline__ uint32_t lowbias32(uint32_t x) {
    x ^= x >> 16;
    x *= 0x7feb352du;
    x ^= x >> 15;
    x *= 0x846ca68bu;
    x ^= x >> 16;
    return x;
}

__global__ void __launch_bounds__(kProbeBlock) atomic_min_probe_kernel(unsigned long long* __restrict__ slots,
                                                                       const uint64_t mask, const uint32_t ops,
                                                                       const uint32_t pattern, const uint32_t seed) {
    const uint32_t t = blockIdx.x * kProbeBlock + threadIdx.x;
    const uint32_t base = lowbias32(t ^ seed);
    const uint64_t row = static_cast<uint64_t>(base) * 2048u;
    for (uint32_t i = 0; i < ops; ++i) {
        const uint32_t h = lowbias32(base + i * 0x9E3779B9u);
        const uint64_t slot = (pattern == 0 ? static_cast<uint64_t>(h) : row + i) & mask;
        const unsigned long long value = (static_cast<unsigned long long>(h) << 32) | t;
        asm volatile("red.relaxed.gpu.global.min.u64 [%0], %1;" ::"l"(slots + slot), "l"(value) : "memory");
    }
}

}  // namespace

cudaError_t launch_atomic_min_probe(unsigned long long* slots, const uint64_t n_slots, const uint32_t ops,
                                    const uint32_t blocks, const uint32_t pattern, const uint32_t seed,
                                    cudaStream_t stream) {
    atomic_min_probe_kernel<<<blocks, kProbeBlock, 0, stream>>>(slots, n_slots - 1, ops, pattern, seed);
    return cudaGetLastError();
}

}  // namespace sgs
