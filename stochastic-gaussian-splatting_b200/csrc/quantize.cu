// Quantised Gaussian layout, the second improvement the reference's README lists (README.md:143-147):
// smaller encodings of the parameters every sample reads, for memory and bandwidth. One block of
// 256 threads encodes one chunk of kQuantChunk consecutive Gaussians (Morton order keeps a chunk
// compact): the chunk's box (lo, extent) from a block-wide min/max of the means, then per Gaussian a
// 16-byte record (sgs_project.cuh): position 11-10-11 bits inside the box, rotation as the three
// smallest components of the normalised quaternion (10 bits each, levels 0..1022 so that 0 is exact)
// with the index of the largest, log-scales and opacity logit as IEEE half; the SH coefficients become
// IEEE half. 16 bytes instead of 44 per Gaussian for the accumulate pass, 96 instead of 192 for a
// winner's SH. Every operation of the encoder is rounded explicitly (no contraction, correctly
// rounded division and square root), so a float32 restatement reproduces the records bit for bit.
// Renders from the records are not bit-identical to the float32 ones; they are checked statistically.
#include <cstdint>
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include "../../include/sgs_b200.h"
#include "sgs_internal.h"

namespace sgs {
namespace {

constexpr uint32_t kQuantBlock = kQuantChunk;

__device__ __forceinline__ uint32_t quant_level(const float t, const float top) {
    const float q = rintf(__fmul_rn(t, top));
    return static_cast<uint32_t>(fminf(fmaxf(q, 0.0f), top));
}

__device__ __forceinline__ uint32_t half_bits(const float v) {
    return static_cast<uint32_t>(__half_as_ushort(__float2half_rn(v)));
}

__global__ void __launch_bounds__(kQuantBlock) quantize_kernel(
    const float* __restrict__ means, const float* __restrict__ scales, const float4* __restrict__ rotations,
    const float* __restrict__ opacities, const float* __restrict__ sh, const uint32_t sh_floats, const uint32_t n,
    uint4* __restrict__ records, float4* __restrict__ chunks, __half* __restrict__ sh_half) {
    __shared__ float s_lo[3][kQuantBlock / 32], s_hi[3][kQuantBlock / 32];
    __shared__ float s_box[6];
    const uint32_t g = blockIdx.x * kQuantBlock + threadIdx.x;
    const bool valid = g < n;
    float m[3];
    for (int c = 0; c < 3; ++c) m[c] = valid ? means[3 * static_cast<size_t>(g) + c] : 0.0f;
    // the chunk's box: warp min/max, then across the block's warps
    for (int c = 0; c < 3; ++c) {
        float lo = valid ? m[c] : __int_as_float(0x7f800000), hi = valid ? m[c] : -__int_as_float(0x7f800000);
        for (int o = 16; o > 0; o >>= 1) {
            lo = fminf(lo, __shfl_xor_sync(0xffffffffu, lo, o));
            hi = fmaxf(hi, __shfl_xor_sync(0xffffffffu, hi, o));
        }
        if ((threadIdx.x & 31u) == 0) {
            s_lo[c][threadIdx.x >> 5] = lo;
            s_hi[c][threadIdx.x >> 5] = hi;
        }
    }
    __syncthreads();
    if (threadIdx.x < 3) {
        float lo = s_lo[threadIdx.x][0], hi = s_hi[threadIdx.x][0];
        for (uint32_t w = 1; w < kQuantBlock / 32; ++w) {
            lo = fminf(lo, s_lo[threadIdx.x][w]);
            hi = fmaxf(hi, s_hi[threadIdx.x][w]);
        }
        s_box[threadIdx.x] = lo;
        s_box[3 + threadIdx.x] = __fsub_rn(hi, lo);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        chunks[2 * blockIdx.x] = make_float4(s_box[0], s_box[1], s_box[2], 0.0f);
        chunks[2 * blockIdx.x + 1] = make_float4(s_box[3], s_box[4], s_box[5], 0.0f);
    }
    if (!valid) return;

    // position: 11, 10 and 11 bits inside the box
    const float tops[3] = {2047.0f, 1023.0f, 2047.0f};
    const uint32_t shifts[3] = {21u, 11u, 0u};
    uint32_t w0 = 0;
    for (int c = 0; c < 3; ++c) {
        const float ext = s_box[3 + c];
        const float t = ext > 0.0f ? __fdiv_rn(__fsub_rn(m[c], s_box[c]), ext) : 0.0f;
        w0 |= quant_level(t, tops[c]) << shifts[c];
    }
    // rotation: the three smallest components of the normalised quaternion, the largest made positive
    const float4 r = rotations[g];
    const float rv[4] = {r.x, r.y, r.z, r.w};
    const float sq = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(r.x, r.x), __fmul_rn(r.y, r.y)), __fmul_rn(r.z, r.z)),
                               __fmul_rn(r.w, r.w));
    const float norm = __fsqrt_rn(sq);
    float u[4];
    for (int k = 0; k < 4; ++k) u[k] = norm > 0.0f ? __fdiv_rn(rv[k], norm) : (k == 0 ? 1.0f : 0.0f);
    uint32_t big = 0;
    float best = fabsf(u[0]);
    for (uint32_t k = 1; k < 4; ++k)
        if (fabsf(u[k]) > best) {
            best = fabsf(u[k]);
            big = k;
        }
    const float sign = u[big] < 0.0f ? -1.0f : 1.0f;
    uint32_t w1 = big << 30;
    uint32_t slot = 0;
    for (uint32_t k = 0; k < 4; ++k) {
        if (k == big) continue;
        const float c = __fmul_rn(u[k], sign);
        const float v = __fmul_rn(__fadd_rn(__fmul_rn(c, 1.41421356f), 1.0f), 0.5f);
        w1 |= quant_level(v, 1022.0f) << (20u - 10u * slot);
        ++slot;
    }
    const uint32_t w2 = half_bits(scales[3 * static_cast<size_t>(g)]) |
                        (half_bits(scales[3 * static_cast<size_t>(g) + 1]) << 16);
    const uint32_t w3 = half_bits(scales[3 * static_cast<size_t>(g) + 2]) | (half_bits(opacities[g]) << 16);
    records[g] = make_uint4(w0, w1, w2, w3);
    if (sh_half != nullptr)
        for (uint32_t i = 0; i < sh_floats; ++i)
            sh_half[static_cast<size_t>(g) * sh_floats + i] = __float2half_rn(sh[static_cast<size_t>(g) * sh_floats + i]);
}

}  // namespace

cudaError_t launch_quantize(const float* means, const float* scales, const float4* rotations, const float* opacities,
                            const float* sh, const uint32_t sh_floats, const uint32_t n, uint4* records,
                            float4* chunks, __half* sh_half, cudaStream_t stream) {
    if (n == 0) return cudaSuccess;
    quantize_kernel<<<(n + kQuantBlock - 1) / kQuantBlock, kQuantBlock, 0, stream>>>(
        means, scales, rotations, opacities, sh, sh_floats, n, records, chunks, sh_half);
    return cudaGetLastError();
}

}  // namespace sgs

extern "C" uint32_t sgs_quantized_chunks(uint32_t n_gaussians) {
    return (n_gaussians + sgs::kQuantChunk - 1) / sgs::kQuantChunk;
}

extern "C" int sgs_quantize(const sgs_gaussians* g, void* records, float* chunks, void* sh_half, void* stream) {
    if (g == nullptr) return sgs::record_error(SGS_ERROR_INVALID_ARGUMENT, "sgs_quantize: null argument");
    if (g->n_gaussians == 0) return SGS_OK;
    if (!g->means || !g->scales || !g->rotations || !g->opacities || records == nullptr || chunks == nullptr)
        return sgs::record_error(SGS_ERROR_INVALID_ARGUMENT, "sgs_quantize: null Gaussian array or output");
    if ((reinterpret_cast<uintptr_t>(g->rotations) | reinterpret_cast<uintptr_t>(records) |
         reinterpret_cast<uintptr_t>(chunks)) & 15u)
        return sgs::record_error(SGS_ERROR_INVALID_ARGUMENT,
                                 "sgs_quantize: rotations, records and chunks must be 16-byte aligned");
    if (sh_half != nullptr && (g->sh_coefficients == nullptr ||
                               (g->sh_bases != 1 && g->sh_bases != 4 && g->sh_bases != 9 && g->sh_bases != 16)))
        return sgs::record_error(SGS_ERROR_INVALID_ARGUMENT, "sgs_quantize: SH needs 1, 4, 9 or 16 bases");
    const cudaError_t err = sgs::launch_quantize(
        g->means, g->scales, reinterpret_cast<const float4*>(g->rotations), g->opacities, g->sh_coefficients,
        g->sh_bases * 3, g->n_gaussians, static_cast<uint4*>(records), reinterpret_cast<float4*>(chunks),
        static_cast<__half*>(sh_half), static_cast<cudaStream_t>(stream));
    if (err != cudaSuccess) return sgs::record_error(SGS_ERROR_CUDA, "sgs_quantize launch: %s", cudaGetErrorString(err));
    return SGS_OK;
}
