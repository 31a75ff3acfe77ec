// Host interface of the Gaussian-point-splatting form of the fused backward walk (backward_st.cu),
// beside the backward interface of sgs_internal.h: the walk needs the table of the point count's law,
// which it builds in caller scratch before walking.
#pragma once

#include <cstddef>
#include <cuda_runtime.h>
#include "sgs_internal.h"

namespace sgs {

// Bytes of the count-law table (1025 rows x 32 (P, dP/dlambda) float pairs).
size_t gps_count_law_bytes();

// Builds the count-law table in `law` alone.
cudaError_t launch_gps_count_law(float2* law, cudaStream_t stream);

// launch_backward_fragments_samples for GPS: builds the table in `law` (gps_count_law_bytes()), then
// walks every Gaussian's fragments with the GPS hit probability in place of alpha.
cudaError_t launch_backward_fragments_samples_gps(const BackwardParams& p, float2* law, cudaStream_t stream);

}  // namespace sgs
