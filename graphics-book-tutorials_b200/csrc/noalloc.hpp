// Allocation-free render entry (noalloc.cu).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include "engine.hpp"

namespace wfb {

// Adds samples [first_sample, first_sample + count) of the resident scene (its own camera and
// resolution) to the caller's device film sums, on `stream`, with all scratch in a static device
// array. Throws wfb::Error for a scene resident on another device or pixels * count above
// WFB_NOALLOC_MAX_SAMPLES.
void render_passes_noalloc(const ResidentScene& scene, int first_sample, int count, uint32_t seed, int max_depth,
                           float* rgb_sum, float* lum_sum, float* lum2_sum, cudaStream_t stream);

}  // namespace wfb
