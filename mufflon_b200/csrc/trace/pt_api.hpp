// Host-side launch interface of the path-tracing kernels.
#pragma once

#include <cuda_runtime.h>
#include "scene_types.hpp"

namespace mb {

cudaError_t launch_seed_rng(uint64_t* states, uint32_t numPixels, int32_t seed, cudaStream_t stream);

// One path-tracing iteration over pixels [pixelBegin, pixelEnd).
cudaError_t launch_pt(const DScene& scene, const PtParams& params, const RenderState& state,
                      unsigned int* workCounter, TraceCounters* counters, uint32_t pixelBegin,
                      uint32_t pixelEnd, int blocksPerSm, cudaStream_t stream);

cudaError_t launch_trace_rays(const DScene& scene, const float* rays, const float* geoNormals, float tmax,
                              uint32_t n, float* t, int32_t* inst, int32_t* prim, float* sp,
                              cudaStream_t stream);

cudaError_t launch_occlusion(const DScene& scene, const float* a, const float* b, uint32_t n, uint8_t* out,
                             cudaStream_t stream);

// Read bandwidth of an L2-resident buffer of `bytes` (GB/s).
cudaError_t measure_l2_bandwidth(size_t bytes, int reps, float* gbs);

} // namespace mb
