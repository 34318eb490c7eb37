// Host-side launch interface of the light tracer (the CUDA "Lighttracer").
#pragma once

#include <cuda_runtime.h>
#include "scene_types.hpp"

namespace mb {

// lt_params.hpp:8-12
struct LtParams {
	int32_t seed;
	int32_t minPathLength;
	int32_t maxPathLength;
};

// Output of one light-tracing iteration. Photons land in arbitrary pixels, so
// they are added to an iteration buffer with atomics; the running means are
// updated from it after all photons have finished.
struct LtTargets {
	uint64_t* rngState;   // one PCG64 state per photon (photon i uses the generator of pixel i)
	float4* iter;         // iteration buffer: radiance rgb, lightness (zeroed by launch_lt)
	float* iterDensity;   // iteration buffer of the density (zeroed by launch_lt)
	float* radiance;      // cumulative means: 3 per pixel (may be null)
	float* lightness;     // 1 per pixel (may be null)
	float* density;       // 1 per pixel; null: the Density target is off, which also
	                      // skips the connections that carry no radiance (lt_common.hpp:51)
	float* radianceVar;   // running variances of Radiance and Lightness, and the running
	float* lightnessVar;  // mean of Density (its target reduces moments); null: not recorded
	float* densityMean;
	int32_t* recPixel;    // optional connection records: maxPathLength slots per photon,
	float* recValue;      // pixel (-1: none) and radiance rgb, lightness, density as added
	uint32_t width, height;
	int32_t iteration;    // 0 for the first iteration after a reset
};

// One light-tracing iteration (width * height photons): clears the iteration
// buffers and records, traces the photons, updates the running means. With
// `wavefront` (ltw_bytes(width * height) bytes of device memory) in stages
// per path length; without, in one persistent kernel. Both give the same
// connections; the wavefront takes at most LTW_MAX_LAUNCHES path lengths.
constexpr int LTW_MAX_LAUNCHES = 64;
size_t ltw_bytes(size_t numPhotons);
cudaError_t launch_lt(const DScene& scene, const LtParams& params, const LtTargets& targets,
                      unsigned int* workCounter, TraceCounters* counters, cudaStream_t stream, void* wavefront);

// Bytes of the bidirectional path tracer's per-lane light-subpath storage
// (one slice of max. path length vertices per resident thread), used by the
// single-kernel schedule.
size_t bpt_scratch_bytes(int maxPathLength);

// Bytes of the staged schedule's device memory for numPixels pixels: every
// pixel's light subpath, its last two view vertices, the segment queues and
// up to max. path length connections per pixel and path length.
constexpr int BPTW_MAX_PATH = 64;
size_t bptw_bytes(size_t numPixels, int maxPathLength);

// One bidirectional path-tracing iteration (one light and one view subpath
// per pixel) into the same targets as the light tracer (radiance and
// lightness; no density); records hold 4 floats per slot, M*M + M slots per
// pixel for maximum path length M. With `wavefront` (bptw_bytes bytes) in
// stages per path length (at most BPTW_MAX_PATH); without, in one persistent
// kernel with `scratch` (bpt_scratch_bytes bytes). Both give the same
// contributions.
cudaError_t launch_bpt(const DScene& scene, const LtParams& params, const LtTargets& targets, void* scratch,
                       unsigned int* workCounter, TraceCounters* counters, cudaStream_t stream, void* wavefront);

// vcm_params.hpp:8-14 beyond the light tracer's three: "Relative merge
// radius" (of the scene's diagonal, default 0.001) and "Progressive" (the
// radius shrinks as iteration^(-1/6)).
struct VcmSettings {
	float mergeRadius;
	int32_t progressive;
};

// The photon map's bucket count for `capacity` photon slots
// (photon_map.hpp:216-229), and the device memory of one vertex connection
// and merging iteration over numPixels pixels: the bidirectional stages'
// state plus the photon grid (keys, sort buffers, bucket ranges, 80 B of merge
// data per photon slot).
uint32_t vcm_map_size(uint32_t capacity);
size_t vcm_bytes(size_t numPixels, int maxPathLength);

// One vertex connection and merging iteration (cpu_vcm.cpp:148-290) in stages
// per path length, into the light tracer's targets (radiance, lightness);
// records hold 4 floats per slot, M*M + 2M slots per pixel for max. path
// length M (connections [view length][light vertex], emitter hits and merges
// [view length - 1]). memory: vcm_bytes bytes.
cudaError_t launch_vcm(const DScene& scene, const LtParams& params, const VcmSettings& vcm, const LtTargets& targets,
                       TraceCounters* counters, cudaStream_t stream, void* memory);

// wireframe_params.hpp:6-26
struct WireParams {
	float lineWidth;        // "Line width" in pixels (default 1)
	int32_t maxTraceDepth;  // "Maximum trace depth" (default 1000)
};

// One wireframe iteration: one camera ray per pixel (generators in
// targets.rngState), the "Border" value per pixel into targets.iter and its
// running mean into targets.radiance. instToWorld: 12 floats per instance.
cudaError_t launch_wireframe(const DScene& scene, const float* instToWorld, const WireParams& params,
                             const LtTargets& targets, TraceCounters* counters, cudaStream_t stream);

} // namespace mb
