// GPU LBVH builder (replaces LBVHBuilder::build of
// src/core/scene/accel_structs/build_lbvh.cu:587-811 and the cub calls of
// src/core/cuda/cu_lib_wrapper.cu:13-58, 364-405).
//
// Stages, each one kernel launch on the builder's stream:
//   1. Morton codes (63 bit) of primitive / instance centroids,
//   2. onesweep LSD radix sort of (code, index) pairs, 8 passes of 8 bits,
//      warp-level __match_any_sync ranking, shared-memory digit histograms,
//      decoupled look-back between tiles with bounded waits,
//   3. Karras hierarchy emit (parents, explicit child links),
//   4. bottom-up AABB / SAH / primitive-count merge with atomic arrival flags,
//   5. SAH collapse marks, inclusive scan, compaction into the reference's
//      32-byte BvhNode pair layout (lbvh.hpp:14-44),
//   6. for LoDs: a leaf-ordered triangle soup (3 x float4 per leaf slot),
//   7. conversion of the binary hierarchy into the compressed 8-wide one used
//      for traversal (wide.hpp), with its own primitive order and soup.
// All temporary storage is owned by the builder and reused across builds.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>
#include "../trace/scene_types.hpp"
#include "wide.hpp"

namespace mb {

struct LodBuildInput {
	uint32_t numTriangles, numQuads, numSpheres;
	const float* vertices;   // device, 3 per vertex
	const uint32_t* indices; // device, 3 per triangle then 4 per quad
	const float4* spheres;   // device
	float aabbMin[3], aabbMax[3];
};

struct SceneBuildInput {
	uint32_t numInstances;
	uint32_t activeInstances;
	const float* instBoxes;     // device, 6 per instance (min, max)
	const float* instCentroids; // device, 3 per instance
	const uint32_t* instanceLod;// device, UINT32_MAX = masked
	float aabbMin[3], aabbMax[3];
	// device, 6 per instance, or nullptr: boxes the 8-wide hierarchy is refitted
	// to (the binary hierarchy in the reference layout keeps instBoxes)
	const float* wideBoxes;
};

struct BvhBuffers {
	BvhNode* nodes = nullptr;      // device, capacity 2 * (n - 1)
	int32_t* primIds = nullptr;    // device, n
	float4* triSoup = nullptr;     // device, 3 * n (LoDs only)
	int32_t numPrims = 0;
	int32_t numInternal = 0;       // after collapse
	size_t nodeCapacity = 0;
	size_t primCapacity = 0;
	size_t soupCapacity = 0;
	// compressed 8-wide hierarchy used for traversal (wide.hpp)
	WideNode* wnodes = nullptr;    // device, numWide nodes
	int32_t* wprims = nullptr;     // device, n: wide leaf slot -> primitive id
	float4* wsoup = nullptr;       // device, 3 * n (LoDs only)
	int32_t numWide = 0;
	size_t wideCapacity = 0;
	size_t wprimCapacity = 0;
	size_t wsoupCapacity = 0;
	void release();
};

struct StageTimes { float morton, sort, emit, merge, mark, scan, compact, soup, wide; };

class LbvhBuilder {
public:
	LbvhBuilder() = default;
	~LbvhBuilder();
	LbvhBuilder(const LbvhBuilder&) = delete;
	LbvhBuilder& operator=(const LbvhBuilder&) = delete;

	// Builds into `out` (grown as needed). Returns cudaSuccess or the first
	// CUDA error; a failed bounded wait inside the sort is reported as
	// cudaErrorLaunchTimeout.
	cudaError_t build_lod(const LodBuildInput& in, BvhBuffers& out, cudaStream_t stream, bool withSoup = true);
	cudaError_t build_scene(const SceneBuildInput& in, BvhBuffers& out, cudaStream_t stream);

	// Intermediate results of the last build (device pointers, valid until the
	// next build): sorted Morton codes and the Karras parent array.
	const uint64_t* sorted_keys() const { return m_keysA; }
	const int32_t* parents() const { return m_parents; }
	int32_t last_num_prims() const { return m_lastN; }

	// Per-stage device times of the last build when timing is enabled.
	void enable_timing(bool on) { m_timing = on; }
	StageTimes last_times() const { return m_times; }

	// Standalone stable sort of (u64 key, i32 value) pairs; used by the
	// builder and exposed for tests. Results land in keys/values.
	// Stable sort by the low 8 * passes key bits (passes even, at most 8).
	cudaError_t sort_pairs(uint64_t* keys, int32_t* values, uint32_t n, cudaStream_t stream, int passes = 8);
	// Morton code width of the hierarchies: 63 (the reference's, default) or 30.
	void set_morton_bits(int bits) { m_mortonBits = bits == 30 ? 30 : 63; }

private:
	cudaError_t reserve(uint32_t n);
	cudaError_t build_common(int mode, const LodBuildInput* lod, const SceneBuildInput* scene,
	                         uint32_t numPrimitives, uint32_t used, BvhBuffers& out, cudaStream_t stream,
	                         bool withSoup);

	uint32_t m_capacity = 0;
	uint64_t* m_keysA = nullptr;
	uint64_t* m_keysB = nullptr;
	int32_t* m_valsA = nullptr;
	int32_t* m_valsB = nullptr;
	int32_t* m_parents = nullptr;     // 2n - 1
	int32_t* m_children = nullptr;    // 2 (n - 1)
	float4* m_nodeData = nullptr;     // 2 (2n - 1)
	unsigned int* m_flags = nullptr;  // n - 1
	int32_t* m_marks = nullptr;       // n - 1 (scanned in place)
	int2* m_ranges = nullptr;         // n - 1: sorted leaf range per internal node
	uint32_t* m_wideCounters = nullptr;
	int2* m_wideQueueA = nullptr;
	int2* m_wideQueueB = nullptr;
	uint32_t m_wideQueueCapacity = 0;
	int32_t* m_blockSums = nullptr;
	uint32_t* m_hist = nullptr;       // 8 * 256
	uint32_t* m_status = nullptr;     // tiles * 256
	uint32_t m_statusCapacity = 0;
	unsigned int* m_tileCounter = nullptr; // 8
	unsigned int* m_error = nullptr;
	int32_t* m_hostCount = nullptr;   // pinned
	int32_t m_lastN = 0;
	bool m_timing = false;
	int m_mortonBits = 63;
	StageTimes m_times{};
	cudaEvent_t m_ev[10] = {};
	// The 8-wide conversion of an object hierarchy runs on a stream of its own,
	// beside the reference-layout collapse: both only read the merged tree.
	cudaStream_t m_side = nullptr;
	cudaEvent_t m_fork = nullptr, m_join = nullptr;
	cudaEvent_t m_wideEv[2] = {};     // the conversion's start and end (timing)
};

} // namespace mb
