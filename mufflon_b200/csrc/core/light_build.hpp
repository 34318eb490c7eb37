// GPU construction of the scene's light list and light tree
// (world_container.cpp:869-990 area and point lights; light_tree.cpp:120-447
// LightTreeBuilder::build: Hilbert-order sort, balanced tree with extra bottom
// nodes, per-node fluxes, the (instance, primitive) -> node-path code map).
//
// The host decides what emits (a scan of each used LoD's face materials) and
// hands over, per instance, its instance-to-world matrix, mirroring flag and
// first light index; everything per light — transforming the corners,
// the Hilbert keys, the stable two-key sort, the flux of each light, the
// tree and the sorted code map — runs on the device, with the
// same float operations as the CPU restatement, so the tree is bit-identical.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "../trace/scene_types.hpp"

namespace mb {

class LbvhBuilder;

// Per used LoD: where its geometry is on the device and which of its faces emit.
struct LightLodInfo {
	const float* vertices;
	const float* uvs;             // nullptr: the LoD has no uvs (zeros are used)
	const uint32_t* indices;      // 3 per triangle, then 4 per quad
	uint32_t numTriangles;
	uint32_t faceListStart;       // into LightBuildInput::emissiveFaces
	uint32_t numQuads;
	const float4* spheres;        // centre, radius
};

struct LightBuildInput {
	uint32_t numInstances;
	const uint32_t* instLod;      // device: used-LoD index per instance (0xFFFFFFFF: none)
	const float* instToWorld;     // device: 12 floats per instance
	const uint8_t* mirroring;     // device: per instance, det of the 3x3 part < 0
	const uint32_t* instFirstLight; // device: numInstances + 1 prefix sums of emissive faces
	const LightLodInfo* lods;     // device: per used LoD
	const uint32_t* emissiveFaces;// device: per LoD, its emissive primitives (triangles, quads, then spheres; primitive index)
	const uint16_t* faceMaterial; // device: material slot of each entry of emissiveFaces
	uint32_t numArea;             // area lights (emissive faces over all instances)
	const float* pointLights;     // device: 6 floats (position, intensity) per point light
	uint32_t numPoint;
	const DMaterial* materials;   // device
	float sceneScale[3];          // scene box extent: lights are ordered along a Hilbert curve of centre * extent
};

// Grow-only device scratch of the build.
struct LightBuildScratch {
	uint32_t capacity = 0;
	DLight* unsorted = nullptr;
	int32_t* primInst = nullptr;  // per light before sorting: (instance, primitive) or -1
	int32_t* primId = nullptr;
	uint64_t* keyHi = nullptr;
	uint64_t* keyLo = nullptr;
	int32_t* order = nullptr;
	float* flux = nullptr;
	int32_t* sortedInst = nullptr;
	int32_t* sortedPrim = nullptr;
	void release();
};

struct LightBuildOutput {
	DLight* lights;               // device, numLights (sorted order)
	DLightNode* nodes;            // device, numLights - 1 when numLights > 1
	uint64_t* primKeys;           // device, numLights: sorted (instance << 32 | primitive); the first numArea are area lights
	uint32_t* primCodes;          // device, numLights
};

struct LightTreeInfo {
	float rootFlux = 0.0f;
	uint16_t rootType = LT_INTERNAL;
	int32_t rootIndex = 0;
	uint32_t numNodes = 0;
};

// Builds the light list and tree of numArea + numPoint lights into `out`
// (buffers sized for that many lights) and returns the root in `info`.
// Synchronises the stream once (for the root flux).
cudaError_t build_lights_gpu(const LightBuildInput& in, LightBuildScratch& scratch, LbvhBuilder& sorter,
                             const LightBuildOutput& out, LightTreeInfo& info, cudaStream_t stream);

} // namespace mb
