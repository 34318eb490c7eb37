// Host-side world model of the C API: objects, LoDs, instances, materials,
// textures, cameras, lights and scenarios (the parts of
// src/core/scene/world_container.hpp, object.hpp, lod.hpp, scenario.hpp that
// the path tracer consumes), plus the device-resident scene they are
// flattened into.
#pragma once

#include <algorithm>
#include <cstdint>
#include <map>
#include <new>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "../../../include/mufflon_core.h"
#include "../trace/scene_types.hpp"
#include "../lbvh/lbvh.hpp"
#include "../trace/wavefront.hpp"
#include "../trace/lt_api.hpp"
#include "light_build.hpp"

namespace mb {

// Page-locked host memory for geometry, so that a scene load copies it to
// the GPU at full link speed without a staging copy.
template < class T >
struct PinnedAllocator {
	using value_type = T;
	PinnedAllocator() = default;
	template < class U > PinnedAllocator(const PinnedAllocator<U>&) {}
	T* allocate(size_t n) {
		void* p = nullptr;
		if(cudaMallocHost(&p, std::max<size_t>(n, 1) * sizeof(T)) != cudaSuccess) throw std::bad_alloc();
		return static_cast<T*>(p);
	}
	void deallocate(T* p, size_t) { cudaFreeHost(p); }
	template < class U > bool operator==(const PinnedAllocator<U>&) const { return true; }
	template < class U > bool operator!=(const PinnedAllocator<U>&) const { return false; }
};
template < class T > using pinned_vector = std::vector<T, PinnedAllocator<T>>;

struct HostLod {
	pinned_vector<float> vertices, normals, uvs; // 3, 3, 2 per vertex
	pinned_vector<uint32_t> triIdx, quadIdx;     // 3 per triangle, 4 per quad
	pinned_vector<uint16_t> triMat, quadMat;
	pinned_vector<float> spheres;                // 4 per sphere
	pinned_vector<uint16_t> sphereMat;
	uint32_t num_vertices() const { return uint32_t(vertices.size() / 3); }
	uint32_t num_triangles() const { return uint32_t(triMat.size()); }
	uint32_t num_quads() const { return uint32_t(quadMat.size()); }
	uint32_t num_spheres() const { return uint32_t(sphereMat.size()); }
	uint32_t num_prims() const { return num_triangles() + num_quads() + num_spheres(); }
	bool bounds(float mn[3], float mx[3]) const;
};

struct HostObject {
	std::string name;
	uint32_t flags = 0;
	uint32_t id = 0;        // creation index (object_get_id)
	uint32_t lodSlots = 0;  // object_allocate_lod_slots; 0: highest added level + 1
	std::map<uint32_t, std::unique_ptr<HostLod>> lods;
	uint32_t lod_slot_count() const {
		if(lodSlots > 0) return lodSlots;
		return lods.empty() ? 1u : lods.rbegin()->first + 1u;
	}
};

// Instances of animation frame NO_FRAME exist in every frame; the world is
// shown at frame 0, so a scene holds the NO_FRAME and frame-0 instances.
constexpr uint32_t NO_FRAME = 0xFFFFFFFFu;

struct HostInstance {
	HostObject* object = nullptr;
	uint32_t index = 0;
	uint32_t frame = NO_FRAME;
	float worldToInstance[12] = { 1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0 };
};

struct HostTexture {
	std::string name;
	uint32_t width = 1, height = 1, channels = 4;
	std::vector<float> texels; // 4 per texel
};

struct HostMaterial {
	std::string name;
	int32_t type = MAT_LAMBERT;
	HostTexture* albedo = nullptr;
	HostTexture* roughness = nullptr;
	HostTexture* radiance = nullptr;
	HostTexture* alpha = nullptr;   // MaterialParams::alpha: cut-out where its first channel < 0.5
	float scale[3] = { 1, 1, 1 };
	int32_t shadowing = 1, ndf = 1;
	bool supported = true;
	bool emissionOverride = false; // mufflon_set_emitted_radiance: emission replaces radiance x scale
	float emission[3] = { 0, 0, 0 };
};

struct HostCamera {
	std::string name;
	float position[3] = { 0, 0, 0 };
	float dir[3] = { 0, 0, -1 };
	float up[3] = { 0, 1, 0 };
	float vFov = 0.7853982f;
	float nearPlane = 1e-4f, farPlane = 1e10f;
};

struct HostPointLight { std::string name; uint32_t frames = 1; float position[3] = { 0, 0, 0 }; float intensity[3] = { 1, 1, 1 }; };
struct HostBackground { std::string name; int32_t type = 0; float color[3] = { 0, 0, 0 }; float scale[3] = { 1, 1, 1 }; };

struct HostScenario {
	std::string name;
	uint32_t width = 800, height = 600;
	HostCamera* camera = nullptr;
	std::vector<uint32_t> pointLights;
	int32_t background = -1;
	std::vector<std::string> slotNames;
	std::vector<HostMaterial*> slotMaterials;
	std::vector<uint32_t> maskedInstances;
	// level of detail: per-instance over per-object over global (scenario.cpp:131-154)
	uint32_t globalLod = 0;
	std::map<const HostObject*, uint32_t> objectLods;
	std::map<uint32_t, uint32_t> instanceLods;    // instance index -> level
	std::vector<const HostObject*> maskedObjects;
	uint32_t effective_lod(const HostInstance& inst) const;
};

// Callbacks through which a scene loader supplies object LoDs on demand
// (mufflon_set_lod_loader, core_interface.h:355-357).
struct LodLoader {
	Boolean (*loadLod)(void*, ObjectHdl, uint32_t, Boolean) = nullptr;
	Boolean (*loadMatIndices)(void*, uint32_t, uint16_t*, uint32_t*) = nullptr;
	Boolean (*loadMetadata)(void*, LodMetadata*, size_t*) = nullptr;
	void* userParams = nullptr;
};

// Device buffers of one LoD. Buffers only grow: a reload of the same scene
// reuses them (capacities in elements).
struct DeviceLod {
	float* vertices = nullptr;
	float* normals = nullptr;
	float* uvs = nullptr;
	uint32_t* indices = nullptr;
	uint16_t* faceMat = nullptr;
	float4* spheres = nullptr;
	uint16_t* sphereMat = nullptr;
	size_t cap[7] = {};
	BvhBuffers bvh;
	DLod desc{};
	void release();
};

// The flattened scene resident in HBM (see scene_types.hpp).
struct DeviceScene {
	std::vector<DeviceLod> lods;
	std::vector<const HostLod*> lodSources;
	DLod* dLods = nullptr;
	float4* dW2I = nullptr;
	uint32_t* dInstLod = nullptr;
	float* dInstBoxes = nullptr;
	float* dInstCentroids = nullptr;
	BvhBuffers tlas;
	DMaterial* dMaterials = nullptr;
	std::vector<float4*> textureBuffers;
	std::vector<const HostTexture*> textureSources; // host texture of each device texture
	DTexture* dTextures = nullptr;
	DLight* dLights = nullptr;
	DLightNode* dLightNodes = nullptr;
	uint64_t* dLightKeys = nullptr;
	uint32_t* dLightCodes = nullptr;
	uint32_t numLights = 0, numLightNodes = 0;
	float* dInstI2W = nullptr;          // 12 per instance: instance-to-world
	float* dWideInstBoxes = nullptr;    // 6 per instance: tight boxes of the 8-wide instance level
	size_t wideBoxCap = 0;
	// inputs and scratch of the GPU light-tree build
	uint8_t* dLightMirror = nullptr;
	uint32_t* dLightFirst = nullptr;
	LightLodInfo* dLightLods = nullptr;
	uint32_t* dEmissiveQuads = nullptr;
	uint16_t* dQuadMaterial = nullptr;
	float* dPointLights = nullptr;
	size_t lightCap[7] = {};
	LightBuildScratch lightScratch;
	DScene desc{};
	float aabb[6] = { 0, 0, 0, 0, 0, 0 };
	bool valid = false;
	size_t cap[12] = {};
	// host-side times of the last load (ms) and its host-to-device bytes
	float loadMs[5] = {};          // total, geometry upload, object BVHs, instance BVH, lights/materials
	uint64_t loadH2dBytes = 0;
	void release();
};

struct MufflonInstance;
// Builds (or rebuilds) the device scene of the current scenario.
bool build_device_scene(MufflonInstance& inst, std::string& error);

struct RendererState {
	bool enabled = false;
	PtParams params{ 0, 0, 16, 1, 0 };
	int32_t blocksPerSm = 8;
	int32_t megakernel = 0;       // 0: wavefront stages (default), 1: single megakernel
	WfState wf{};
	void* wfMemory = nullptr;
	int32_t wfNee = 0;
	size_t wfPixels = 0;
	int32_t stageTiming = 0;      // record device time per stage kernel
	int32_t traversalStats = 0;   // count node visits, primitive tests, instance entries (wavefront kernels)
	int32_t traceBlocksPerSm = 6; // register budget of the wavefront trace kernel
	int32_t wavefrontBounces = 2; // bounces run as separate stage launches before the tail launch
	int32_t refillLanes = 32;     // idle trace lanes refilled together
	int32_t tailPaths = 98304;    // queue length at or below which the tail launch takes over
	int32_t iterationGraph = 1;   // replay the wavefront launches of an iteration as one CUDA graph
	int32_t planTail = 1;         // plan the tail bounce from the previous iteration's queue lengths
	int32_t stepLimit = 0;        // "Traversal step limit" of every renderer; 0: MAX_TRAVERSAL_STEPS
	int32_t sortBits = 12;        // "Ray sort bits": coherence binning of queued rays (0: off, <= 16)
	int32_t sortDirBits = 3;      // "Ray sort direction bits": 0, 3 (octant) or 6
	std::vector<unsigned char> planKey;
	int32_t plannedTail = -1;
	cudaGraphExec_t graphExec = nullptr;
	std::vector<unsigned char> graphKey;
	int32_t graphLaunches = 0;
	int32_t* dIteration = nullptr; // device copy of the iteration number read by the graph
	int32_t* hIteration = nullptr; // page-locked staging of it
	std::vector<cudaEvent_t> stageEvents;
	std::vector<unsigned char> stageKinds;
	float stageMs[WF_STAGES] = {};
	int32_t lastLaunches = 0;
	TraceCounters lastExtend{}, lastShadow{};
	bool targetRadiance = true;
	bool targetHitId = false;
	bool targetLightness = false;  // light tracer targets (lt_params.hpp:14-17)
	bool targetDensity = false;
	int32_t kind = 0;              // 0: "Pathtracer", 1: "Lighttracer", 2: "Wireframe", 3: "Bidirectional Pathtracer"
	WireParams wireParams{ 1.0f, 1000 }; // the wireframe renderer's "Line width" and "Maximum trace depth"
	bool targetBorder = true;      // its "Border" target
	// Variance recording per target (render_enable_render_target(name, true),
	// output_handler.hpp:391-431) and the buffers, allocated when first used:
	// running variances, and for "Density" (which reduces moments) its running mean.
	bool varRadiance = false, varHitId = false, varLightness = false, varDensity = false, varBorder = false;
	float* radianceVar = nullptr;  // 3 per pixel (also the "Border" variance)
	float* hitIdVar = nullptr;     // 2 per pixel
	float* lightnessVar = nullptr; // 1 per pixel
	float* densityMean = nullptr;  // 1 per pixel
	// The path tracer's auxiliary targets Position, Depth, Normal, UV, Albedo
	// (3, 1, 3, 2, 3 channels; "Lightness" uses the light tracer's flags and
	// buffers above): record / record-variance flags, cumulative and variance
	// buffers, and the per-path iteration state of the wavefront schedule.
	bool auxTarget[5] = {}, auxVarOn[5] = {};
	float* auxCum[5] = {};
	float* auxVarBuf[5] = {};
	void* auxMem = nullptr;
	size_t auxMemPixels = 0;
	LtParams ltParams{ 0, 0, 16 }; // the light tracer's own Seed / Min. / Max. path length
	int32_t ltRecord = 0;          // keep the light tracer's camera connections of the last iteration
	int32_t ltMegakernel = 0;      // light tracer: 0 stages per path length (default), 1 one persistent kernel
	void* ltWavefront = nullptr;   // its stage queues
	size_t ltWavefrontBytes = 0;
	LtParams bptParams{ 0, 0, 16 }; // the bidirectional path tracer's own parameters
	int32_t bptRecord = 0;         // keep its contributions of the last iteration
	int32_t bptMegakernel = 0;     // 0 stages per path length (default), 1 one persistent kernel
	void* bptScratch = nullptr;    // the persistent kernel's per-lane light subpaths
	size_t bptScratchBytes = 0;
	void* bptWavefront = nullptr;  // the stages' subpaths and queues
	size_t bptWavefrontBytes = 0;
	LtParams vcmParams{ 0, 0, 16 }; // vertex connection and merging: its own Seed / Min. / Max. path length
	float vcmMergeRadius = 0.001f; // "Relative merge radius" (of the scene's diagonal)
	int32_t vcmProgressive = 0;    // "Progressive"
	int32_t vcmRecord = 0;         // keep its contributions of the last iteration
	void* vcmMemory = nullptr;     // its stages' state and photon grid
	size_t vcmMemoryBytes = 0;
	size_t ltRecFloats = 0;        // floats allocated at ltRecValue
	float4* ltIter = nullptr;      // light tracer iteration buffers (radiance rgb + lightness, density)
	float* ltIterDensity = nullptr;
	float* lightness = nullptr;    // cumulative means of the 1-channel light tracer targets
	float* density = nullptr;
	int32_t* ltRecPixel = nullptr;
	float* ltRecValue = nullptr;
	size_t ltRecSlots = 0;
	bool needsReset = true;
	int32_t iteration = -1;
	uint32_t width = 0, height = 0;
	uint64_t* rng = nullptr;
	float* radiance = nullptr;
	float* hitId = nullptr;
	unsigned int* workCounter = nullptr;
	TraceCounters* counters = nullptr; // [0] extension rays, [1] shadow rays
	cudaEvent_t evStart = nullptr, evStop = nullptr;
	TraceCounters lastCounters{};
	float lastKernelMs = 0.0f;
	float* screen = nullptr;       // page-locked copy of the last target read back (library-owned)
	size_t screenCap = 0;          // its capacity in floats
	int screenChannels = 0;
	void release();
};

struct MufflonInstance {
	std::recursive_mutex iterationMutex;
	int device = 0;
	cudaStream_t stream = nullptr;
	std::vector<std::unique_ptr<HostObject>> objects;
	std::vector<std::unique_ptr<HostInstance>> instances;
	std::vector<std::unique_ptr<HostMaterial>> materials;
	std::vector<std::unique_ptr<HostTexture>> textures;
	std::vector<std::unique_ptr<HostCamera>> cameras;
	std::vector<HostPointLight> pointLights;
	std::vector<HostBackground> backgrounds;
	std::vector<std::unique_ptr<HostScenario>> scenarios;
	HostScenario* current = nullptr;
	LodLoader lodLoader;
	bool sceneDirty = true;
	DeviceScene scene;
	LbvhBuilder builder;
	RendererState renderer;
	~MufflonInstance();
};

} // namespace mb
