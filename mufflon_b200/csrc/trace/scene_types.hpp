// Flat device-side scene layout consumed by the path-tracing kernels.
//
// The layout is a B200-oriented restatement of the reference's
// SceneDescriptor / LodDescriptor (src/core/scene/descriptors.hpp:26-222):
// plain arrays in HBM, no virtual dispatch, and per-LoD a "leaf-ordered
// triangle soup" so that a BVH leaf's triangles are read with consecutive
// 128-bit loads.
#pragma once

#include <cstdint>
#include <vector_types.h>

namespace mb {

struct WideNode; // lbvh/wide.hpp

enum : int32_t { MAT_LAMBERT = 0, MAT_TORRANCE = 1, MAT_EMISSIVE = 2 };
// Torrance shadowing models, numbered as core_interface.h ShadowingModel
enum : int32_t { SHADOW_VCAVITY = 0, SHADOW_SMITH = 1 };
enum : uint16_t { LT_POINT = 0, LT_TRI = 2, LT_QUAD = 3, LT_SPHERE = 4, LT_INTERNAL = 0xFFFF };

// Reference binary node (src/core/scene/accel_structs/lbvh.hpp:14-18):
// 32 bytes, two per internal node.
struct BvhNode {
	float mn[3];
	float mx[3];
	int32_t index;
	int32_t primCount;
};
static_assert(sizeof(BvhNode) == 32, "BvhNode layout");

struct DLod {
	uint32_t numTriangles, numQuads, numSpheres;
	int32_t numPrims;
	int32_t numInternal;          // nodes of the collapsed BVH (2 BvhNode each)
	const BvhNode* nodes;
	const int32_t* primIds;       // leaf slot -> primitive id
	const float4* triSoup;        // 3 float4 per leaf slot (only for triangle slots)
	const float* vertices;        // 3 per vertex
	const float* normals;         // 3 per vertex
	const float* uvs;             // 2 per vertex
	const uint32_t* indices;      // 3 per triangle, then 4 per quad
	const uint16_t* faceMaterials;
	const float4* spheres;        // center, radius
	const uint16_t* sphereMaterials;
	float aabbMin[3], aabbMax[3];
	// compressed 8-wide hierarchy used for traversal (lbvh/wide.hpp)
	const WideNode* wnodes;
	const int32_t* wprims;        // wide leaf slot -> primitive id
	const float4* wsoup;          // 3 float4 per wide leaf slot, primitive id in the first .w
	int32_t numWide;
};

struct DMaterial {
	int32_t type;
	float albedo[3];
	float roughness[2];
	float radiance[3];            // emission * scale
	int32_t albedoTex;            // -1: constant albedo
	int32_t shadowing;            // Torrance: SHADOW_VCAVITY or SHADOW_SMITH
	int32_t alphaTex;             // -1: opaque; else the alpha texture (first channel < 0.5 cuts)
};

struct DTexture {
	uint32_t width, height;
	const float4* texels;
};

struct DLight {
	uint16_t type;
	uint16_t material;
	float position[3];
	float intensity[3];
	float posV[4][3];             // quad: v0, v3-v0, v1-v0, v2-v3-(v1-v0); triangle: v0, v1-v0, v2-v0
	float uvV[4][2];
	float radius;                 // sphere (centre in position)
};

struct DLightNode {
	float leftFlux, rightFlux;
	int32_t leftIndex, rightIndex;
	uint16_t leftType, rightType;
};

struct DCamera {
	float position[3];
	float viewDir[3];
	float up[3];
	float tanVFov;
	uint16_t resX, resY;
};

// Per-pixel iteration channels of the path tracer's auxiliary targets
// (Position 3, Depth 1, Normal 3, UV 2, Albedo 3, Lightness 1).
constexpr int AUX_CHANNELS = 13;

// Default traversal step limit of a ray (DScene::maxSteps).
constexpr int32_t MAX_TRAVERSAL_STEPS = 1 << 22;

struct DScene {
	const DLod* lods;
	uint32_t numLods;
	const float4* worldToInstance; // 3 float4 (rows) per instance
	const uint32_t* instanceLod;
	uint32_t numInstances;
	int32_t activeInstances;
	uint32_t validInstance;
	const BvhNode* tlasNodes;
	const int32_t* tlasPrimIds;
	int32_t tlasNumInternal;
	const WideNode* tlasWide;
	const int32_t* tlasWidePrims; // wide leaf slot -> instance id
	int32_t tlasNumWide;
	const DMaterial* materials;
	const DTexture* textures;
	// light tree (src/core/scene/lights/light_tree.hpp)
	const DLight* lights;
	const DLightNode* lightNodes;
	const uint64_t* lightPrimKeys;  // sorted (instance << 32 | primitive) of hitable lights
	const uint32_t* lightPrimCodes; // node path codes matching lightPrimKeys
	uint32_t numLightPrims;
	float rootFlux;
	uint16_t rootType;
	int32_t rootIndex;
	float dirFlux;
	float bgFlux[3];
	int32_t hasBackground;
	float bgColor[3], bgScale[3];
	float aabbMin[3], aabbMax[3];
	DCamera camera;
	int32_t hasAlpha;             // some material has an alpha texture
	int32_t sphereLights;         // emissive spheres in the light list (their hit pdf needs the previous vertex)
	// Traversal steps a ray may take (per traversal loop of the binary
	// hierarchies, per ray of the 8-wide ones) before it is abandoned and
	// counted as an error; MAX_TRAVERSAL_STEPS unless the renderer parameter
	// "Traversal step limit" sets it.
	int32_t maxSteps;
};

struct PtParams {
	int32_t seed;
	int32_t minPathLength;
	int32_t maxPathLength;
	int32_t neeCount;
	int32_t rrStartDepth;
};

// Per-render-target device buffers and the per-pixel generator state.
struct RenderState {
	uint64_t* rngState;     // one PCG64 state per pixel
	float* radiance;        // cumulative mean, 3 per pixel (may be null)
	float* hitId;           // cumulative mean, 2 per pixel (may be null)
	float* iterRadiance;    // optional per-iteration radiance (may be null)
	float* radianceVar;     // running variances of the two targets (null: not recorded)
	float* hitIdVar;
	// the auxiliary targets Position, Depth, Normal, UV, Albedo, Lightness
	// (3, 1, 3, 2, 3, 1 channels per pixel): cumulative means and variances,
	// null where not recorded; auxOn: any of them is recorded
	float* aux[6];
	float* auxVar[6];
	int32_t auxOn;
	uint32_t width, height;
	int32_t iteration;      // 0 for the first iteration after a reset
	const int32_t* dIteration; // if set: the iteration number is read here (a replayed CUDA graph)
};

// Counters accumulated by the kernels (one atomic per thread at exit).
struct TraceCounters {
	unsigned long long rays;
	unsigned long long shadowRays;
	unsigned long long nodeVisits;
	unsigned long long primTests;
	unsigned long long instanceVisits;
	unsigned int errors;       // stack overflow or bounded-wait expiry
	unsigned int waitErrors;   // expired bounded waits outside traversal (the photon-grid sort)
};

} // namespace mb
