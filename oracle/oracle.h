/*
 * CPU oracle for the Mufflon path-tracer hot path: TEST INFRASTRUCTURE ONLY.
 *
 * This library is a CPU restatement of the reference renderer's CPU path
 * (LBVH build, two-level traversal, pt_sample, the light tree, and the light
 * tracer's and bidirectional path tracer's samplers), written to check the
 * CUDA implementation in mufflon_b200/ bit for bit. Only tests/, the smoke()
 * entry point and bench.py's CPU-baseline leg load it. The product library
 * never links, loads or calls it.
 *
 * Parity status: the reference cannot be built here (its math library
 * "epsilon" and its cub dependency are missing), so there are no reference
 * outputs to pin against. The restatement is checked against hand-derived
 * known answers (Morton codes, PCG64 streams, Karras hierarchies, ray tests)
 * in tests/test_oracle_*.py; beyond those, parity is unpinned.
 */
#ifndef MUFFLON_ORACLE_H
#define MUFFLON_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
	uint32_t numVertices;
	uint32_t numTriangles;
	uint32_t numQuads;
	uint32_t numSpheres;
	const float* vertices;       /* 3 * numVertices */
	const float* normals;        /* 3 * numVertices */
	const float* uvs;            /* 2 * numVertices */
	const uint32_t* indices;     /* 3 * numTriangles, then 4 * numQuads */
	const uint16_t* faceMaterials; /* numTriangles + numQuads */
	const float* spheres;        /* 4 * numSpheres: center xyz, radius */
	const uint16_t* sphereMaterials; /* numSpheres */
} OrLod;

enum { OR_MAT_LAMBERT = 0, OR_MAT_TORRANCE = 1, OR_MAT_EMISSIVE = 2 };

typedef struct {
	int32_t type;
	float albedo[3];
	float roughness[2];
	int32_t shadowing;    /* 0 v-cavity, 1 smith */
	int32_t ndf;          /* 0 ggx (only GGX is supported) */
	float radiance[3];
	float scale[3];
	int32_t albedoTexture; /* index into the texture table or -1 */
	int32_t alphaTexture;  /* cut-out texture (first channel < 0.5 is transparent) or -1 */
} OrMaterial;

typedef struct {
	uint32_t width, height;
	const float* texels; /* width*height*4, row-major, y = 0 first */
} OrTexture;

typedef struct {
	uint32_t numLods;
	const OrLod* lods;
	uint32_t numInstances;
	const float* worldToInstance; /* 12 floats per instance, row-major 3x4 */
	const uint32_t* instanceLod;  /* UINT32_MAX marks a masked instance */
	uint32_t numMaterials;
	const OrMaterial* materials;
	uint32_t numTextures;
	const OrTexture* textures;
	uint32_t numPointLights;
	const float* pointLights;     /* 6 floats: position, intensity */
	int32_t hasBackground;
	float backgroundColor[3];
	float backgroundScale[3];
	float camPos[3], camDir[3], camUp[3];
	float vFov, nearPlane, farPlane;
	uint32_t width, height;
} OrSceneDesc;

typedef struct {
	int32_t seed;
	int32_t minPathLength;
	int32_t maxPathLength;
	int32_t neeCount;
	int32_t neePositionGuide;
	int32_t rrStartDepth;   /* extension: Russian roulette from this path length (0 = always, as the reference) */
} OrPtParams;

typedef struct {
	uint64_t rays;          /* extension + shadow rays traced */
	uint64_t shadowRays;
	uint64_t nodeVisits;    /* binary BVH nodes (64 B each) fetched */
	uint64_t instanceVisits;
	uint64_t triTests, quadTests, sphereTests;
} OrStats;

void* oracle_scene_create(const OrSceneDesc* desc);
void oracle_scene_destroy(void* scene);

/* BVH inspection. which = -1 selects the instance-level BVH, otherwise a LoD.
 * Returns the number of build primitives and internal nodes after collapse. */
int oracle_bvh_info(void* scene, int32_t which, int32_t* numPrims, int32_t* numInternal);
int oracle_bvh_get(void* scene, int32_t which, uint64_t* mortonSorted, int32_t* parents,
                   float* nodes /* 8 words per node: min3 max3 index primCount (as int bits) */,
                   int32_t* primIds);
int oracle_scene_aabb(void* scene, float* aabb6);
/* Light list (108 bytes per light) and tree (20 bytes per node) in the core's
 * device layout, and the sorted (instance << 32 | primitive) -> node-path code
 * map of the area lights. Arrays may be NULL to query the counts. */
/* Host time (ms, one thread) that building the scene's light list and tree took. */
double oracle_light_build_ms(void* scene);
int oracle_light_tree(void* scene, uint32_t* numLights, uint32_t* numNodes, uint32_t* numCodes, void* lights,
                      void* nodes, uint64_t* keys, uint32_t* codes, float* rootFlux);

/* Ray queries. rays: 6 floats per ray (origin, direction). */
int oracle_trace_first(void* scene, const float* rays, const float* geoNormals, float tmax,
                       uint32_t n, float* tOut, int32_t* instOut, int32_t* primOut,
                       float* surfParamsOut);
int oracle_trace_any(void* scene, const float* pointsA, const float* pointsB, uint32_t n,
                     uint8_t* occludedOut);

/* Path tracer (CpuPathTracer equivalent). */
void* oracle_pt_create(void* scene, const OrPtParams* params);
void oracle_pt_destroy(void* pt);
/* Gradient of a loss with respect to albedo texture texIndex (Lambert
 * vertices) by replaying spp samples per pixel from a fresh seed, with the
 * suffix sums and the gradient in double precision; imageGrad = dLoss/dImage
 * (W*H*3), gradOut = W_t*H_t*3 doubles. Requires Russian roulette off.
 * Returns 0 on invalid arguments. */
int oracle_albedo_gradient(void* pt, int32_t texIndex, uint32_t spp, const float* imageGrad, double* gradOut,
                           int32_t threads);
/* dLoss/dL (3 doubles) for the emitted radiance L = radiance x scale of
 * emissive material matIndex: the same replay of spp samples per pixel, each
 * term that material emits (emitter hits and next-event samples) adding
 * term / L. Russian roulette may be on. Returns 0 on invalid arguments. */
int oracle_emission_gradient(void* pt, int32_t matIndex, uint32_t spp, const float* imageGrad, double* gradOut,
                             int32_t threads);
int oracle_pt_iterate(void* pt, int32_t numThreads);
/* Cumulative target: 0 radiance (3 ch), 1 hit id (2 ch) */
int oracle_pt_get_target(void* pt, int32_t target, float* out);
int oracle_pt_stats(void* pt, OrStats* stats);
/* One iteration restricted to rows [y0, y1) (for bounded CPU baselines). */
int oracle_pt_iterate_rows(void* pt, int32_t numThreads, uint32_t y0, uint32_t y1);

/* Light tracer (CpuLightTracer equivalent, lt_common.hpp). */
typedef struct {
	int32_t seed;
	int32_t minPathLength;
	int32_t maxPathLength;
	int32_t density;        /* the Density target is enabled (it changes which connections are tested) */
} OrLtParams;
/* Photons leave point, triangle and quad lights and the colored background. */
void* oracle_lt_create(void* scene, const OrLtParams* params);
void oracle_lt_destroy(void* lt);
int oracle_lt_iterate(void* lt, int32_t numThreads);
/* Cumulative target: 0 radiance (3 ch), 1 lightness (1 ch), 2 density (1 ch) */
int oracle_lt_get_target(void* lt, int32_t target, float* out);
/* The last iteration's camera connections, W*H*maxPathLength slots (photon
 * major, then path length): pixels[k] = pixel index or -1, values[5k..5k+4] =
 * radiance rgb, lightness, density as added to the iteration buffer. */
int oracle_lt_records(void* lt, int32_t* pixels, float* values);
int oracle_lt_stats(void* lt, OrStats* stats);
/* Bidirectional path tracer (CpuBidirPathTracer equivalent, cpu_bpt.cpp);
 * the parameters are the light tracer's (density unused). */
void* oracle_bpt_create(void* scene, const OrLtParams* params);
void oracle_bpt_destroy(void* bpt);
int oracle_bpt_iterate(void* bpt, int32_t numThreads);
/* Cumulative target: 0 radiance (3 ch), 1 lightness (1 ch) */
int oracle_bpt_get_target(void* bpt, int32_t target, float* out);
/* The last iteration's contributions, W*H*(M*M + M) slots for maximum path
 * length M (pixel major): first the connections [view path length][light
 * vertex], then the emitter hits [view path length - 1]; pixels[k] = pixel
 * index or -1, values[4k..4k+3] = radiance rgb and lightness as added. */
int oracle_bpt_records(void* bpt, int32_t* pixels, float* values);
int oracle_bpt_stats(void* bpt, OrStats* stats);
/* Vertex connection and merging (CpuVcm equivalent, cpu_vcm.cpp); the
 * parameters are the light tracer's (density unused), the merge radius
 * relative to the scene's diagonal and the progressive switch. */
void* oracle_vcm_create(void* scene, const OrLtParams* params, float mergeRadius, int32_t progressive);
void oracle_vcm_destroy(void* vcm);
int oracle_vcm_iterate(void* vcm, int32_t numThreads);
/* Cumulative target: 0 radiance (3 ch), 1 lightness (1 ch), 2, 3 their variances */
int oracle_vcm_get_target(void* vcm, int32_t target, float* out);
/* The last iteration's contributions, W*H*(M*M + 2M) slots for maximum path
 * length M (pixel major): the connections [view path length][light vertex],
 * the emitter hits [view path length - 1], the merges [view path length - 1];
 * pixels[k] = pixel index or -1, values[4k..4k+3] = radiance rgb, lightness. */
int oracle_vcm_records(void* vcm, int32_t* pixels, float* values);
int oracle_vcm_stats(void* vcm, OrStats* stats);
/* The photon map's bucket count for a capacity, and the Wang hash that picks
 * a pixel's light subpath (for the tests of both). */
uint32_t oracle_vcm_map_size(uint32_t capacity);
uint32_t oracle_wang_hash(uint32_t x);
/* Wireframe renderer (CpuWireframe equivalent, wireframe_common.hpp);
 * the target is the cumulative "Border" image (3 channels). */
void* oracle_wireframe_create(void* scene, float lineWidth, int32_t maxTraceDepth);
void oracle_wireframe_destroy(void* wf);
int oracle_wireframe_iterate(void* wf, int32_t numThreads);
int oracle_wireframe_get_target(void* wf, float* out);
int oracle_wireframe_get_variance(void* wf, float* out);
/* Building blocks exposed for known-answer tests. */
int oracle_karras(const uint64_t* keys, int32_t n, int32_t* parents);
uint64_t oracle_pcg64_next(uint64_t* state);
uint64_t oracle_pcg64_seed(uint32_t seed);
uint64_t oracle_part_by_two21(uint32_t x);
uint32_t oracle_part_by_two10(uint32_t x);
/* Rebuilds the scene's LoD hierarchies with 63- or 30-bit Morton codes. */
int oracle_scene_rebuild_lod_bvhs(void* scene, int32_t mortonBits);
uint64_t oracle_scramble_seed(uint32_t x);
/* The first n outputs of GoldenRatio2D(seed) (rng.hpp:119-140). */
void oracle_golden_ratio2d(uint32_t seed, uint32_t n, uint64_t* out);
uint64_t oracle_part_by_two16(uint32_t x);
uint64_t oracle_morton_code16(uint32_t a, uint32_t b, uint32_t c);
uint64_t oracle_hilbert_code16(uint32_t a, uint32_t b, uint32_t c);
void oracle_sincos(float x, float* s, float* c);
float oracle_atan2(float y, float x);
float oracle_acos(float x);

#ifdef __cplusplus
}
#endif

#endif
