/*
 * C ABI of the B200 path-tracer core (libmufflon_core.so).
 *
 * This is the subset of Mufflon's core interface that examples/example.c,
 * examples/example.cpp and the Python binding (src/pythonbinding/bindings.py)
 * use to build a scene, select the path tracer, iterate and read the image
 * back. Type layouts, enum values and function signatures are identical to
 * src/core/export/core_interface.h so that an existing caller links against
 * this library unchanged; each function names the declaration it replaces.
 *
 * Conventions (src/core/export/interface.cpp:53-83): no exception crosses the
 * ABI; a failing call logs, stores a message for core_get_dll_error() and
 * returns false / NULL / INVALID_INDEX. Handles are opaque pointers owned by
 * the instance. One CUDA device per process.
 *
 * Functions marked EXTENSION have no reference counterpart.
 */
#ifndef MUFFLON_B200_CORE_H
#define MUFFLON_B200_CORE_H

#include <stdint.h>
#include <stddef.h>
#include <stdio.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CORE_API __attribute__((visibility("default")))
#define CDECL

/* ---- types: core_interface.h:16-333 ---- */
typedef uint32_t Boolean;
typedef struct { float x, y; } Vec2;
typedef struct { float x, y, z; } Vec3;
typedef struct { float x, y, z, w; } Vec4;
typedef struct { uint32_t x, y, z; } UVec3;
typedef struct { uint32_t x, y, z, w; } UVec4;
typedef struct { int32_t x, y; } IVec2;
typedef struct { float v[12u]; } Mat3x4;
typedef struct { Vec3 min; Vec3 max; } AABB;
typedef struct { uint64_t cycles; uint64_t microseconds; } ProcessTime;

typedef enum { CAM_PINHOLE, CAM_FOCUS, CAM_COUNT } CameraType;
typedef enum { LIGHT_POINT, LIGHT_SPOT, LIGHT_DIRECTIONAL, LIGHT_ENVMAP, LIGHT_COUNT } LightType;
typedef enum { BACKGROUND_MONOCHROME, BACKGROUND_ENVMAP, BACKGROUND_SKY_HOSEK, BACKGROUND_COUNT } BackgroundType;
typedef enum { SAMPLING_NEAREST, SAMPLING_LINEAR } TextureSampling;
typedef enum { SHADOWING_VCAVITY, SHADOWING_SMITH } ShadowingModel;
typedef enum { NDF_BECKMANN, NDF_GGX, NDF_COSINE } NormalDistFunction;
typedef enum {
	MATERIAL_EMISSIVE, MATERIAL_LAMBERT, MATERIAL_ORENNAYAR, MATERIAL_TORRANCE, MATERIAL_WALTER,
	MATERIAL_BLEND, MATERIAL_FRESNEL, MATERIAL_MICROFACET, MATERIAL_NUM
} MaterialParamType;
typedef enum { MEDIUM_NONE, MEDIUM_DIELECTRIC, MEDIUM_CONDUCTOR } OuterMediumType;
typedef enum { MIPMAP_NONE, MIPMAP_AVG, MIPMAP_MIN, MIPMAP_MAX } MipmapType;
/* texture_data.h:10-31 */
typedef enum {
	FORMAT_R8U, FORMAT_RG8U, FORMAT_RGBA8U, FORMAT_R16U, FORMAT_RG16U, FORMAT_RGBA16U, FORMAT_R16F, FORMAT_RG16F,
	FORMAT_RGBA16F, FORMAT_R32F, FORMAT_RG32F, FORMAT_RGBA32F, FORMAT_RGB8U, FORMAT_RGB16U, FORMAT_RGB16F,
	FORMAT_RGB32F, FORMAT_NUM
} TextureFormat;
typedef enum { LOG_PEDANTIC, LOG_INFO, LOG_WARNING, LOG_ERROR, LOG_FATAL_ERROR } LogLevel;
typedef enum { NONE = 0, OBJ_EMISSIVE = 1 } ObjectFlags;
typedef enum { PARAM_INT, PARAM_FLOAT, PARAM_BOOL, PARAM_ENUM } ParameterType;
typedef enum { BULK_FILE, BULK_ARRAY } BulkType;
typedef enum { DEVICE_NONE = 0u, DEVICE_CPU = 1u, DEVICE_CUDA = 2u, DEVICE_OPENGL = 4u } RenderDevice;

typedef struct { uint32_t type : 3; uint32_t index : 29; } LightHdl;

typedef int32_t IndexType;
typedef IndexType VertexHdl;
typedef IndexType FaceHdl;
typedef IndexType SphereHdl;
typedef uint32_t LodLevel;
typedef uint16_t MatIdx;
typedef void* ObjectHdl;
typedef void* ConstObjectHdl;
typedef void* LodHdl;
typedef void* InstanceHdl;
typedef void* ScenarioHdl;
typedef const void* ConstScenarioHdl;
typedef void* SceneHdl;
typedef void* MaterialHdl;
typedef void* CameraHdl;
typedef void* TextureHdl;
/* core_interface.h:237-239 */
typedef Vec4 (*TextureCallback)(uint32_t x, uint32_t y, uint32_t layer, TextureFormat format, Vec4 value, void* userParams);
typedef const void* ConstCameraHdl;
typedef void* MufflonInstanceHdl;
typedef const void* ConstMufflonInstanceHdl;

typedef struct { Vec2 refractionIndex; Vec3 absorption; } Medium;
typedef struct { TextureHdl albedo; } LambertParams;
typedef struct { TextureHdl roughness; ShadowingModel shadowingModel; NormalDistFunction ndf; TextureHdl albedo; } TorranceParams;
typedef struct { TextureHdl roughness; ShadowingModel shadowingModel; NormalDistFunction ndf; Vec3 absorption; float refractionIndex; } WalterParams;
typedef struct { TextureHdl radiance; Vec3 scale; } EmissiveParams;
typedef struct { TextureHdl albedo; float roughness; } OrennayarParams;
struct MaterialParamsStruct;
typedef struct { float factor; struct MaterialParamsStruct* mat; } BlendLayer;
typedef struct { BlendLayer a; BlendLayer b; } BlendParams;
typedef struct { Vec2 refractionIndex; struct MaterialParamsStruct* a; struct MaterialParamsStruct* b; } FresnelParams;
typedef struct { TextureHdl map; TextureHdl maxMips; float bias; float scale; } MaterialParamsDisplacement;
typedef struct MaterialParamsStruct {
	Medium outerMedium;
	MaterialParamType innerType;
	TextureHdl alpha;
	MaterialParamsDisplacement displacement;
	union {
		LambertParams lambert;
		TorranceParams torrance;
		WalterParams walter;
		EmissiveParams emissive;
		OrennayarParams orennayar;
		BlendParams blend;
		FresnelParams fresnel;
	} inner;
} MaterialParams;

typedef struct {
	BulkType type;
	union { FILE* file; const char* bytes; } descriptor;
} BulkLoader;

/* core_interface.h:77-83 */
typedef struct {
	uint32_t vertices;
	uint32_t triangles;
	uint32_t quads;
	uint32_t edges;
	uint32_t spheres;
} LodMetadata;

#define INVALID_INDEX ((int32_t)-1)

/* ---- instance, logging: core_interface.h:345-353 ---- */
CORE_API const char* CDECL core_get_dll_error(void);
CORE_API Boolean CDECL core_set_logger(void (*logCallback)(const char*, int));
CORE_API Boolean CDECL core_set_log_level(LogLevel level);
CORE_API MufflonInstanceHdl CDECL mufflon_initialize(void);
CORE_API void CDECL mufflon_destroy(MufflonInstanceHdl instHdl);
CORE_API int32_t CDECL mufflon_get_cuda_device_index(void);
CORE_API Boolean CDECL mufflon_is_cuda_available(void);
/* core_interface.h:355-357: a scene loader registers these; the core calls
 * func(userParams, obj, lod, asReduced) when a scenario needs a LoD that the
 * object does not hold yet (objFunc and metaFunc are kept for the loader's
 * own use). Passing func = NULL unregisters. */
CORE_API Boolean CDECL mufflon_set_lod_loader(MufflonInstanceHdl instHdl, Boolean (*func)(void*, ObjectHdl, uint32_t, Boolean),
                                              Boolean (*objFunc)(void*, uint32_t, uint16_t*, uint32_t*),
                                              Boolean (*metaFunc)(void*, LodMetadata*, size_t*), void* userParams);

/* ---- image readback: core_interface.h:359-360 ---- */
CORE_API Boolean CDECL mufflon_get_target_image(MufflonInstanceHdl instHdl, const char* name, Boolean variance, const float** ptr);
CORE_API Boolean CDECL mufflon_get_target_image_num_channels(MufflonInstanceHdl instHdl, int* numChannels);

/* ---- world: core_interface.h:365-366 ---- */
CORE_API void CDECL world_clear_all(MufflonInstanceHdl instHdl);
CORE_API Boolean CDECL world_finalize(MufflonInstanceHdl instHdl, const Vec3 min, const Vec3 max, const char** msg);

/* ---- polygons: core_interface.h:369-408 ---- */
CORE_API Boolean CDECL polygon_reserve(LodHdl lvlDtl, size_t vertices, size_t tris, size_t quads);
CORE_API VertexHdl CDECL polygon_add_vertex(LodHdl lvlDtl, Vec3 point, Vec3 normal, Vec2 uv);
CORE_API FaceHdl CDECL polygon_add_triangle(LodHdl lvlDtl, UVec3 vertices);
CORE_API FaceHdl CDECL polygon_add_triangle_material(LodHdl lvlDtl, UVec3 vertices, MatIdx idx);
CORE_API FaceHdl CDECL polygon_add_quad(LodHdl lvlDtl, UVec4 vertices);
CORE_API FaceHdl CDECL polygon_add_quad_material(LodHdl lvlDtl, UVec4 vertices, MatIdx idx);
CORE_API VertexHdl CDECL polygon_add_vertex_bulk(LodHdl lvlDtl, size_t count, const BulkLoader* points,
                                                 const BulkLoader* normals, const BulkLoader* uvs,
                                                 const AABB* aabb, size_t* pointsRead, size_t* normalsRead,
                                                 size_t* uvsRead);
CORE_API Boolean CDECL polygon_set_material_idx(LodHdl lvlDtl, FaceHdl face, MatIdx idx);
CORE_API size_t CDECL polygon_set_material_idx_bulk(LodHdl lvlDtl, FaceHdl startFace, size_t count, const BulkLoader* stream);
CORE_API size_t CDECL polygon_get_vertex_count(LodHdl lvlDtl);
CORE_API size_t CDECL polygon_get_face_count(LodHdl lvlDtl);
CORE_API size_t CDECL polygon_get_triangle_count(LodHdl lvlDtl);
CORE_API size_t CDECL polygon_get_quad_count(LodHdl lvlDtl);
CORE_API Boolean CDECL polygon_get_bounding_box(LodHdl lvlDtl, Vec3* min, Vec3* max);
/* EXTENSION: add `count` triangles / quads at once (vertex indices and slot indices). */
CORE_API FaceHdl CDECL polygon_add_triangle_bulk(LodHdl lvlDtl, size_t count, const UVec3* vertices, const MatIdx* materials);
CORE_API FaceHdl CDECL polygon_add_quad_bulk(LodHdl lvlDtl, size_t count, const UVec4* vertices, const MatIdx* materials);

/* ---- spheres: core_interface.h:411-428 ---- */
CORE_API Boolean CDECL spheres_reserve(LodHdl lvlDtl, size_t count);
CORE_API SphereHdl CDECL spheres_add_sphere(LodHdl lvlDtl, Vec3 point, float radius);
CORE_API SphereHdl CDECL spheres_add_sphere_material(LodHdl lvlDtl, Vec3 point, float radius, MatIdx idx);
CORE_API SphereHdl CDECL spheres_add_sphere_bulk(LodHdl lvlDtl, size_t count, const BulkLoader* stream,
                                                 const AABB* aabb, size_t* readSpheres);
CORE_API Boolean CDECL spheres_set_material_idx(LodHdl lvlDtl, SphereHdl sphere, MatIdx idx);
CORE_API size_t CDECL spheres_set_material_idx_bulk(LodHdl lvlDtl, SphereHdl startSphere, size_t count, const BulkLoader* stream);
CORE_API size_t CDECL spheres_get_sphere_count(LodHdl lvlDtl);
CORE_API Boolean CDECL spheres_get_bounding_box(LodHdl lvlDtl, Vec3* min, Vec3* max);

/* ---- objects and instances: core_interface.h:431-448 ---- */
CORE_API ObjectHdl CDECL world_create_object(MufflonInstanceHdl instHdl, const char* name, ObjectFlags flags);
CORE_API ObjectHdl CDECL world_get_object(MufflonInstanceHdl instHdl, const char* name);
CORE_API const char* CDECL world_get_object_name(ObjectHdl obj);
CORE_API Boolean CDECL object_has_lod(ConstObjectHdl obj, LodLevel level);
CORE_API Boolean CDECL object_allocate_lod_slots(ObjectHdl obj, LodLevel slots);
CORE_API LodHdl CDECL object_add_lod(ObjectHdl obj, LodLevel level, Boolean asReduced);
CORE_API Boolean CDECL object_get_id(ObjectHdl obj, uint32_t* id);
CORE_API void CDECL world_reserve_objects_instances(MufflonInstanceHdl instHdl, const uint32_t objects, const uint32_t instances);
CORE_API InstanceHdl CDECL world_create_instance(MufflonInstanceHdl instHdl, ObjectHdl obj, const uint32_t animationFrame);
CORE_API uint32_t CDECL world_get_instance_count(MufflonInstanceHdl instHdl, const uint32_t frame);
CORE_API Boolean CDECL instance_set_transformation_matrix(MufflonInstanceHdl instHdl, InstanceHdl inst, const Mat3x4* mat, const Boolean isWorldToInst);
CORE_API Boolean CDECL instance_get_transformation_matrix(MufflonInstanceHdl instHdl, InstanceHdl inst, Mat3x4* mat);
/* core_interface.h:450: the world holds one animation frame (frame 0), so this is 1 */
CORE_API Boolean CDECL world_get_frame_count(MufflonInstanceHdl instHdl, uint32_t* frameCount);

/* ---- materials and textures: core_interface.h:462-475 ---- */
CORE_API MaterialHdl CDECL world_add_material(MufflonInstanceHdl instHdl, const char* name, const MaterialParams* mat);
CORE_API IndexType CDECL world_get_material_count(MufflonInstanceHdl instHdl);
CORE_API TextureHdl CDECL world_add_texture_value(MufflonInstanceHdl instHdl, const float* value, int num, TextureSampling sampling);
/* core_interface.h:469-477. world_add_texture reads a texture file: the core
 * reads PFM ("PF" RGB, "Pf" one channel) itself, any other format fails (the
 * reference's texture plugins). The callback, if given, rewrites each texel
 * once. Textures are sampled with the nearest texel and have no mipmaps. */
CORE_API TextureHdl CDECL world_get_texture(MufflonInstanceHdl instHdl, const char* path);
CORE_API TextureHdl CDECL world_add_texture(MufflonInstanceHdl instHdl, const char* path, TextureSampling sampling, MipmapType type,
                                            TextureCallback callback, void* userParams);
CORE_API const char* CDECL world_get_texture_name(TextureHdl hdl);
CORE_API Boolean CDECL world_get_texture_size(TextureHdl hdl, IVec2* size);
/* EXTENSION: an RGBA float texture from memory (width * height * 4 floats, row 0 first). */
CORE_API TextureHdl CDECL world_add_texture_rgba32f(MufflonInstanceHdl instHdl, const char* name, uint32_t width, uint32_t height, const float* texels, TextureSampling sampling);

/* ---- cameras: core_interface.h:481-519 ---- */
CORE_API CameraHdl CDECL world_add_pinhole_camera(MufflonInstanceHdl instHdl, const char* name, const Vec3* position, const Vec3* dir,
                                                  const Vec3* up, const uint32_t pathCount, float near, float far, float vFov);
CORE_API CameraHdl CDECL world_get_camera(MufflonInstanceHdl instHdl, const char* name);
CORE_API Boolean CDECL world_set_camera_position(CameraHdl cam, Vec3 pos, const uint32_t pathIndex);
CORE_API Boolean CDECL world_set_camera_direction(CameraHdl cam, Vec3 dir, Vec3 up, const uint32_t pathIndex);
CORE_API Boolean CDECL world_set_pinhole_camera_fov(CameraHdl cam, float vFov);
CORE_API Boolean CDECL world_set_camera_near(CameraHdl cam, float near);
CORE_API Boolean CDECL world_set_camera_far(CameraHdl cam, float far);

/* ---- scenarios: core_interface.h:522-566 ---- */
CORE_API void CDECL world_reserve_scenarios(MufflonInstanceHdl instHdl, const uint32_t scenarios);
CORE_API ScenarioHdl CDECL world_create_scenario(MufflonInstanceHdl instHdl, const char* name);
CORE_API ScenarioHdl CDECL world_find_scenario(MufflonInstanceHdl instHdl, const char* name);
CORE_API ConstScenarioHdl CDECL world_get_current_scenario(MufflonInstanceHdl instHdl);
CORE_API Boolean CDECL world_finalize_scenario(MufflonInstanceHdl instHdl, ScenarioHdl scenario, const char** msg);
CORE_API SceneHdl CDECL world_load_scenario(MufflonInstanceHdl instHdl, ScenarioHdl scenario);
CORE_API const char* CDECL scenario_get_name(ScenarioHdl scenario);
CORE_API Boolean CDECL scenario_get_resolution(ScenarioHdl scenario, uint32_t* width, uint32_t* height);
CORE_API Boolean CDECL scenario_set_resolution(ScenarioHdl scenario, uint32_t width, uint32_t height);
CORE_API CameraHdl CDECL scenario_get_camera(ScenarioHdl scenario);
CORE_API Boolean CDECL scenario_set_camera(MufflonInstanceHdl instHdl, ScenarioHdl scenario, CameraHdl cam);
CORE_API Boolean CDECL scenario_mask_instance(ScenarioHdl scenario, InstanceHdl inst);
CORE_API Boolean CDECL scenario_mask_object(ScenarioHdl scenario, ObjectHdl obj);
CORE_API Boolean CDECL scenario_is_object_masked(ScenarioHdl scenario, ObjectHdl obj);
/* Level of detail of an instance: its own level if set, else its object's,
 * else the scenario's global level, clamped to the object's LoD slots
 * (scenario.cpp:131-154). */
CORE_API LodLevel CDECL scenario_get_global_lod_level(ScenarioHdl scenario);
CORE_API Boolean CDECL scenario_set_global_lod_level(ScenarioHdl scenario, LodLevel level);
CORE_API LodLevel CDECL scenario_get_object_lod(ScenarioHdl scenario, ObjectHdl obj);
CORE_API Boolean CDECL scenario_set_object_lod(ScenarioHdl scenario, ObjectHdl obj, LodLevel level);
CORE_API Boolean CDECL scenario_set_instance_lod(ScenarioHdl scenario, InstanceHdl inst, LodLevel level);
CORE_API void CDECL scenario_reserve_material_slots(ScenarioHdl scenario, size_t count);
CORE_API void CDECL scenario_reserve_custom_object_properties(ScenarioHdl scenario, size_t objects);
CORE_API void CDECL scenario_reserve_custom_instance_properties(ScenarioHdl scenario, size_t instances);
CORE_API Boolean CDECL scenario_add_light(MufflonInstanceHdl instHdl, ScenarioHdl scenario, LightHdl hdl);
CORE_API MatIdx CDECL scenario_declare_material_slot(ScenarioHdl scenario, const char* name, size_t nameLength);
CORE_API MatIdx CDECL scenario_get_material_slot(ScenarioHdl scenario, const char* name, size_t nameLength);
CORE_API Boolean CDECL scenario_assign_material(ScenarioHdl scenario, MatIdx index, MaterialHdl handle);
CORE_API SceneHdl CDECL world_get_current_scene(MufflonInstanceHdl instHdl);
CORE_API Boolean CDECL scene_get_bounding_box(SceneHdl scene, Vec3* min, Vec3* max);

/* ---- lights: core_interface.h:577-622 ---- */
CORE_API LightHdl CDECL world_add_light(MufflonInstanceHdl instHdl, const char* name, LightType type, const uint32_t count);
CORE_API LightHdl CDECL world_add_background_light(MufflonInstanceHdl instHdl, const char* name, BackgroundType type);
CORE_API Boolean CDECL world_set_point_light_position(MufflonInstanceHdl instHdl, LightHdl hdl, Vec3 pos, const uint32_t frame);
CORE_API Boolean CDECL world_set_point_light_intensity(MufflonInstanceHdl instHdl, LightHdl hdl, Vec3 intensity, const uint32_t frame);
CORE_API Boolean CDECL world_set_env_light_color(MufflonInstanceHdl instHdl, LightHdl hdl, Vec3 color);
CORE_API Boolean CDECL world_set_env_light_scale(MufflonInstanceHdl instHdl, LightHdl hdl, Vec3 color);

/* ---- renderers: core_interface.h:625-657 ---- */
CORE_API uint32_t CDECL render_get_renderer_count(MufflonInstanceHdl instHdl);
CORE_API uint32_t CDECL render_get_renderer_variations(MufflonInstanceHdl instHdl, uint32_t index);
CORE_API const char* CDECL render_get_renderer_name(MufflonInstanceHdl instHdl, uint32_t index);
CORE_API const char* CDECL render_get_renderer_short_name(MufflonInstanceHdl instHdl, uint32_t index);
CORE_API RenderDevice CDECL render_get_renderer_devices(MufflonInstanceHdl instHdl, uint32_t index, uint32_t variation);
CORE_API Boolean CDECL render_enable_renderer(MufflonInstanceHdl instHdl, uint32_t index, uint32_t variation);
CORE_API Boolean CDECL render_iterate(MufflonInstanceHdl instHdl, ProcessTime* time, ProcessTime* preTime, ProcessTime* postTime);
CORE_API uint32_t CDECL render_get_current_iteration(ConstMufflonInstanceHdl instHdl);
CORE_API Boolean CDECL render_reset(MufflonInstanceHdl instHdl);
CORE_API Boolean CDECL render_save_screenshot(MufflonInstanceHdl instHdl, const char* filename, const char* targetName, Boolean variance);
CORE_API uint32_t CDECL render_get_render_target_count(MufflonInstanceHdl instHdl);
CORE_API const char* CDECL render_get_render_target_name(MufflonInstanceHdl instHdl, uint32_t index);
CORE_API Boolean CDECL render_enable_render_target(MufflonInstanceHdl instHdl, const char* target, Boolean variance);
CORE_API Boolean CDECL render_disable_render_target(MufflonInstanceHdl instHdl, const char* target, Boolean variance);
CORE_API Boolean CDECL render_is_render_target_enabled(MufflonInstanceHdl instHdl, const char* name, Boolean variance);
CORE_API uint32_t CDECL renderer_get_num_parameters(MufflonInstanceHdl instHdl);
CORE_API const char* CDECL renderer_get_parameter_desc(MufflonInstanceHdl instHdl, uint32_t idx, ParameterType* type);
CORE_API Boolean CDECL renderer_set_parameter_int(MufflonInstanceHdl instHdl, const char* name, int32_t value);
CORE_API Boolean CDECL renderer_get_parameter_int(MufflonInstanceHdl instHdl, const char* name, int32_t* value);
CORE_API Boolean CDECL renderer_set_parameter_float(MufflonInstanceHdl instHdl, const char* name, float value);
CORE_API Boolean CDECL renderer_get_parameter_float(MufflonInstanceHdl instHdl, const char* name, float* value);
CORE_API Boolean CDECL renderer_set_parameter_bool(MufflonInstanceHdl instHdl, const char* name, Boolean value);
CORE_API Boolean CDECL renderer_get_parameter_bool(MufflonInstanceHdl instHdl, const char* name, Boolean* value);
CORE_API Boolean CDECL renderer_set_parameter_enum(MufflonInstanceHdl instHdl, const char* name, int value);
CORE_API Boolean CDECL renderer_get_parameter_enum(MufflonInstanceHdl instHdl, const char* name, int* value);

/* ---- EXTENSIONS: measurement and parity hooks ---- */

/* Counters of the last render_iterate: rays (extension + shadow), shadow rays,
 * BVH node-pair fetches, primitive tests, instance entries, and the device time
 * of the path-tracing kernel in milliseconds. */
typedef struct {
	uint64_t rays, shadowRays, nodeVisits, primTests, instanceVisits;
	uint32_t errors;
	float kernelMs;
} MufflonRenderStats;
CORE_API Boolean CDECL mufflon_get_render_stats(MufflonInstanceHdl instHdl, MufflonRenderStats* stats);

/* Per-stage view of the last render_iterate. With the wavefront schedule the
 * traversal counters are split into extension rays (closest hit) and shadow
 * rays (any hit); with the megakernel all of them are in the extension
 * fields. The stage times are filled only while the integer renderer
 * parameter "Stage timing" is non-zero (events around every stage launch):
 * camera rays, the trace launches of the wavefront bounces (extension and
 * shadow rays), the launch that finishes the remaining paths, the shade
 * launches, the accumulation, and the binning of queued rays by coherence
 * (renderer parameter "Ray sort bits"). With the wavefront schedule the
 * node-visit, primitive-test and instance-entry counts (here and in
 * MufflonRenderStats) are kept only while the integer renderer parameter
 * "Traversal statistics" is non-zero, by counting variants of its kernels;
 * ray counts are always kept. */
typedef struct {
	uint64_t extensionRays, extendNodeVisits, extendPrimTests, extendInstanceVisits;
	uint64_t shadowRays, shadowNodeVisits, shadowPrimTests, shadowInstanceVisits;
	float cameraMs, extendMs, tailMs, shadeMs, finalizeMs;
	uint32_t launches;  /* kernel launches of the iteration */
	uint32_t wavefront; /* 1: wavefront stages, 0: megakernel */
	float binMs;
} MufflonStageStats;
CORE_API Boolean CDECL mufflon_get_stage_stats(MufflonInstanceHdl instHdl, MufflonStageStats* stats);

/* EXTENSION with no counterpart in the reference: the contributions of the
 * last iteration of the light tracer or the bidirectional path tracer, kept
 * while the renderer's integer parameter "Record connections" is non-zero.
 * pixels[k] receives the pixel index a contribution was added to, or -1.
 * Light tracer: slots = width * height * M (M = "Max. path length"; photon
 * major, then the photon's path length at the camera connection) and
 * values[5k..5k+4] = radiance rgb, lightness, density. Bidirectional path
 * tracer: slots = width * height * (M * M + M) (pixel major; first the
 * connections [view path length][light vertex], then the emitter hits [view
 * path length - 1]) and values[4k..4k+3] = radiance rgb, lightness. */
CORE_API Boolean CDECL mufflon_get_lt_records(MufflonInstanceHdl instHdl, int32_t* pixels, float* values,
                                              uint64_t slots);

/* EXTENSION with no counterpart in the reference: renders many jobs at once.
 * A job is the loaded scenario of a library instance (so jobs may use
 * different scenes), rendered at its own resolution (0 = the scenario's),
 * sample count and path-tracer parameters. All jobs' paths go through the
 * same wavefront queues, one iteration (sample) of every unfinished job per
 * launch sequence; with useGraph the whole batch is captured as one CUDA
 * graph and launched once. radiance[j] (width*height*3 floats) and hitId[j]
 * (width*height*2) receive job j's cumulative means; either array or entry may
 * be NULL. jobDoneMs[j] (may be NULL) receives the device time from the start
 * of the batch until job j's last sample was accumulated. All jobs must use
 * the same NEE count; the instances must be on one device. Each job's result
 * is identical to rendering it alone with render_iterate. */
typedef struct {
	MufflonInstanceHdl instance;
	uint32_t width, height;
	uint32_t spp;
	int32_t seed;
	int32_t minPathLength, maxPathLength, rrStartDepth, neeCount;
} MufflonBatchJob;
typedef struct {
	float deviceMs;     /* device time of the whole batch */
	uint32_t launches;  /* kernel launches (captured as graph nodes when useGraph) */
	uint32_t usedGraph;
	uint32_t pixels;    /* pixels of all jobs */
} MufflonBatchStats;
CORE_API Boolean CDECL mufflon_render_batch(const MufflonBatchJob* jobs, uint32_t count, int32_t useGraph,
                                            float* const* radiance, float* const* hitId, float* jobDoneMs,
                                            MufflonBatchStats* stats);

/* EXTENSIONS for differentiable rendering, with no counterpart in the
 * reference.
 * mufflon_texture_update replaces the texels (width*height*4 floats, RGBA)
 * of a texture created by the world API, also on the GPU if the loaded scene
 * uses it, without reloading the scene; the accumulation is reset.
 * mufflon_albedo_gradient computes the gradient of a loss with respect to an
 * albedo texture by path replay: given imageGrad = dLoss/dImage (W*H*3 floats
 * for the scenario's resolution, image = mean of spp samples as rendered by
 * spp render_iterate calls after a reset), it writes dLoss/dTexel to
 * textureGrad (width*height*3 floats, RGB) for the Lambert materials that
 * use the texture as albedo (nearest-texel lookup). It uses the renderer's
 * parameters and requires Russian roulette off (RR start depth >= Max. path
 * length, at most 32). deviceMs (may be NULL) receives the kernels' time. */
CORE_API Boolean CDECL mufflon_texture_update(MufflonInstanceHdl instHdl, TextureHdl texture, const float* rgba);
CORE_API Boolean CDECL mufflon_albedo_gradient(MufflonInstanceHdl instHdl, TextureHdl texture, uint32_t spp,
                                               const float* imageGrad, float* textureGrad, float* deviceMs);
/* mufflon_emission_gradient: the same path replay for the emitted radiance
 * L = radiance x scale of an emissive material (EmissiveParams,
 * core_interface.h:263-266; the CUDA renderer takes a constant radiance, a
 * 1x1 value texture, so L is that texel times the scale): radianceGrad
 * receives dLoss/dL (3 floats, RGB), summed over every material slot of the
 * scenario that uses the material. Each term the material emits (hits of its
 * surfaces and next-event samples of its area lights) is linear in L, and the
 * sampling probabilities and MIS weights are held fixed; Russian roulette may
 * be on. Channels with L = 0 get 0. mufflon_set_emitted_radiance replaces L
 * (3 floats) of an emissive material; the scene, whose light fluxes depend
 * on it, is rebuilt before the next render, and the accumulation is reset. */
CORE_API Boolean CDECL mufflon_emission_gradient(MufflonInstanceHdl instHdl, MaterialHdl material, uint32_t spp,
                                                 const float* imageGrad, float* radianceGrad, float* deviceMs);
CORE_API Boolean CDECL mufflon_set_emitted_radiance(MufflonInstanceHdl instHdl, MaterialHdl material, const float* rgb);

/* Host-side times (ms) of the last scene load (world_load_scenario or the
 * implicit load of the first render_iterate): the whole load, the geometry
 * upload, the object BVH builds (LBVH + 8-wide conversion), the instance BVH,
 * and lights / materials / textures; plus the geometry bytes copied to the GPU. */
typedef struct {
	float totalMs, uploadMs, bvhMs, instanceBvhMs, otherMs;
	uint32_t pad;
	uint64_t h2dBytes;
} MufflonLoadStats;
CORE_API Boolean CDECL mufflon_get_load_stats(MufflonInstanceHdl instHdl, MufflonLoadStats* stats);
/* EXTENSION: the loaded scene's light list (112 bytes per light: u16 type,
 * u16 material, position[3], intensity[3], quad vectors[4][3], uv vectors[4][2],
 * sphere radius)
 * and light tree (20 bytes per node: left/right flux, left/right index,
 * left/right type), as built on the GPU, plus the sorted
 * (instance << 32 | primitive) -> node-path code map of the area lights.
 * Counts are always written; arrays may be NULL. */
CORE_API Boolean CDECL mufflon_get_light_tree(MufflonInstanceHdl instHdl, uint32_t* numLights, uint32_t* numNodes,
                                              uint32_t* numAreaLights, void* lights, void* nodes, uint64_t* primKeys,
                                              uint32_t* primCodes, float* rootFlux);

/* Closest hits of n rays (6 floats: origin, direction) against the loaded
 * scene, with the path tracer's epsilon offset along geoNormals (may be NULL). */
CORE_API Boolean CDECL mufflon_trace_rays(MufflonInstanceHdl instHdl, const float* rays, const float* geoNormals,
                                          float tmax, uint32_t n, float* t, int32_t* instanceIds,
                                          int32_t* primIds, float* surfaceParams);
/* Shadow-ray test between point pairs (3 floats each). */
CORE_API Boolean CDECL mufflon_trace_occlusion(MufflonInstanceHdl instHdl, const float* a, const float* b,
                                               uint32_t n, uint8_t* occluded);
/* BVH of the loaded scene: which = -1 for the instance BVH, else the LoD
 * index in load order. Pass NULL buffers to query the sizes first. nodes
 * receives the reference's 32-byte BvhNode pairs (2 * numInternal). */
CORE_API Boolean CDECL mufflon_get_bvh(MufflonInstanceHdl instHdl, int32_t which, int32_t* numPrims,
                                       int32_t* numInternal, void* nodes, int32_t* primIds);

/* Standalone LBVH build of one LoD from host arrays (no instance needed).
 * Outputs: sorted Morton codes (numPrims), Karras parents (2*numPrims-1),
 * nodes (2*(numPrims-1) capacity), primIds (numPrims), the internal-node
 * count after collapse, and per-stage device times in ms (9 floats: morton,
 * sort, emit, merge, mark, scan, compact, soup, and the conversion into the
 * compressed 8-wide traversal hierarchy; may be NULL). */
CORE_API Boolean CDECL mufflon_lbvh_build(const float* vertices, uint32_t numVertices, const uint32_t* indices,
                                          uint32_t numTriangles, uint32_t numQuads, const float* spheres,
                                          uint32_t numSpheres, uint64_t* mortonSorted, int32_t* parents,
                                          void* nodes, int32_t* primIds, int32_t* numInternal, float* stageMs);
/* The same build with the Morton code width chosen: 63 bits (what
 * mufflon_lbvh_build and every scene load use, the reference's choice for LoD
 * and instance hierarchies, build_lbvh.cu:35-48) or the reference's unused
 * 30-bit code (build_lbvh.cu:59-69: 10 bits per axis). mortonSorted then holds
 * the 30-bit codes, zero-extended. */
CORE_API Boolean CDECL mufflon_lbvh_build_ex(const float* vertices, uint32_t numVertices, const uint32_t* indices,
                                             uint32_t numTriangles, uint32_t numQuads, const float* spheres,
                                             uint32_t numSpheres, int32_t mortonBits, uint64_t* mortonSorted,
                                             int32_t* parents, void* nodes, int32_t* primIds, int32_t* numInternal,
                                             float* stageMs);
/* Same build on device-resident inputs; outputs stay on the device. Times
 * the whole build with CUDA events (ms), 8-wide conversion included. Returns
 * the node count after collapse; stageMs as above (9 floats). */
CORE_API Boolean CDECL mufflon_lbvh_build_device(const float* dVertices, const uint32_t* dIndices, uint32_t numTriangles,
                                                 uint32_t numQuads, const float* dSpheres, uint32_t numSpheres,
                                                 const float* aabb6, int32_t* numInternal, float* buildMs,
                                                 float* stageMs);
/* Measured read bandwidth (GB/s) of an L2-resident buffer of `bytes`, read
 * `repetitions` times; the denominator of the traversal roofline. */
CORE_API Boolean CDECL mufflon_measure_l2_bandwidth(uint64_t bytes, int32_t repetitions, float* gbs);
/* Stable radix sort of (uint64 key, int32 value) pairs in host memory. */
CORE_API Boolean CDECL mufflon_sort_pairs(uint64_t* keys, int32_t* values, uint32_t n);

/* EXTENSION with no counterpart in the reference: the same stable sort of n
 * device-resident pairs, in place, without allocating any device memory.
 * For callers that cannot call cudaMalloc: an engine that has reserved all
 * device memory for its own allocator, or a frame loop that must not stall in
 * cudaMalloc/cudaFree (they may synchronise the device). The scratch space is
 * a fixed array of about 12.5 MiB inside the library, held by every GPU that
 * loads the library until the process exits; n above
 * MUFFLON_SORT_NOALLOC_MAX_PAIRS is rejected with an error. Set-up:
 * mufflon_initialize looks up the array's address on the device it selects
 * and loads the sort's kernels there; on any other device the first call does
 * it. That set-up loads the library's device code, which takes device memory
 * under CUDA's lazy module loading, so it must come before the caller
 * reserves its device memory and before any stream capture. Later calls take
 * no device memory. All calls share the array, so calls that overlap on the
 * GPU race. keys/values are device pointers owned by the caller; stream is a
 * cudaStream_t (NULL: default stream); the call returns after the pairs are
 * sorted. */
#define MUFFLON_SORT_NOALLOC_MAX_PAIRS (1u << 20)
CORE_API Boolean CDECL mufflon_sort_pairs_device_noalloc(uint64_t* keys, int32_t* values, uint32_t n, void* stream);

#ifdef __cplusplus
}
#endif

#endif
