// C API of the B200 path-tracer core: the subset of
// src/core/export/interface.cpp that builds a world, runs the "Pathtracer"
// renderer and reads its targets back. Every function catches all
// exceptions, logs, stores the message for core_get_dll_error() and returns
// false / nullptr / INVALID_INDEX, as interface.cpp:53-83 does.
#include "../../../include/mufflon_core.h"
#include "world.hpp"
#include "../trace/pt_api.hpp"
#include "../lbvh/sort_noalloc.hpp"
#include "../common/pfm.hpp"

#include <algorithm>
#include <cstdio>
#include <chrono>
#include <cstdarg>
#include <cstring>
#include <exception>
#include <fstream>
#include <iterator>
#include <stdexcept>
#include <string>
#include <vector>

using namespace mb;

namespace {

thread_local std::string s_lastError;
void (*s_logger)(const char*, int) = nullptr;
int s_logLevel = LOG_INFO;

void log_msg(int level, const std::string& msg) {
	if(level < s_logLevel) return;
	if(s_logger) s_logger(msg.c_str(), level);
}

struct ApiError : std::runtime_error { using std::runtime_error::runtime_error; };

#define TRY try {
#define CATCH_ALL(ret) } catch(const std::exception& ex) { s_lastError = std::string(__func__) + ": " + ex.what(); log_msg(LOG_ERROR, s_lastError); return ret; } \
	catch(...) { s_lastError = std::string(__func__) + ": unknown error"; log_msg(LOG_ERROR, s_lastError); return ret; }
#define CHECK(cond, msg) do { if(!(cond)) throw ApiError(msg); } while(0)
#define CHECK_CUDA(expr) do { cudaError_t e_ = (expr); if(e_ != cudaSuccess) throw ApiError(std::string("CUDA: ") + cudaGetErrorString(e_) + " (" #expr ", line " + std::to_string(__LINE__) + ")"); } while(0)

MufflonInstance& minst(void* h) {
	if(!h) throw ApiError("invalid mufflon instance");
	return *static_cast<MufflonInstance*>(h);
}
HostLod& mlod(void* h) {
	if(!h) throw ApiError("invalid LoD handle");
	return *static_cast<HostLod*>(h);
}

// Parameters of the path tracer (pt_params.hpp:8-14, parameter.hpp:327-365)
// plus two extensions.
struct ParamDesc { const char* name; ParameterType type; };
const ParamDesc PT_PARAMS[] = {
	{ "Seed", PARAM_INT }, { "Min. path length", PARAM_INT }, { "Max. path length", PARAM_INT },
	{ "NEE count", PARAM_INT }, { "NEE position guide", PARAM_BOOL },
	{ "RR start depth", PARAM_INT }, { "Blocks per SM", PARAM_INT }, { "Megakernel", PARAM_INT },
	{ "Stage timing", PARAM_INT }, { "Traversal statistics", PARAM_INT }, { "Trace blocks per SM", PARAM_INT }, { "Wavefront bounces", PARAM_INT },
	{ "Trace refill lanes", PARAM_INT }, { "Tail paths", PARAM_INT }, { "Iteration graph", PARAM_INT },
	{ "Planned tail", PARAM_INT }, { "Ray sort bits", PARAM_INT }, { "Ray sort direction bits", PARAM_INT },
	{ "Traversal step limit", PARAM_INT },
};
// lt_params.hpp:8-12, plus the recording switch of the parity tests
const ParamDesc LT_PARAMS[] = {
	{ "Seed", PARAM_INT }, { "Min. path length", PARAM_INT }, { "Max. path length", PARAM_INT },
	{ "Record connections", PARAM_INT }, { "Traversal step limit", PARAM_INT }, { "Megakernel", PARAM_INT },
};
// vcm_params.hpp:8-14, plus the recording switch of the parity tests
const ParamDesc VCM_PARAMS[] = {
	{ "Seed", PARAM_INT }, { "Min. path length", PARAM_INT }, { "Max. path length", PARAM_INT },
	{ "Relative merge radius", PARAM_FLOAT }, { "Progressive", PARAM_BOOL }, { "Record connections", PARAM_INT },
	{ "Traversal step limit", PARAM_INT },
};
// wireframe_params.hpp:6-26
const ParamDesc WIRE_PARAMS[] = { { "Line width", PARAM_FLOAT }, { "Maximum trace depth", PARAM_INT },
                                  { "Traversal step limit", PARAM_INT } };
// Render targets of the path tracer (pt_params.hpp:16-26). The CUDA path
// implements all eight (the six auxiliary ones: aux_targets.cuh).
const char* TARGETS[] = { "Radiance", "Position", "Depth", "Normal", "UV", "Albedo", "Lightness", "Hit ID" };
// Render targets of the light tracer (lt_params.hpp:14-17) and of the
// bidirectional path tracer (bpt_params.hpp:14-17, its first two), all implemented.
const char* LT_TARGETS[] = { "Radiance", "Lightness", "Density" };

int32_t* param_ptr(RendererState& r, const char* name) {
	// every renderer: the traversal steps a ray may take before it is
	// abandoned, which fails the iteration (0: the default limit)
	if(!std::strcmp(name, "Traversal step limit")) return &r.stepLimit;
	if(r.kind == 2) {
		if(!std::strcmp(name, "Maximum trace depth")) return &r.wireParams.maxTraceDepth;
		return nullptr;
	}
	if(r.kind == 1 || r.kind == 3 || r.kind == 4) {
		LtParams& p = r.kind == 1 ? r.ltParams : r.kind == 3 ? r.bptParams : r.vcmParams;
		if(!std::strcmp(name, "Seed")) return &p.seed;
		if(!std::strcmp(name, "Min. path length")) return &p.minPathLength;
		if(!std::strcmp(name, "Max. path length")) return &p.maxPathLength;
		if(!std::strcmp(name, "Record connections")) return r.kind == 1 ? &r.ltRecord : r.kind == 3 ? &r.bptRecord : &r.vcmRecord;
		if(r.kind != 4 && !std::strcmp(name, "Megakernel")) return r.kind == 1 ? &r.ltMegakernel : &r.bptMegakernel;
		return nullptr;
	}
	if(!std::strcmp(name, "Seed")) return &r.params.seed;
	if(!std::strcmp(name, "Min. path length")) return &r.params.minPathLength;
	if(!std::strcmp(name, "Max. path length")) return &r.params.maxPathLength;
	if(!std::strcmp(name, "NEE count")) return &r.params.neeCount;
	if(!std::strcmp(name, "RR start depth")) return &r.params.rrStartDepth;
	if(!std::strcmp(name, "Blocks per SM")) return &r.blocksPerSm;
	if(!std::strcmp(name, "Megakernel")) return &r.megakernel;
	if(!std::strcmp(name, "Stage timing")) return &r.stageTiming;
	if(!std::strcmp(name, "Traversal statistics")) return &r.traversalStats;
	if(!std::strcmp(name, "Trace blocks per SM")) return &r.traceBlocksPerSm;
	if(!std::strcmp(name, "Wavefront bounces")) return &r.wavefrontBounces;
	if(!std::strcmp(name, "Trace refill lanes")) return &r.refillLanes;
	if(!std::strcmp(name, "Tail paths")) return &r.tailPaths;
	if(!std::strcmp(name, "Iteration graph")) return &r.iterationGraph;
	if(!std::strcmp(name, "Planned tail")) return &r.planTail;
	if(!std::strcmp(name, "Ray sort bits")) return &r.sortBits;
	if(!std::strcmp(name, "Ray sort direction bits")) return &r.sortDirBits;
	return nullptr;
}

size_t read_bulk(const BulkLoader* b, void* dst, size_t bytes) {
	if(!b) return 0;
	if(b->type == BULK_ARRAY) { std::memcpy(dst, b->descriptor.bytes, bytes); return bytes; }
	return std::fread(dst, 1, bytes, b->descriptor.file);
}

int32_t step_limit(const RendererState& r) { return r.stepLimit > 0 ? r.stepLimit : MAX_TRAVERSAL_STEPS; }

// The reference's error convention (interface.cpp:53-83) for rays whose
// traversal was abandoned: the call fails with a message rather than
// returning an image with silently wrong pixels.
void check_traversal(unsigned errors, int32_t limit) {
	if(errors)
		throw ApiError("traversal abandoned " + std::to_string(errors) + " rays (step limit of " + std::to_string(limit) +
		               " exceeded or traversal stack overflow); the result of this call is incomplete");
}

void ensure_render_buffers(MufflonInstance& I) {
	RendererState& r = I.renderer;
	HostScenario* sc = I.current;
	CHECK(sc != nullptr, "no scenario loaded");
	if(r.width == sc->width && r.height == sc->height && r.rng) return;
	r.release();
	r.width = sc->width; r.height = sc->height;
	const size_t n = size_t(r.width) * r.height;
	CHECK_CUDA(cudaMalloc(&r.rng, n * sizeof(uint64_t)));
	CHECK_CUDA(cudaMalloc(&r.radiance, n * 3 * sizeof(float)));
	CHECK_CUDA(cudaMalloc(&r.hitId, n * 2 * sizeof(float)));
	CHECK_CUDA(cudaMalloc(&r.workCounter, sizeof(unsigned int)));
	CHECK_CUDA(cudaMalloc(&r.counters, 2 * sizeof(TraceCounters)));
	CHECK_CUDA(cudaEventCreate(&r.evStart));
	CHECK_CUDA(cudaEventCreate(&r.evStop));
	r.needsReset = true;
}

// Variance buffers of the targets whose variance is recorded (grow-only until
// the resolution changes; cleared at every reset).
void ensure_variance_buffers(MufflonInstance& I) {
	RendererState& r = I.renderer;
	const size_t n = size_t(r.width) * r.height;
	auto need = [&](float*& buf, bool on, size_t channels) {
		if(on && !buf) {
			CHECK_CUDA(cudaMalloc(&buf, n * channels * sizeof(float)));
			CHECK_CUDA(cudaMemsetAsync(buf, 0, n * channels * sizeof(float), I.stream));
		}
	};
	need(r.radianceVar, r.varRadiance || r.varBorder, 3);
	need(r.hitIdVar, r.varHitId, 2);
	need(r.lightnessVar, r.varLightness, 1);
	need(r.densityMean, r.varDensity, 1);
}

// The path tracer's auxiliary-target buffers (cumulative, variance and, for
// the wavefront schedule, the per-path iteration state) of the enabled
// targets; "Lightness" uses the light tracer's buffers. Cleared at every reset.
constexpr int AUX_CH[5] = { 3, 1, 3, 2, 3 };
bool aux_wanted(const RendererState& r) {
	bool any = r.targetLightness;
	for(int a = 0; a < 5; ++a) any = any || r.auxTarget[a];
	return any;
}
void ensure_aux_buffers(MufflonInstance& I) {
	RendererState& r = I.renderer;
	const size_t n = size_t(r.width) * r.height;
	for(int a = 0; a < 5; ++a) {
		if(r.auxTarget[a] && !r.auxCum[a]) {
			CHECK_CUDA(cudaMalloc(&r.auxCum[a], n * AUX_CH[a] * sizeof(float)));
			CHECK_CUDA(cudaMemsetAsync(r.auxCum[a], 0, n * AUX_CH[a] * sizeof(float), I.stream));
		}
		if(r.auxTarget[a] && r.auxVarOn[a] && !r.auxVarBuf[a]) {
			CHECK_CUDA(cudaMalloc(&r.auxVarBuf[a], n * AUX_CH[a] * sizeof(float)));
			CHECK_CUDA(cudaMemsetAsync(r.auxVarBuf[a], 0, n * AUX_CH[a] * sizeof(float), I.stream));
		}
	}
	if(r.targetLightness && !r.lightness) {
		CHECK_CUDA(cudaMalloc(&r.lightness, n * sizeof(float)));
		CHECK_CUDA(cudaMemsetAsync(r.lightness, 0, n * sizeof(float), I.stream));
	}
	if(aux_wanted(r) && r.auxMemPixels != n) {
		cudaFree(r.auxMem);
		r.auxMem = nullptr; r.auxMemPixels = 0;
		CHECK_CUDA(cudaMalloc(&r.auxMem, n * (sizeof(float2) + AUX_CHANNELS * sizeof(float))));
		r.auxMemPixels = n;
	}
}

// Wavefront state for the current resolution and NEE count (one slab).
void ensure_wavefront_buffers(MufflonInstance& I) {
	RendererState& r = I.renderer;
	const size_t n = size_t(r.width) * r.height;
	const int nee = r.params.neeCount > 0 ? r.params.neeCount : 1;
	if(r.wfMemory && r.wfNee == nee && r.wfPixels == n) return;
	if(r.wfMemory) cudaFree(r.wfMemory);
	r.wfMemory = nullptr;
	r.wfNee = 0;
	r.wfPixels = 0;
	CHECK_CUDA(cudaMalloc(&r.wfMemory, wavefront_bytes(n, nee)));
	wavefront_carve(r.wfMemory, n, nee, r.wf);
	r.wfNee = nee;
	r.wfPixels = n;
}

// Light tracer buffers for the current resolution: the iteration buffers, the
// cumulative 1-channel targets and, when recording, the connection records.
void ensure_lt_buffers(MufflonInstance& I) {
	RendererState& r = I.renderer;
	const size_t n = size_t(r.width) * r.height;
	if(!r.ltIter) {
		CHECK_CUDA(cudaMalloc(&r.ltIter, n * sizeof(float4)));
		CHECK_CUDA(cudaMalloc(&r.ltIterDensity, n * sizeof(float)));
		CHECK_CUDA(cudaMalloc(&r.lightness, n * sizeof(float)));
		CHECK_CUDA(cudaMalloc(&r.density, n * sizeof(float)));
		CHECK_CUDA(cudaMemsetAsync(r.lightness, 0, n * sizeof(float), I.stream));
		CHECK_CUDA(cudaMemsetAsync(r.density, 0, n * sizeof(float), I.stream));
	}
	// records: light tracer M slots of 5 floats per photon; bidirectional path
	// tracer M*M + M, vertex connection and merging M*M + 2M slots of 4 floats
	// per pixel (M = max. path length)
	const size_t m = size_t(std::max(1, r.kind == 3 ? r.bptParams.maxPathLength : r.kind == 4 ? r.vcmParams.maxPathLength
	                                                                            : r.ltParams.maxPathLength));
	const bool record = r.kind == 3 ? r.bptRecord != 0 : r.kind == 4 ? r.vcmRecord != 0 : r.kind == 1 ? r.ltRecord != 0 : false;
	const size_t slots = record ? (r.kind == 3 ? n * (m * m + m) : r.kind == 4 ? n * (m * m + 2 * m) : n * m) : 0;
	const size_t floats = slots * (r.kind == 3 || r.kind == 4 ? 4 : 5);
	if(slots != r.ltRecSlots || floats != r.ltRecFloats) {
		cudaFree(r.ltRecPixel); cudaFree(r.ltRecValue);
		r.ltRecPixel = nullptr; r.ltRecValue = nullptr; r.ltRecSlots = 0; r.ltRecFloats = 0;
		if(slots) {
			CHECK_CUDA(cudaMalloc(&r.ltRecPixel, slots * sizeof(int32_t)));
			CHECK_CUDA(cudaMalloc(&r.ltRecValue, floats * sizeof(float)));
			CHECK_CUDA(cudaMemsetAsync(r.ltRecPixel, 0xFF, slots * sizeof(int32_t), I.stream));
			CHECK_CUDA(cudaMemsetAsync(r.ltRecValue, 0, floats * sizeof(float), I.stream));
			r.ltRecSlots = slots;
			r.ltRecFloats = floats;
		}
	}
	if(r.kind == 1 && !r.ltMegakernel) {
		const size_t bytes = ltw_bytes(n);
		if(bytes > r.ltWavefrontBytes) {
			cudaFree(r.ltWavefront);
			r.ltWavefront = nullptr;
			r.ltWavefrontBytes = 0;
			CHECK_CUDA(cudaMalloc(&r.ltWavefront, bytes));
			r.ltWavefrontBytes = bytes;
		}
	}
	if(r.kind == 3 && r.bptMegakernel) {
		const size_t bytes = bpt_scratch_bytes(r.bptParams.maxPathLength);
		if(bytes > r.bptScratchBytes) {
			cudaFree(r.bptScratch);
			r.bptScratch = nullptr;
			r.bptScratchBytes = 0;
			CHECK_CUDA(cudaMalloc(&r.bptScratch, bytes));
			r.bptScratchBytes = bytes;
		}
	}
	if(r.kind == 4) {
		CHECK(r.vcmParams.maxPathLength <= BPTW_MAX_PATH, "vertex connection and merging takes at most 64 path lengths");
		const size_t bytes = vcm_bytes(n, r.vcmParams.maxPathLength);
		if(bytes > r.vcmMemoryBytes) {
			cudaFree(r.vcmMemory);
			r.vcmMemory = nullptr;
			r.vcmMemoryBytes = 0;
			CHECK_CUDA(cudaMalloc(&r.vcmMemory, bytes));
			r.vcmMemoryBytes = bytes;
		}
	}
	if(r.kind == 3 && !r.bptMegakernel) {
		const size_t bytes = bptw_bytes(n, r.bptParams.maxPathLength);
		if(bytes > r.bptWavefrontBytes) {
			cudaFree(r.bptWavefront);
			r.bptWavefront = nullptr;
			r.bptWavefrontBytes = 0;
			CHECK_CUDA(cudaMalloc(&r.bptWavefront, bytes));
			r.bptWavefrontBytes = bytes;
		}
	}
}

// One light-tracing iteration (gpu_lt.cpp / lt_common.hpp): width * height
// photons, each walk's vertices connected to the camera; or one
// bidirectional path-tracing iteration (cpu_bpt.cpp), into the same buffers.
void iterate_lt(MufflonInstance& I) {
	RendererState& r = I.renderer;
	const DScene& S = I.scene.desc;
	LtTargets t{};
	t.rngState = r.rng;
	t.iter = r.ltIter;
	t.iterDensity = r.ltIterDensity;
	t.radiance = r.targetRadiance ? r.radiance : nullptr;
	t.lightness = r.targetLightness ? r.lightness : nullptr;
	t.density = r.targetDensity ? r.density : nullptr;
	t.radianceVar = r.targetRadiance && r.varRadiance ? r.radianceVar : nullptr;
	t.lightnessVar = r.targetLightness && r.varLightness ? r.lightnessVar : nullptr;
	t.densityMean = r.targetDensity && r.varDensity ? r.densityMean : nullptr;
	t.recPixel = r.ltRecSlots ? r.ltRecPixel : nullptr;
	t.recValue = r.ltRecSlots ? r.ltRecValue : nullptr;
	t.width = r.width; t.height = r.height;
	t.iteration = r.iteration;
	CHECK_CUDA(cudaMemsetAsync(r.counters, 0, 2 * sizeof(TraceCounters), I.stream));
	CHECK_CUDA(cudaEventRecord(r.evStart, I.stream));
	if(r.kind == 4) {
		t.density = nullptr;
		t.densityMean = nullptr;
		const VcmSettings v{ r.vcmMergeRadius, r.vcmProgressive };
		CHECK_CUDA(launch_vcm(S, r.vcmParams, v, t, r.counters, I.stream, r.vcmMemory));
	} else if(r.kind == 3) {
		t.density = nullptr;
		t.densityMean = nullptr;
		CHECK(r.bptMegakernel || r.bptParams.maxPathLength <= BPTW_MAX_PATH,
		      "the bidirectional path tracer's stages take at most 64 path lengths (set \"Megakernel\" to 1 for longer paths)");
		CHECK_CUDA(launch_bpt(S, r.bptParams, t, r.bptScratch, r.workCounter, r.counters, I.stream,
		                      r.bptMegakernel ? nullptr : r.bptWavefront));
	} else if(r.kind == 2) {
		t.radiance = r.radiance; // the "Border" target
		t.radianceVar = r.varBorder ? r.radianceVar : nullptr;
		t.lightness = nullptr; t.density = nullptr; t.recPixel = nullptr; t.recValue = nullptr;
		t.lightnessVar = nullptr; t.densityMean = nullptr;
		CHECK_CUDA(launch_wireframe(S, I.scene.dInstI2W, r.wireParams, t, r.counters, I.stream));
	} else {
		CHECK(r.ltMegakernel || r.ltParams.maxPathLength <= LTW_MAX_LAUNCHES,
		      "the light tracer's stages take at most 64 path lengths (set \"Megakernel\" to 1 for longer paths)");
		CHECK_CUDA(launch_lt(S, r.ltParams, t, r.workCounter, r.counters, I.stream, r.ltMegakernel ? nullptr : r.ltWavefront));
	}
	CHECK_CUDA(cudaEventRecord(r.evStop, I.stream));
	TraceCounters c{};
	CHECK_CUDA(cudaMemcpyAsync(&c, r.counters, sizeof(TraceCounters), cudaMemcpyDeviceToHost, I.stream));
	CHECK_CUDA(cudaStreamSynchronize(I.stream));
	CHECK_CUDA(cudaEventElapsedTime(&r.lastKernelMs, r.evStart, r.evStop));
	r.lastCounters = c;
	r.lastExtend = TraceCounters{};
	r.lastShadow = TraceCounters{};
	r.lastLaunches = 2;
	for(float& m : r.stageMs) m = 0.0f;
	check_traversal(c.errors, S.maxSteps);
	CHECK(c.waitErrors == 0, "a bounded wait of the photon-grid sort expired; the result of this call is incomplete");
}

// Brings in, through the registered LoD loader, every LoD the current
// scenario shows but its object does not hold yet (world_container.cpp
// load_scene: missing LoDs are requested from the loader).
void load_missing_lods(MufflonInstance& I) {
	HostScenario* sc = I.current;
	if(!sc || !I.lodLoader.loadLod) return;
	for(const auto& inst : I.instances) {
		if(inst->frame != NO_FRAME && inst->frame != 0) continue;
		HostObject* obj = inst->object;
		if(!obj) continue;
		if(std::find(sc->maskedInstances.begin(), sc->maskedInstances.end(), inst->index) != sc->maskedInstances.end()) continue;
		if(std::find(sc->maskedObjects.begin(), sc->maskedObjects.end(), obj) != sc->maskedObjects.end()) continue;
		const uint32_t lod = sc->effective_lod(*inst);
		if(obj->lods.count(lod)) continue;
		if(!I.lodLoader.loadLod(I.lodLoader.userParams, obj, lod, false))
			throw ApiError("the LoD loader failed to load LoD " + std::to_string(lod) + " of object '" + obj->name + "'");
		CHECK(obj->lods.count(lod), "the LoD loader did not add LoD " + std::to_string(lod) + " of object '" + obj->name + "'");
	}
}

void load_scene_if_needed(MufflonInstance& I) {
	if(!I.sceneDirty && I.scene.valid) return;
	load_missing_lods(I);
	std::string err;
	if(!build_device_scene(I, err)) throw ApiError(err);
	I.sceneDirty = false;
	I.renderer.needsReset = true;
}

} // namespace

namespace mb {
void RendererState::release() {
	if(graphExec) cudaGraphExecDestroy(graphExec);
	graphExec = nullptr;
	graphKey.clear();
	if(dIteration) cudaFree(dIteration);
	if(hIteration) cudaFreeHost(hIteration);
	dIteration = nullptr; hIteration = nullptr;
	if(wfMemory) cudaFree(wfMemory);
	wfMemory = nullptr;
	wf = WfState{};
	for(cudaEvent_t e : stageEvents) cudaEventDestroy(e);
	stageEvents.clear();
	cudaFree(rng); cudaFree(radiance); cudaFree(hitId); cudaFree(workCounter); cudaFree(counters);
	cudaFree(ltIter); cudaFree(ltIterDensity); cudaFree(lightness); cudaFree(density);
	cudaFree(ltRecPixel); cudaFree(ltRecValue);
	ltIter = nullptr; ltIterDensity = nullptr; lightness = nullptr; density = nullptr;
	ltRecPixel = nullptr; ltRecValue = nullptr; ltRecSlots = 0; ltRecFloats = 0;
	cudaFree(bptScratch);
	bptScratch = nullptr; bptScratchBytes = 0;
	cudaFree(ltWavefront);
	ltWavefront = nullptr; ltWavefrontBytes = 0;
	cudaFree(bptWavefront);
	bptWavefront = nullptr; bptWavefrontBytes = 0;
	cudaFree(vcmMemory);
	vcmMemory = nullptr; vcmMemoryBytes = 0;
	cudaFree(radianceVar); cudaFree(hitIdVar); cudaFree(lightnessVar); cudaFree(densityMean);
	radianceVar = nullptr; hitIdVar = nullptr; lightnessVar = nullptr; densityMean = nullptr;
	for(int a = 0; a < 5; ++a) { cudaFree(auxCum[a]); cudaFree(auxVarBuf[a]); auxCum[a] = nullptr; auxVarBuf[a] = nullptr; }
	cudaFree(auxMem);
	auxMem = nullptr; auxMemPixels = 0;
	if(screen) cudaFreeHost(screen);
	screen = nullptr; screenCap = 0;
	if(evStart) cudaEventDestroy(evStart);
	if(evStop) cudaEventDestroy(evStop);
	rng = nullptr; radiance = nullptr; hitId = nullptr; workCounter = nullptr; counters = nullptr;
	evStart = evStop = nullptr;
	width = height = 0;
}
MufflonInstance::~MufflonInstance() {
	renderer.release();
	scene.release();
	if(stream) cudaStreamDestroy(stream);
}
} // namespace mb

extern "C" {

const char* core_get_dll_error(void) { return s_lastError.c_str(); }
Boolean core_set_logger(void (*cb)(const char*, int)) { s_logger = cb; return true; }
Boolean core_set_log_level(LogLevel level) { s_logLevel = int(level); return true; }

// interface.cpp:4295-4414: pick the CUDA device with the highest compute capability.
MufflonInstanceHdl mufflon_initialize(void) {
	TRY
	int count = 0;
	CHECK_CUDA(cudaGetDeviceCount(&count));
	CHECK(count > 0, "no CUDA device");
	int best = 0, bestCc = -1;
	for(int d = 0; d < count; ++d) {
		cudaDeviceProp p;
		CHECK_CUDA(cudaGetDeviceProperties(&p, d));
		const int cc = p.major * 100 + p.minor;
		if(p.unifiedAddressing && cc > bestCc) { best = d; bestCc = cc; }
	}
	CHECK_CUDA(cudaSetDevice(best));
	// The allocation-free sort's device array and kernels are loaded now, so
	// that its later calls on this device take no device memory.
	CHECK_CUDA(noalloc_prepare_current_device());
	auto* I = new MufflonInstance();
	I->device = best;
	CHECK_CUDA(cudaStreamCreateWithFlags(&I->stream, cudaStreamNonBlocking));
	return I;
	CATCH_ALL(nullptr)
}

void mufflon_destroy(MufflonInstanceHdl h) {
	TRY
	delete static_cast<MufflonInstance*>(h);
	CATCH_ALL()
}

int32_t mufflon_get_cuda_device_index(void) {
	int d = -1;
	if(cudaGetDevice(&d) != cudaSuccess) return -1;
	return d;
}
Boolean mufflon_is_cuda_available(void) {
	int count = 0;
	return cudaGetDeviceCount(&count) == cudaSuccess && count > 0;
}

Boolean mufflon_set_lod_loader(MufflonInstanceHdl h, Boolean (*func)(void*, ObjectHdl, uint32_t, Boolean),
                               Boolean (*objFunc)(void*, uint32_t, uint16_t*, uint32_t*),
                               Boolean (*metaFunc)(void*, LodMetadata*, size_t*), void* userParams) {
	TRY
	MufflonInstance& I = minst(h);
	std::lock_guard<std::recursive_mutex> lock(I.iterationMutex);
	I.lodLoader.loadLod = func;
	I.lodLoader.loadMatIndices = objFunc;
	I.lodLoader.loadMetadata = metaFunc;
	I.lodLoader.userParams = userParams;
	return true;
	CATCH_ALL(false)
}

// The page-locked read-back buffer of mufflon_get_target_image (grow-only:
// a device-to-host copy into page-locked memory runs at the link's speed,
// into pageable memory it is staged through a driver buffer).
static float* screen_buffer(RendererState& r, size_t floats) {
	if(floats > r.screenCap) {
		if(r.screen) cudaFreeHost(r.screen);
		r.screen = nullptr;
		r.screenCap = 0;
		CHECK_CUDA(cudaMallocHost(&r.screen, floats * sizeof(float)));
		r.screenCap = floats;
	}
	return r.screen;
}

// interface.cpp:241-262: a library-owned copy of the cumulative target
Boolean mufflon_get_target_image(MufflonInstanceHdl h, const char* name, Boolean variance, const float** ptr) {
	TRY
	MufflonInstance& I = minst(h);
	std::lock_guard<std::recursive_mutex> lock(I.iterationMutex);
	CHECK(I.renderer.enabled, "no renderer enabled");
	CHECK(name != nullptr, "target name is null");
	RendererState& r = I.renderer;
	if(!r.rng || r.iteration < 0) { if(ptr) *ptr = nullptr; return true; }
	const size_t n = size_t(r.width) * r.height;
	// output_handler.hpp:301-318: the cumulative buffer, or with `variance`
	// the variance buffer, which must be recorded
	auto read = [&](const char* tname, bool enabled, bool varEnabled, const float* cum, const float* var, int channels) {
		CHECK(enabled, std::string("target '") + tname + "' is not enabled");
		CHECK(!variance || varEnabled, std::string("render target '") + tname + "' does not record variance");
		const float* src = variance ? var : cum;
		CHECK(src != nullptr, "no image yet");
		CHECK_CUDA(cudaMemcpyAsync(screen_buffer(r, n * size_t(channels)), src, n * size_t(channels) * sizeof(float),
		                           cudaMemcpyDeviceToHost, I.stream));
		r.screenChannels = channels;
	};
	if(!std::strcmp(name, "Radiance") && r.kind != 2) {
		read("Radiance", r.targetRadiance, r.varRadiance, r.radiance, r.radianceVar, 3);
	} else if((r.kind == 1 && (!std::strcmp(name, "Lightness") || !std::strcmp(name, "Density"))) ||
	          ((r.kind == 3 || r.kind == 4) && !std::strcmp(name, "Lightness"))) {
		if(!std::strcmp(name, "Lightness")) read("Lightness", r.targetLightness, r.varLightness, r.lightness, r.lightnessVar, 1);
		else read("Density", r.targetDensity, r.varDensity, r.density, r.densityMean, 1);
	} else if(r.kind == 2 && !std::strcmp(name, "Border")) {
		read("Border", r.targetBorder, r.varBorder, r.radiance, r.radianceVar, 3);
	} else if(r.kind == 0 && !std::strcmp(name, "Hit ID")) {
		read("Hit ID", r.targetHitId, r.varHitId, r.hitId, r.hitIdVar, 2);
	} else if(r.kind == 0 && !std::strcmp(name, "Lightness")) {
		read("Lightness", r.targetLightness, r.varLightness, r.lightness, r.lightnessVar, 1);
	} else if(r.kind == 0 && (!std::strcmp(name, "Position") || !std::strcmp(name, "Depth") || !std::strcmp(name, "Normal") ||
	                          !std::strcmp(name, "UV") || !std::strcmp(name, "Albedo"))) {
		static const char* AUX_NAMES[5] = { "Position", "Depth", "Normal", "UV", "Albedo" };
		int a = 0;
		while(std::strcmp(name, AUX_NAMES[a])) ++a;
		read(AUX_NAMES[a], r.auxTarget[a], r.auxVarOn[a], r.auxCum[a], r.auxVarBuf[a], AUX_CH[a]);
	} else {
		throw ApiError(std::string("render target '") + name + "' is not produced by the CUDA " +
		               (r.kind == 1 ? "light tracer" : r.kind == 2 ? "wireframe renderer" : r.kind == 3 ? "bidirectional path tracer"
		                : r.kind == 4 ? "vertex connection and merging renderer" : "path tracer"));
	}
	CHECK_CUDA(cudaStreamSynchronize(I.stream));
	if(ptr) *ptr = r.screen;
	return true;
	CATCH_ALL(false)
}

Boolean mufflon_get_target_image_num_channels(MufflonInstanceHdl h, int* numChannels) {
	TRY
	MufflonInstance& I = minst(h);
	if(numChannels) *numChannels = I.renderer.screenChannels;
	return true;
	CATCH_ALL(false)
}

void world_clear_all(MufflonInstanceHdl h) {
	TRY
	MufflonInstance& I = minst(h);
	std::lock_guard<std::recursive_mutex> lock(I.iterationMutex);
	I.scene.release();
	I.objects.clear(); I.instances.clear(); I.materials.clear(); I.textures.clear(); I.cameras.clear();
	I.pointLights.clear(); I.backgrounds.clear(); I.scenarios.clear(); I.current = nullptr;
	I.sceneDirty = true;
	I.renderer.needsReset = true;
	CATCH_ALL()
}

Boolean world_finalize(MufflonInstanceHdl h, const Vec3, const Vec3, const char** msg) {
	TRY
	MufflonInstance& I = minst(h);
	if(msg) *msg = "";
	CHECK(!I.cameras.empty(), "world has no camera");
	return true;
	CATCH_ALL(false)
}

// ---------------------------------------------------------------- polygons
Boolean polygon_reserve(LodHdl l, size_t v, size_t t, size_t q) {
	TRY
	HostLod& L = mlod(l);
	L.vertices.reserve(3 * v); L.normals.reserve(3 * v); L.uvs.reserve(2 * v);
	L.triIdx.reserve(3 * t); L.triMat.reserve(t); L.quadIdx.reserve(4 * q); L.quadMat.reserve(q);
	return true;
	CATCH_ALL(false)
}

VertexHdl polygon_add_vertex(LodHdl l, Vec3 p, Vec3 n, Vec2 uv) {
	TRY
	HostLod& L = mlod(l);
	const VertexHdl idx = VertexHdl(L.num_vertices());
	L.vertices.insert(L.vertices.end(), { p.x, p.y, p.z });
	L.normals.insert(L.normals.end(), { n.x, n.y, n.z });
	L.uvs.insert(L.uvs.end(), { uv.x, uv.y });
	return idx;
	CATCH_ALL(INVALID_INDEX)
}

static FaceHdl add_tri(HostLod& L, UVec3 v, MatIdx m) {
	const uint32_t nv = L.num_vertices();
	CHECK(v.x < nv && v.y < nv && v.z < nv, "triangle index out of range");
	CHECK(L.quadMat.empty(), "triangles must be added before quads");
	L.triIdx.insert(L.triIdx.end(), { v.x, v.y, v.z });
	L.triMat.push_back(m);
	return FaceHdl(L.num_triangles() - 1);
}
static FaceHdl add_quad(HostLod& L, UVec4 v, MatIdx m) {
	const uint32_t nv = L.num_vertices();
	CHECK(v.x < nv && v.y < nv && v.z < nv && v.w < nv, "quad index out of range");
	L.quadIdx.insert(L.quadIdx.end(), { v.x, v.y, v.z, v.w });
	L.quadMat.push_back(m);
	return FaceHdl(L.num_triangles() + L.num_quads() - 1);
}

FaceHdl polygon_add_triangle(LodHdl l, UVec3 v) { TRY return add_tri(mlod(l), v, 0); CATCH_ALL(INVALID_INDEX) }
FaceHdl polygon_add_triangle_material(LodHdl l, UVec3 v, MatIdx m) { TRY return add_tri(mlod(l), v, m); CATCH_ALL(INVALID_INDEX) }
FaceHdl polygon_add_quad(LodHdl l, UVec4 v) { TRY return add_quad(mlod(l), v, 0); CATCH_ALL(INVALID_INDEX) }
FaceHdl polygon_add_quad_material(LodHdl l, UVec4 v, MatIdx m) { TRY return add_quad(mlod(l), v, m); CATCH_ALL(INVALID_INDEX) }

FaceHdl polygon_add_triangle_bulk(LodHdl l, size_t count, const UVec3* v, const MatIdx* m) {
	TRY
	HostLod& L = mlod(l);
	CHECK(L.quadMat.empty(), "triangles must be added before quads");
	const uint32_t nv = L.num_vertices();
	const FaceHdl first = FaceHdl(L.num_triangles());
	L.triIdx.reserve(L.triIdx.size() + 3 * count);
	L.triMat.reserve(L.triMat.size() + count);
	for(size_t i = 0; i < count; ++i) {
		CHECK(v[i].x < nv && v[i].y < nv && v[i].z < nv, "triangle index out of range");
		L.triIdx.insert(L.triIdx.end(), { v[i].x, v[i].y, v[i].z });
		L.triMat.push_back(m ? m[i] : MatIdx(0));
	}
	return first;
	CATCH_ALL(INVALID_INDEX)
}

FaceHdl polygon_add_quad_bulk(LodHdl l, size_t count, const UVec4* v, const MatIdx* m) {
	TRY
	HostLod& L = mlod(l);
	const uint32_t nv = L.num_vertices();
	const FaceHdl first = FaceHdl(L.num_triangles() + L.num_quads());
	for(size_t i = 0; i < count; ++i) {
		CHECK(v[i].x < nv && v[i].y < nv && v[i].z < nv && v[i].w < nv, "quad index out of range");
		L.quadIdx.insert(L.quadIdx.end(), { v[i].x, v[i].y, v[i].z, v[i].w });
		L.quadMat.push_back(m ? m[i] : MatIdx(0));
	}
	return first;
	CATCH_ALL(INVALID_INDEX)
}

VertexHdl polygon_add_vertex_bulk(LodHdl l, size_t count, const BulkLoader* points, const BulkLoader* normals,
                                  const BulkLoader* uvs, const AABB*, size_t* pr, size_t* nr, size_t* ur) {
	TRY
	HostLod& L = mlod(l);
	CHECK(points != nullptr, "points stream is required");
	const VertexHdl first = VertexHdl(L.num_vertices());
	const size_t v0 = L.vertices.size(), n0 = L.normals.size(), u0 = L.uvs.size();
	L.vertices.resize(v0 + 3 * count);
	L.normals.resize(n0 + 3 * count, 0.0f);
	L.uvs.resize(u0 + 2 * count, 0.0f);
	const size_t a = read_bulk(points, L.vertices.data() + v0, 12 * count) / 12;
	const size_t b = normals ? read_bulk(normals, L.normals.data() + n0, 12 * count) / 12 : 0;
	const size_t c = uvs ? read_bulk(uvs, L.uvs.data() + u0, 8 * count) / 8 : 0;
	if(pr) *pr = a;
	if(nr) *nr = b;
	if(ur) *ur = c;
	CHECK(a == count, "short read of vertex positions");
	return first;
	CATCH_ALL(INVALID_INDEX)
}

Boolean polygon_set_material_idx(LodHdl l, FaceHdl f, MatIdx m) {
	TRY
	HostLod& L = mlod(l);
	CHECK(f >= 0 && uint32_t(f) < L.num_triangles() + L.num_quads(), "face index out of range");
	if(uint32_t(f) < L.num_triangles()) L.triMat[f] = m; else L.quadMat[f - L.num_triangles()] = m;
	return true;
	CATCH_ALL(false)
}

size_t polygon_set_material_idx_bulk(LodHdl l, FaceHdl start, size_t count, const BulkLoader* stream) {
	TRY
	HostLod& L = mlod(l);
	std::vector<MatIdx> buf(count);
	const size_t got = read_bulk(stream, buf.data(), count * sizeof(MatIdx)) / sizeof(MatIdx);
	for(size_t i = 0; i < got; ++i) {
		const size_t f = size_t(start) + i;
		CHECK(f < L.num_triangles() + L.num_quads(), "face index out of range");
		if(f < L.num_triangles()) L.triMat[f] = buf[i]; else L.quadMat[f - L.num_triangles()] = buf[i];
	}
	return got;
	CATCH_ALL(size_t(-1))
}

size_t polygon_get_vertex_count(LodHdl l) { TRY return mlod(l).num_vertices(); CATCH_ALL(0) }
size_t polygon_get_face_count(LodHdl l) { TRY return mlod(l).num_triangles() + mlod(l).num_quads(); CATCH_ALL(0) }
size_t polygon_get_triangle_count(LodHdl l) { TRY return mlod(l).num_triangles(); CATCH_ALL(0) }
size_t polygon_get_quad_count(LodHdl l) { TRY return mlod(l).num_quads(); CATCH_ALL(0) }
Boolean polygon_get_bounding_box(LodHdl l, Vec3* mn, Vec3* mx) {
	TRY
	float a[3], b[3];
	mlod(l).bounds(a, b);
	if(mn) *mn = { a[0], a[1], a[2] };
	if(mx) *mx = { b[0], b[1], b[2] };
	return true;
	CATCH_ALL(false)
}

// ---------------------------------------------------------------- spheres
Boolean spheres_reserve(LodHdl l, size_t c) { TRY mlod(l).spheres.reserve(4 * c); mlod(l).sphereMat.reserve(c); return true; CATCH_ALL(false) }
SphereHdl spheres_add_sphere(LodHdl l, Vec3 p, float r) { return spheres_add_sphere_material(l, p, r, 0); }
SphereHdl spheres_add_sphere_material(LodHdl l, Vec3 p, float r, MatIdx m) {
	TRY
	HostLod& L = mlod(l);
	CHECK(r > 0.0f, "sphere radius must be positive");
	L.spheres.insert(L.spheres.end(), { p.x, p.y, p.z, r });
	L.sphereMat.push_back(m);
	return SphereHdl(L.num_spheres() - 1);
	CATCH_ALL(INVALID_INDEX)
}
SphereHdl spheres_add_sphere_bulk(LodHdl l, size_t count, const BulkLoader* stream, const AABB*, size_t* read) {
	TRY
	HostLod& L = mlod(l);
	const SphereHdl first = SphereHdl(L.num_spheres());
	const size_t s0 = L.spheres.size();
	L.spheres.resize(s0 + 4 * count);
	const size_t got = read_bulk(stream, L.spheres.data() + s0, 16 * count) / 16;
	L.spheres.resize(s0 + 4 * got);
	L.sphereMat.resize(L.sphereMat.size() + got, 0);
	if(read) *read = got;
	return first;
	CATCH_ALL(INVALID_INDEX)
}
Boolean spheres_set_material_idx(LodHdl l, SphereHdl s, MatIdx m) {
	TRY
	HostLod& L = mlod(l);
	CHECK(s >= 0 && uint32_t(s) < L.num_spheres(), "sphere index out of range");
	L.sphereMat[s] = m;
	return true;
	CATCH_ALL(false)
}
size_t spheres_set_material_idx_bulk(LodHdl l, SphereHdl start, size_t count, const BulkLoader* stream) {
	TRY
	HostLod& L = mlod(l);
	std::vector<MatIdx> buf(count);
	const size_t got = read_bulk(stream, buf.data(), count * sizeof(MatIdx)) / sizeof(MatIdx);
	for(size_t i = 0; i < got; ++i) {
		CHECK(size_t(start) + i < L.num_spheres(), "sphere index out of range");
		L.sphereMat[size_t(start) + i] = buf[i];
	}
	return got;
	CATCH_ALL(size_t(-1))
}
size_t spheres_get_sphere_count(LodHdl l) { TRY return mlod(l).num_spheres(); CATCH_ALL(0) }
Boolean spheres_get_bounding_box(LodHdl l, Vec3* mn, Vec3* mx) { return polygon_get_bounding_box(l, mn, mx); }

// ---------------------------------------------------------------- objects / instances
ObjectHdl world_create_object(MufflonInstanceHdl h, const char* name, ObjectFlags flags) {
	TRY
	MufflonInstance& I = minst(h);
	auto o = std::make_unique<HostObject>();
	o->name = name ? name : "";
	o->flags = uint32_t(flags);
	o->id = uint32_t(I.objects.size());
	I.objects.push_back(std::move(o));
	I.sceneDirty = true;
	return I.objects.back().get();
	CATCH_ALL(nullptr)
}
ObjectHdl world_get_object(MufflonInstanceHdl h, const char* name) {
	TRY
	for(auto& o : minst(h).objects) if(name && o->name == name) return o.get();
	throw ApiError("object not found");
	CATCH_ALL(nullptr)
}
const char* world_get_object_name(ObjectHdl o) { TRY CHECK(o, "invalid object"); return static_cast<HostObject*>(o)->name.c_str(); CATCH_ALL(nullptr) }
Boolean object_has_lod(ConstObjectHdl o, LodLevel level) {
	TRY CHECK(o, "invalid object"); return static_cast<const HostObject*>(o)->lods.count(level) > 0; CATCH_ALL(false)
}
Boolean object_allocate_lod_slots(ObjectHdl o, LodLevel slots) {
	TRY
	CHECK(o, "invalid object");
	CHECK(slots >= 1, "an object needs at least one LoD slot");
	static_cast<HostObject*>(o)->lodSlots = slots;
	return true;
	CATCH_ALL(false)
}
Boolean object_get_id(ObjectHdl o, uint32_t* id) {
	TRY
	CHECK(o && id, "invalid object or id pointer");
	*id = static_cast<HostObject*>(o)->id;
	return true;
	CATCH_ALL(false)
}
LodHdl object_add_lod(ObjectHdl o, LodLevel level, Boolean) {
	TRY
	CHECK(o, "invalid object");
	CHECK(static_cast<HostObject*>(o)->lodSlots == 0 || level < static_cast<HostObject*>(o)->lodSlots,
	      "LoD level beyond the object's LoD slots");
	auto& slot = static_cast<HostObject*>(o)->lods[level];
	if(!slot) slot = std::make_unique<HostLod>();
	return slot.get();
	CATCH_ALL(nullptr)
}
void world_reserve_objects_instances(MufflonInstanceHdl h, const uint32_t o, const uint32_t i) {
	TRY minst(h).objects.reserve(o); minst(h).instances.reserve(i); CATCH_ALL()
}
InstanceHdl world_create_instance(MufflonInstanceHdl h, ObjectHdl obj, const uint32_t animationFrame) {
	TRY
	MufflonInstance& I = minst(h);
	CHECK(obj, "invalid object");
	auto inst = std::make_unique<HostInstance>();
	inst->object = static_cast<HostObject*>(obj);
	inst->index = uint32_t(I.instances.size());
	inst->frame = animationFrame;
	I.instances.push_back(std::move(inst));
	I.sceneDirty = true;
	return I.instances.back().get();
	CATCH_ALL(nullptr)
}
uint32_t world_get_instance_count(MufflonInstanceHdl h, const uint32_t frame) {
	TRY
	uint32_t n = 0;
	for(const auto& i : minst(h).instances) n += (i->frame == frame) ? 1u : 0u;
	return n;
	CATCH_ALL(0)
}
Boolean world_get_frame_count(MufflonInstanceHdl h, uint32_t* frameCount) {
	TRY (void)minst(h); CHECK(frameCount, "frame count pointer is null"); *frameCount = 1u; return true; CATCH_ALL(false)
}

// Inverse of an affine 3x4 (row-major, translation in the last column), as
// InstanceData::compute_instance_to_world_transformation computes it; the same
// formula maps either direction.
static void invert_affine(const float* r, float* o) {
	const float m00 = r[5] * r[10] - r[9] * r[6], m01 = r[9] * r[2] - r[1] * r[10], m02 = r[1] * r[6] - r[5] * r[2];
	const float m10 = r[8] * r[6] - r[4] * r[10], m11 = r[0] * r[10] - r[8] * r[2], m12 = r[4] * r[2] - r[0] * r[6];
	const float m20 = r[4] * r[9] - r[8] * r[5], m21 = r[8] * r[1] - r[0] * r[9], m22 = r[0] * r[5] - r[4] * r[1];
	const float det = r[0] * m00 + r[1] * m10 + r[2] * m20;
	CHECK(det != 0.0f, "singular transformation");
	const float id = 1.0f / det;
	const float i[9] = { id * m00, id * m01, id * m02, id * m10, id * m11, id * m12, id * m20, id * m21, id * m22 };
	for(int row = 0; row < 3; ++row) {
		o[4 * row] = i[3 * row]; o[4 * row + 1] = i[3 * row + 1]; o[4 * row + 2] = i[3 * row + 2];
		o[4 * row + 3] = -(i[3 * row] * r[3] + i[3 * row + 1] * r[7] + i[3 * row + 2] * r[11]);
	}
}

// instance_set_transformation_matrix: the stored matrix is world-to-instance;
// an instance-to-world input is inverted.
Boolean instance_set_transformation_matrix(MufflonInstanceHdl h, InstanceHdl inst, const Mat3x4* mat, const Boolean isWorldToInst) {
	TRY
	MufflonInstance& I = minst(h);
	CHECK(inst && mat, "invalid instance or matrix");
	HostInstance& in = *static_cast<HostInstance*>(inst);
	if(isWorldToInst) std::memcpy(in.worldToInstance, mat->v, sizeof(in.worldToInstance));
	else invert_affine(mat->v, in.worldToInstance);
	I.sceneDirty = true;
	return true;
	CATCH_ALL(false)
}
// interface.cpp:1017-1027: returns the instance-to-world transformation
Boolean instance_get_transformation_matrix(MufflonInstanceHdl h, InstanceHdl inst, Mat3x4* mat) {
	TRY
	(void)minst(h);
	CHECK(inst && mat, "invalid instance or matrix");
	invert_affine(static_cast<HostInstance*>(inst)->worldToInstance, mat->v);
	return true;
	CATCH_ALL(false)
}

// ---------------------------------------------------------------- materials / textures
MaterialHdl world_add_material(MufflonInstanceHdl h, const char* name, const MaterialParams* p) {
	TRY
	MufflonInstance& I = minst(h);
	CHECK(p, "material parameters are null");
	auto m = std::make_unique<HostMaterial>();
	m->name = name ? name : "";
	switch(p->innerType) {
		case MATERIAL_LAMBERT:
			m->type = MAT_LAMBERT;
			m->albedo = static_cast<HostTexture*>(p->inner.lambert.albedo);
			break;
		case MATERIAL_TORRANCE:
			CHECK(p->inner.torrance.ndf == NDF_GGX, "the CUDA path tracer implements Torrance with the GGX distribution");
			CHECK(p->inner.torrance.shadowingModel == SHADOWING_SMITH || p->inner.torrance.shadowingModel == SHADOWING_VCAVITY,
			      "unknown shadowing model");
			m->type = MAT_TORRANCE;
			m->shadowing = p->inner.torrance.shadowingModel == SHADOWING_SMITH ? SHADOW_SMITH : SHADOW_VCAVITY;
			m->albedo = static_cast<HostTexture*>(p->inner.torrance.albedo);
			m->roughness = static_cast<HostTexture*>(p->inner.torrance.roughness);
			CHECK(!m->roughness || (m->roughness->width == 1 && m->roughness->height == 1),
			      "the CUDA path tracer takes a constant roughness (a 1x1 value texture)");
			break;
		case MATERIAL_EMISSIVE:
			m->type = MAT_EMISSIVE;
			m->radiance = static_cast<HostTexture*>(p->inner.emissive.radiance);
			CHECK(!m->radiance || (m->radiance->width == 1 && m->radiance->height == 1),
			      "the CUDA path tracer takes a constant emitted radiance (a 1x1 value texture)");
			m->scale[0] = p->inner.emissive.scale.x; m->scale[1] = p->inner.emissive.scale.y; m->scale[2] = p->inner.emissive.scale.z;
			break;
		default:
			throw ApiError("material type not implemented by the CUDA path tracer");
	}
	m->alpha = static_cast<HostTexture*>(p->alpha); // interface.cpp:1350-1351
	I.materials.push_back(std::move(m));
	I.sceneDirty = true;
	return I.materials.back().get();
	CATCH_ALL(nullptr)
}
IndexType world_get_material_count(MufflonInstanceHdl h) { TRY return IndexType(minst(h).materials.size()); CATCH_ALL(INVALID_INDEX) }

TextureHdl world_add_texture_value(MufflonInstanceHdl h, const float* value, int num, TextureSampling) {
	TRY
	MufflonInstance& I = minst(h);
	CHECK(value && num >= 1 && num <= 4, "texture value needs 1 to 4 channels");
	auto t = std::make_unique<HostTexture>();
	t->width = t->height = 1;
	t->channels = uint32_t(num);
	t->texels.assign(4, 0.0f);
	for(int i = 0; i < num; ++i) t->texels[i] = value[i];
	I.textures.push_back(std::move(t));
	return I.textures.back().get();
	CATCH_ALL(nullptr)
}

TextureHdl world_add_texture_rgba32f(MufflonInstanceHdl h, const char* name, uint32_t w, uint32_t hh, const float* texels, TextureSampling) {
	TRY
	MufflonInstance& I = minst(h);
	CHECK(texels && w > 0 && hh > 0, "invalid texture");
	auto t = std::make_unique<HostTexture>();
	t->name = name ? name : "";
	t->width = w; t->height = hh; t->channels = 4;
	t->texels.assign(texels, texels + size_t(w) * hh * 4);
	I.textures.push_back(std::move(t));
	I.sceneDirty = true;
	return I.textures.back().get();
	CATCH_ALL(nullptr)
}

// core_interface.h:469-477. The core reads texture files itself (it has no
// plugin system): PFM files ("PF" RGB, "Pf" one channel) as the reference's
// PFM plugin reads them (src/pfmloader/interface.cpp:74-160); any other
// format fails with a message, as a path no plugin can load does
// (interface.cpp:1831-1835). A path that is already loaded returns the same
// texture. A callback rewrites every texel once (interface.cpp:1843-1856).
// Textures are sampled with the nearest texel whatever the sampling mode, and
// carry no mipmaps.
TextureHdl world_add_texture(MufflonInstanceHdl h, const char* path, TextureSampling, MipmapType,
                             TextureCallback callback, void* userParams) {
	TRY
	MufflonInstance& I = minst(h);
	CHECK(path, "texture path is null");
	for(auto& t : I.textures)
		if(t->name == path) return t.get();
	const std::string p(path);
	const size_t dot = p.find_last_of('.');
	std::string ext = dot == std::string::npos ? std::string() : p.substr(dot);
	for(char& c : ext) c = char(std::tolower(static_cast<unsigned char>(c)));
	CHECK(ext == ".pfm", "no texture reader for '" + p + "' (the core reads PFM files)");
	std::ifstream f(p, std::ios::binary);
	CHECK(f.good(), "cannot open texture file '" + p + "'");
	const std::string bytes((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
	PfmImage img;
	try {
		img = parse_pfm(bytes);
	} catch(const std::runtime_error& e) {
		throw ApiError("texture '" + p + "': " + e.what());
	}
	auto t = std::make_unique<HostTexture>();
	t->name = p;
	t->width = img.width; t->height = img.height;
	t->channels = img.channels == 1 ? 1u : 4u;
	t->texels = std::move(img.rgba);
	if(callback) {
		const TextureFormat fmt = img.channels == 1 ? FORMAT_R32F : FORMAT_RGBA32F;
		for(uint32_t y = 0; y < t->height; ++y)
			for(uint32_t x = 0; x < t->width; ++x) {
				float* v = &t->texels[(size_t(y) * t->width + x) * 4];
				const Vec4 out = callback(x, y, 0u, fmt, Vec4{ v[0], v[1], v[2], v[3] }, userParams);
				v[0] = out.x;
				if(t->channels == 4) { v[1] = out.y; v[2] = out.z; v[3] = out.w; }
			}
	}
	I.textures.push_back(std::move(t));
	I.sceneDirty = true;
	return I.textures.back().get();
	CATCH_ALL(nullptr)
}

TextureHdl world_get_texture(MufflonInstanceHdl h, const char* path) {
	TRY
	MufflonInstance& I = minst(h);
	CHECK(path, "texture path is null");
	for(auto& t : I.textures)
		if(t->name == path) return t.get();
	throw ApiError(std::string("could not find texture ") + path);
	CATCH_ALL(nullptr)
}

const char* world_get_texture_name(TextureHdl hdl) {
	TRY
	CHECK(hdl, "texture handle is null");
	return static_cast<HostTexture*>(hdl)->name.c_str();
	CATCH_ALL(nullptr)
}

Boolean world_get_texture_size(TextureHdl hdl, IVec2* size) {
	TRY
	CHECK(hdl && size, "texture handle or size is null");
	const HostTexture* t = static_cast<HostTexture*>(hdl);
	size->x = int32_t(t->width);
	size->y = int32_t(t->height);
	return true;
	CATCH_ALL(false)
}

// ---------------------------------------------------------------- cameras
CameraHdl world_add_pinhole_camera(MufflonInstanceHdl h, const char* name, const Vec3* pos, const Vec3* dir,
                                   const Vec3* up, const uint32_t pathCount, float nearP, float farP, float vFov) {
	TRY
	MufflonInstance& I = minst(h);
	CHECK(pos && dir && up && pathCount >= 1, "invalid camera description");
	auto c = std::make_unique<HostCamera>();
	c->name = name ? name : "";
	c->position[0] = pos->x; c->position[1] = pos->y; c->position[2] = pos->z;
	c->dir[0] = dir->x; c->dir[1] = dir->y; c->dir[2] = dir->z;
	c->up[0] = up->x; c->up[1] = up->y; c->up[2] = up->z;
	c->nearPlane = nearP; c->farPlane = farP; c->vFov = vFov;
	I.cameras.push_back(std::move(c));
	return I.cameras.back().get();
	CATCH_ALL(nullptr)
}
CameraHdl world_get_camera(MufflonInstanceHdl h, const char* name) {
	TRY
	for(auto& c : minst(h).cameras) if(name && c->name == name) return c.get();
	throw ApiError("camera not found");
	CATCH_ALL(nullptr)
}
Boolean world_set_camera_position(CameraHdl cam, Vec3 p, const uint32_t) {
	TRY CHECK(cam, "invalid camera"); auto* c = static_cast<HostCamera*>(cam);
	c->position[0] = p.x; c->position[1] = p.y; c->position[2] = p.z; return true; CATCH_ALL(false)
}
Boolean world_set_camera_direction(CameraHdl cam, Vec3 d, Vec3 u, const uint32_t) {
	TRY CHECK(cam, "invalid camera"); auto* c = static_cast<HostCamera*>(cam);
	c->dir[0] = d.x; c->dir[1] = d.y; c->dir[2] = d.z; c->up[0] = u.x; c->up[1] = u.y; c->up[2] = u.z; return true; CATCH_ALL(false)
}
Boolean world_set_pinhole_camera_fov(CameraHdl cam, float vFov) {
	TRY CHECK(cam, "invalid camera"); static_cast<HostCamera*>(cam)->vFov = vFov; return true; CATCH_ALL(false)
}
Boolean world_set_camera_near(CameraHdl cam, float nearP) {
	TRY CHECK(cam, "invalid camera"); CHECK(nearP > 0.0f, "near plane must be positive");
	static_cast<HostCamera*>(cam)->nearPlane = nearP; return true; CATCH_ALL(false)
}
Boolean world_set_camera_far(CameraHdl cam, float farP) {
	TRY CHECK(cam, "invalid camera"); CHECK(farP > 0.0f, "far plane must be positive");
	static_cast<HostCamera*>(cam)->farPlane = farP; return true; CATCH_ALL(false)
}

// ---------------------------------------------------------------- scenarios
void world_reserve_scenarios(MufflonInstanceHdl h, const uint32_t n) { TRY minst(h).scenarios.reserve(n); CATCH_ALL() }
ScenarioHdl world_create_scenario(MufflonInstanceHdl h, const char* name) {
	TRY
	MufflonInstance& I = minst(h);
	auto s = std::make_unique<HostScenario>();
	s->name = name ? name : "";
	I.scenarios.push_back(std::move(s));
	return I.scenarios.back().get();
	CATCH_ALL(nullptr)
}
ScenarioHdl world_find_scenario(MufflonInstanceHdl h, const char* name) {
	TRY
	for(auto& s : minst(h).scenarios) if(name && s->name == name) return s.get();
	throw ApiError("scenario not found");
	CATCH_ALL(nullptr)
}
ConstScenarioHdl world_get_current_scenario(MufflonInstanceHdl h) { TRY return minst(h).current; CATCH_ALL(nullptr) }
Boolean world_finalize_scenario(MufflonInstanceHdl h, ScenarioHdl s, const char** msg) {
	TRY
	(void)minst(h);
	CHECK(s, "invalid scenario");
	if(msg) *msg = "";
	CHECK(static_cast<HostScenario*>(s)->camera != nullptr, "scenario has no camera");
	return true;
	CATCH_ALL(false)
}
SceneHdl world_load_scenario(MufflonInstanceHdl h, ScenarioHdl s) {
	TRY
	MufflonInstance& I = minst(h);
	std::lock_guard<std::recursive_mutex> lock(I.iterationMutex);
	CHECK(s, "invalid scenario");
	I.current = static_cast<HostScenario*>(s);
	I.sceneDirty = true;
	load_scene_if_needed(I);
	return &I.scene;
	CATCH_ALL(nullptr)
}
const char* scenario_get_name(ScenarioHdl s) { TRY CHECK(s, "invalid scenario"); return static_cast<HostScenario*>(s)->name.c_str(); CATCH_ALL(nullptr) }
Boolean scenario_get_resolution(ScenarioHdl s, uint32_t* w, uint32_t* h) {
	TRY CHECK(s, "invalid scenario"); auto* sc = static_cast<HostScenario*>(s); if(w) *w = sc->width; if(h) *h = sc->height; return true; CATCH_ALL(false)
}
Boolean scenario_set_resolution(ScenarioHdl s, uint32_t w, uint32_t h) {
	TRY CHECK(s, "invalid scenario"); CHECK(w > 0 && h > 0 && w <= 65535 && h <= 65535, "resolution out of range");
	auto* sc = static_cast<HostScenario*>(s); sc->width = w; sc->height = h; return true; CATCH_ALL(false)
}
CameraHdl scenario_get_camera(ScenarioHdl s) { TRY CHECK(s, "invalid scenario"); return static_cast<HostScenario*>(s)->camera; CATCH_ALL(nullptr) }
Boolean scenario_set_camera(MufflonInstanceHdl h, ScenarioHdl s, CameraHdl cam) {
	TRY (void)minst(h); CHECK(s && cam, "invalid scenario or camera"); static_cast<HostScenario*>(s)->camera = static_cast<HostCamera*>(cam); return true; CATCH_ALL(false)
}
Boolean scenario_mask_instance(ScenarioHdl s, InstanceHdl inst) {
	TRY CHECK(s && inst, "invalid scenario or instance");
	static_cast<HostScenario*>(s)->maskedInstances.push_back(static_cast<HostInstance*>(inst)->index); return true; CATCH_ALL(false)
}
Boolean scenario_mask_object(ScenarioHdl s, ObjectHdl obj) {
	TRY CHECK(s && obj, "invalid scenario or object");
	auto& m = static_cast<HostScenario*>(s)->maskedObjects;
	if(std::find(m.begin(), m.end(), static_cast<const HostObject*>(obj)) == m.end()) m.push_back(static_cast<const HostObject*>(obj));
	return true;
	CATCH_ALL(false)
}
Boolean scenario_is_object_masked(ScenarioHdl s, ObjectHdl obj) {
	TRY CHECK(s && obj, "invalid scenario or object");
	const auto& m = static_cast<HostScenario*>(s)->maskedObjects;
	return std::find(m.begin(), m.end(), static_cast<const HostObject*>(obj)) != m.end();
	CATCH_ALL(false)
}
LodLevel scenario_get_global_lod_level(ScenarioHdl s) { TRY CHECK(s, "invalid scenario"); return static_cast<HostScenario*>(s)->globalLod; CATCH_ALL(0u) }
Boolean scenario_set_global_lod_level(ScenarioHdl s, LodLevel level) {
	TRY CHECK(s, "invalid scenario"); static_cast<HostScenario*>(s)->globalLod = level; return true; CATCH_ALL(false)
}
LodLevel scenario_get_object_lod(ScenarioHdl s, ObjectHdl obj) {
	TRY CHECK(s && obj, "invalid scenario or object");
	const auto* sc = static_cast<HostScenario*>(s);
	auto it = sc->objectLods.find(static_cast<const HostObject*>(obj));
	return it == sc->objectLods.end() ? sc->globalLod : it->second;
	CATCH_ALL(0u)
}
Boolean scenario_set_object_lod(ScenarioHdl s, ObjectHdl obj, LodLevel level) {
	TRY CHECK(s && obj, "invalid scenario or object");
	static_cast<HostScenario*>(s)->objectLods[static_cast<const HostObject*>(obj)] = level; return true; CATCH_ALL(false)
}
Boolean scenario_set_instance_lod(ScenarioHdl s, InstanceHdl inst, LodLevel level) {
	TRY CHECK(s && inst, "invalid scenario or instance");
	static_cast<HostScenario*>(s)->instanceLods[static_cast<HostInstance*>(inst)->index] = level; return true; CATCH_ALL(false)
}
void scenario_reserve_material_slots(ScenarioHdl s, size_t n) {
	TRY CHECK(s, "invalid scenario"); auto* sc = static_cast<HostScenario*>(s);
	sc->slotNames.reserve(n); sc->slotMaterials.reserve(n); CATCH_ALL()
}
void scenario_reserve_custom_object_properties(ScenarioHdl s, size_t) { TRY CHECK(s, "invalid scenario"); CATCH_ALL() }
void scenario_reserve_custom_instance_properties(ScenarioHdl s, size_t n) {
	TRY CHECK(s, "invalid scenario"); static_cast<HostScenario*>(s)->maskedInstances.reserve(n); CATCH_ALL()
}
Boolean scenario_add_light(MufflonInstanceHdl h, ScenarioHdl s, LightHdl hdl) {
	TRY
	MufflonInstance& I = minst(h);
	CHECK(s, "invalid scenario");
	auto* sc = static_cast<HostScenario*>(s);
	if(hdl.type == LIGHT_POINT) {
		CHECK(hdl.index < I.pointLights.size(), "invalid point light");
		sc->pointLights.push_back(hdl.index);
	} else if(hdl.type == LIGHT_ENVMAP) {
		CHECK(hdl.index < I.backgrounds.size(), "invalid background light");
		sc->background = int32_t(hdl.index);
	} else {
		throw ApiError("light type not implemented by the CUDA path tracer");
	}
	I.sceneDirty = true;
	return true;
	CATCH_ALL(false)
}
MatIdx scenario_declare_material_slot(ScenarioHdl s, const char* name, size_t len) {
	TRY
	CHECK(s, "invalid scenario");
	auto* sc = static_cast<HostScenario*>(s);
	const std::string n(name ? name : "", name ? len : 0);
	for(size_t i = 0; i < sc->slotNames.size(); ++i) if(sc->slotNames[i] == n) return MatIdx(i);
	sc->slotNames.push_back(n);
	sc->slotMaterials.push_back(nullptr);
	return MatIdx(sc->slotNames.size() - 1);
	CATCH_ALL(MatIdx(0xFFFF))
}
MatIdx scenario_get_material_slot(ScenarioHdl s, const char* name, size_t len) {
	TRY
	CHECK(s, "invalid scenario");
	auto* sc = static_cast<HostScenario*>(s);
	const std::string n(name ? name : "", name ? len : 0);
	for(size_t i = 0; i < sc->slotNames.size(); ++i) if(sc->slotNames[i] == n) return MatIdx(i);
	throw ApiError("material slot not found");
	CATCH_ALL(MatIdx(0xFFFF))
}
Boolean scenario_assign_material(ScenarioHdl s, MatIdx idx, MaterialHdl m) {
	TRY
	CHECK(s && m, "invalid scenario or material");
	auto* sc = static_cast<HostScenario*>(s);
	CHECK(idx < sc->slotMaterials.size(), "material slot out of range");
	sc->slotMaterials[idx] = static_cast<HostMaterial*>(m);
	return true;
	CATCH_ALL(false)
}
SceneHdl world_get_current_scene(MufflonInstanceHdl h) { TRY MufflonInstance& I = minst(h); return I.scene.valid ? &I.scene : nullptr; CATCH_ALL(nullptr) }
Boolean scene_get_bounding_box(SceneHdl s, Vec3* mn, Vec3* mx) {
	TRY CHECK(s, "invalid scene"); auto* d = static_cast<DeviceScene*>(s);
	if(mn) *mn = { d->aabb[0], d->aabb[1], d->aabb[2] };
	if(mx) *mx = { d->aabb[3], d->aabb[4], d->aabb[5] };
	return true;
	CATCH_ALL(false)
}

// ---------------------------------------------------------------- lights
LightHdl world_add_light(MufflonInstanceHdl h, const char* name, LightType type, const uint32_t count) {
	LightHdl bad; bad.type = 7; bad.index = 0x1FFFFFFF;
	TRY
	MufflonInstance& I = minst(h);
	CHECK(type == LIGHT_POINT, "the CUDA path tracer implements point, area and environment lights");
	HostPointLight l;
	l.name = name ? name : "";
	l.frames = std::max<uint32_t>(count, 1u);
	I.pointLights.push_back(l);
	LightHdl r; r.type = LIGHT_POINT; r.index = uint32_t(I.pointLights.size() - 1);
	return r;
	CATCH_ALL(bad)
}
LightHdl world_add_background_light(MufflonInstanceHdl h, const char* name, BackgroundType type) {
	LightHdl bad; bad.type = 7; bad.index = 0x1FFFFFFF;
	TRY
	MufflonInstance& I = minst(h);
	CHECK(type == BACKGROUND_MONOCHROME, "the CUDA path tracer implements monochrome backgrounds");
	HostBackground b;
	b.name = name ? name : "";
	I.backgrounds.push_back(b);
	LightHdl r; r.type = LIGHT_ENVMAP; r.index = uint32_t(I.backgrounds.size() - 1);
	return r;
	CATCH_ALL(bad)
}
// Point lights keep the values of animation frame 0, the frame the world shows;
// other frames (< the count given to world_add_light) are accepted and unused.
Boolean world_set_point_light_position(MufflonInstanceHdl h, LightHdl l, Vec3 p, const uint32_t frame) {
	TRY MufflonInstance& I = minst(h); CHECK(l.type == LIGHT_POINT && l.index < I.pointLights.size(), "invalid point light");
	auto& L = I.pointLights[l.index]; CHECK(frame < L.frames, "animation frame out of range");
	if(frame != 0) return true;
	L.position[0] = p.x; L.position[1] = p.y; L.position[2] = p.z; I.sceneDirty = true; return true; CATCH_ALL(false)
}
Boolean world_set_point_light_intensity(MufflonInstanceHdl h, LightHdl l, Vec3 v, const uint32_t frame) {
	TRY MufflonInstance& I = minst(h); CHECK(l.type == LIGHT_POINT && l.index < I.pointLights.size(), "invalid point light");
	auto& L = I.pointLights[l.index]; CHECK(frame < L.frames, "animation frame out of range");
	if(frame != 0) return true;
	L.intensity[0] = v.x; L.intensity[1] = v.y; L.intensity[2] = v.z; I.sceneDirty = true; return true; CATCH_ALL(false)
}
Boolean world_set_env_light_color(MufflonInstanceHdl h, LightHdl l, Vec3 c) {
	TRY MufflonInstance& I = minst(h); CHECK(l.type == LIGHT_ENVMAP && l.index < I.backgrounds.size(), "invalid background light");
	auto& B = I.backgrounds[l.index]; B.color[0] = c.x; B.color[1] = c.y; B.color[2] = c.z; I.sceneDirty = true; return true; CATCH_ALL(false)
}
Boolean world_set_env_light_scale(MufflonInstanceHdl h, LightHdl l, Vec3 c) {
	TRY MufflonInstance& I = minst(h); CHECK(l.type == LIGHT_ENVMAP && l.index < I.backgrounds.size(), "invalid background light");
	auto& B = I.backgrounds[l.index]; B.scale[0] = c.x; B.scale[1] = c.y; B.scale[2] = c.z; I.sceneDirty = true; return true; CATCH_ALL(false)
}

// ---------------------------------------------------------------- renderers
// Renderers grouped by name in the reference's registry order (renderers.hpp:23-31,
// interface.cpp:126-154): the path tracer, the light tracer, the wireframe
// renderer, the bidirectional path tracer and vertex connection and merging
// (the last two CPU-only in the reference), each with a CUDA variation.
const char* RENDERER_NAMES[5][2] = { { "Pathtracer", "PT" }, { "Lighttracer", "LT" }, { "Wireframe", "WF" },
                                     { "Bidirectional Pathtracer", "BPT" }, { "Vertex Connection and Merging", "VCM" } };
constexpr uint32_t NUM_RENDERERS = 5u;
uint32_t render_get_renderer_count(MufflonInstanceHdl h) { TRY (void)minst(h); return NUM_RENDERERS; CATCH_ALL(0u) }
uint32_t render_get_renderer_variations(MufflonInstanceHdl h, uint32_t index) {
	TRY (void)minst(h); CHECK(index < NUM_RENDERERS, "renderer index out of bounds"); return 1u; CATCH_ALL(0u)
}
const char* render_get_renderer_name(MufflonInstanceHdl h, uint32_t index) {
	TRY (void)minst(h); CHECK(index < NUM_RENDERERS, "renderer index out of bounds"); return RENDERER_NAMES[index][0]; CATCH_ALL(nullptr)
}
const char* render_get_renderer_short_name(MufflonInstanceHdl h, uint32_t index) {
	TRY (void)minst(h); CHECK(index < NUM_RENDERERS, "renderer index out of bounds"); return RENDERER_NAMES[index][1]; CATCH_ALL(nullptr)
}
RenderDevice render_get_renderer_devices(MufflonInstanceHdl h, uint32_t index, uint32_t variation) {
	TRY (void)minst(h); CHECK(index < NUM_RENDERERS && variation == 0, "renderer index out of bounds"); return DEVICE_CUDA; CATCH_ALL(DEVICE_NONE)
}
Boolean render_enable_renderer(MufflonInstanceHdl h, uint32_t index, uint32_t variation) {
	TRY
	MufflonInstance& I = minst(h);
	std::lock_guard<std::recursive_mutex> lock(I.iterationMutex);
	CHECK(index < NUM_RENDERERS && variation == 0, "renderer index out of bounds");
	I.renderer.enabled = true;
	I.renderer.kind = int32_t(index);
	I.renderer.needsReset = true;
	return true;
	CATCH_ALL(false)
}

// interface.cpp:3611-3685: one iteration = one sample per pixel
Boolean render_iterate(MufflonInstanceHdl h, ProcessTime* iterTime, ProcessTime* preTime, ProcessTime* postTime) {
	TRY
	MufflonInstance& I = minst(h);
	std::lock_guard<std::recursive_mutex> lock(I.iterationMutex);
	CHECK(I.renderer.enabled, "No renderer is currently set");
	CHECK(I.current != nullptr, "Failed to load scenario");
	using clk = std::chrono::steady_clock;
	auto t0 = clk::now();
	load_scene_if_needed(I);
	ensure_render_buffers(I);
	RendererState& r = I.renderer;
	I.scene.desc.maxSteps = step_limit(r);
	const uint32_t n = r.width * r.height;
	if(r.kind != 0) ensure_lt_buffers(I);
	else ensure_aux_buffers(I);
	ensure_variance_buffers(I);
	if(r.needsReset) {
		// cpu_pt.cpp:40-45, cpu_lt.cpp:33-38: one generator per pixel index
		// the wireframe renderer's generators are seeded with the pixel index (cpu_wireframe.cpp:31-36)
		const int32_t seed = r.kind == 1 ? r.ltParams.seed : r.kind == 3 ? r.bptParams.seed : r.kind == 4 ? r.vcmParams.seed
		                   : r.kind == 2 ? 0 : r.params.seed;
		CHECK_CUDA(launch_seed_rng(r.rng, n, seed, I.stream));
		CHECK_CUDA(cudaMemsetAsync(r.radiance, 0, size_t(n) * 3 * sizeof(float), I.stream));
		CHECK_CUDA(cudaMemsetAsync(r.hitId, 0, size_t(n) * 2 * sizeof(float), I.stream));
		if(r.lightness) CHECK_CUDA(cudaMemsetAsync(r.lightness, 0, size_t(n) * sizeof(float), I.stream));
		if(r.density) CHECK_CUDA(cudaMemsetAsync(r.density, 0, size_t(n) * sizeof(float), I.stream));
		if(r.radianceVar) CHECK_CUDA(cudaMemsetAsync(r.radianceVar, 0, size_t(n) * 3 * sizeof(float), I.stream));
		if(r.hitIdVar) CHECK_CUDA(cudaMemsetAsync(r.hitIdVar, 0, size_t(n) * 2 * sizeof(float), I.stream));
		if(r.lightnessVar) CHECK_CUDA(cudaMemsetAsync(r.lightnessVar, 0, size_t(n) * sizeof(float), I.stream));
		if(r.densityMean) CHECK_CUDA(cudaMemsetAsync(r.densityMean, 0, size_t(n) * sizeof(float), I.stream));
		for(int a = 0; a < 5; ++a) {
			if(r.auxCum[a]) CHECK_CUDA(cudaMemsetAsync(r.auxCum[a], 0, size_t(n) * AUX_CH[a] * sizeof(float), I.stream));
			if(r.auxVarBuf[a]) CHECK_CUDA(cudaMemsetAsync(r.auxVarBuf[a], 0, size_t(n) * AUX_CH[a] * sizeof(float), I.stream));
		}
		r.iteration = 0;
		r.needsReset = false;
	} else {
		++r.iteration;
	}
	auto t1 = clk::now();
	if(r.kind != 0) {
		iterate_lt(I);
		auto t2 = clk::now();
		auto us = [](clk::duration d) { return uint64_t(std::chrono::duration_cast<std::chrono::microseconds>(d).count()); };
		if(preTime) { preTime->cycles = 0; preTime->microseconds = us(t1 - t0); }
		if(iterTime) { iterTime->cycles = 0; iterTime->microseconds = us(t2 - t1); }
		if(postTime) { postTime->cycles = 0; postTime->microseconds = 0; }
		return true;
	}
	RenderState rs{};
	rs.rngState = r.rng;
	rs.radiance = r.targetRadiance ? r.radiance : nullptr;
	rs.hitId = r.targetHitId ? r.hitId : nullptr;
	rs.radianceVar = r.targetRadiance && r.varRadiance ? r.radianceVar : nullptr;
	rs.hitIdVar = r.targetHitId && r.varHitId ? r.hitIdVar : nullptr;
	for(int a = 0; a < 5; ++a) {
		rs.aux[a] = r.auxTarget[a] ? r.auxCum[a] : nullptr;
		rs.auxVar[a] = r.auxTarget[a] && r.auxVarOn[a] ? r.auxVarBuf[a] : nullptr;
	}
	rs.aux[5] = r.targetLightness ? r.lightness : nullptr;
	rs.auxVar[5] = r.targetLightness && r.varLightness ? r.lightnessVar : nullptr;
	rs.auxOn = aux_wanted(r) ? 1 : 0;
	// the wavefront's per-path auxiliary state (in the graph key through r.wf)
	r.wf.guide = nullptr; r.wf.auxIter = nullptr; r.wf.auxStride = 0;
	rs.width = r.width; rs.height = r.height;
	rs.iteration = r.iteration;
	CHECK_CUDA(cudaMemsetAsync(r.counters, 0, 2 * sizeof(TraceCounters), I.stream));
	WfLaunchInfo info;
	if(!r.megakernel) {
		ensure_wavefront_buffers(I);
		if(rs.auxOn) {
			r.wf.guide = static_cast<float2*>(r.auxMem);
			r.wf.auxIter = reinterpret_cast<float*>(static_cast<char*>(r.auxMem) + size_t(n) * sizeof(float2));
			r.wf.auxStride = n;
		}
		if(r.stageTiming) {
			const int pairs = 3 * std::max(1, r.params.maxPathLength) + 2;
			while(int(r.stageEvents.size()) < 2 * pairs) {
				cudaEvent_t e;
				CHECK_CUDA(cudaEventCreate(&e));
				r.stageEvents.push_back(e);
			}
			r.stageKinds.resize(pairs);
			info.events = r.stageEvents.data();
			info.kinds = r.stageKinds.data();
			info.eventPairs = pairs;
		}
	}
	WfTuning tune;
	tune.traceBlocksPerSm = r.traceBlocksPerSm;
	tune.wavefrontBounces = r.wavefrontBounces;
	tune.refillLanes = r.refillLanes;
	tune.tailPaths = r.tailPaths;
	tune.sortBits = r.sortBits;
	tune.sortDirBits = r.sortDirBits;
	tune.counters = r.traversalStats != 0; // the counting kernel variants only when asked for
	// The schedule is planned from the previous iteration's queue lengths
	// when it ran with the same scene and parameters (every schedule renders
	// the same bits; only the launch count differs).
	std::vector<unsigned char> planKey;
	{
		auto addp = [&](const void* p, size_t b) { const unsigned char* c = static_cast<const unsigned char*>(p); planKey.insert(planKey.end(), c, c + b); };
		addp(&I.scene.desc, sizeof(DScene)); addp(&r.params, sizeof(PtParams));
		addp(&r.wavefrontBounces, sizeof(int32_t)); addp(&r.tailPaths, sizeof(int32_t));
		addp(&r.width, sizeof(r.width)); addp(&r.height, sizeof(r.height));
	}
	if(!r.megakernel && r.planTail && planKey == r.planKey) tune.tailBounce = r.plannedTail;
	const bool graph = !r.megakernel && !r.stageTiming && r.iterationGraph;
	if(graph) {
		// The launch sequence of an iteration is the same every iteration
		// (the iteration number is read from device memory), so it is
		// captured once and replayed; it is captured again when anything it
		// was built from changes.
		if(!r.dIteration) {
			CHECK_CUDA(cudaMalloc(&r.dIteration, sizeof(int32_t)));
			CHECK_CUDA(cudaMallocHost(&r.hIteration, sizeof(int32_t)));
		}
		rs.dIteration = r.dIteration;
		rs.iteration = 0; // read from dIteration: not part of the captured launches
		std::vector<unsigned char> key;
		auto add = [&](const void* p, size_t b) { const unsigned char* c = static_cast<const unsigned char*>(p); key.insert(key.end(), c, c + b); };
		add(&I.scene.desc, sizeof(DScene)); add(&r.params, sizeof(PtParams)); add(&tune, sizeof(WfTuning));
		add(&rs, sizeof(RenderState)); add(&r.wf, sizeof(WfState)); add(&r.counters, sizeof(r.counters));
		if(!r.graphExec || key != r.graphKey) {
			if(r.graphExec) cudaGraphExecDestroy(r.graphExec);
			r.graphExec = nullptr;
			r.graphKey.clear();
			WfTuning warm = tune;
			warm.alpha = I.scene.desc.hasAlpha != 0;
			prepare_batch_kernels(warm);
			cudaGraph_t g = nullptr;
			CHECK_CUDA(cudaStreamBeginCapture(I.stream, cudaStreamCaptureModeThreadLocal));
			const cudaError_t e = launch_pt_wavefront(I.scene.desc, r.params, rs, r.wf, r.counters, I.stream, &info, tune);
			const cudaError_t e2 = cudaStreamEndCapture(I.stream, &g);
			if(e != cudaSuccess || e2 != cudaSuccess) { if(g) cudaGraphDestroy(g); CHECK_CUDA(e); CHECK_CUDA(e2); }
			const cudaError_t e3 = cudaGraphInstantiate(&r.graphExec, g, 0);
			cudaGraphDestroy(g);
			CHECK_CUDA(e3);
			r.graphKey = key;
			r.graphLaunches = info.launches;
		}
		*r.hIteration = r.iteration;
		CHECK_CUDA(cudaMemcpyAsync(r.dIteration, r.hIteration, sizeof(int32_t), cudaMemcpyHostToDevice, I.stream));
		CHECK_CUDA(cudaEventRecord(r.evStart, I.stream));
		CHECK_CUDA(cudaGraphLaunch(r.graphExec, I.stream));
		info.launches = r.graphLaunches;
	} else {
		CHECK_CUDA(cudaEventRecord(r.evStart, I.stream));
		if(r.megakernel) CHECK_CUDA(launch_pt(I.scene.desc, r.params, rs, r.workCounter, r.counters, 0u, n, r.blocksPerSm, I.stream));
		else CHECK_CUDA(launch_pt_wavefront(I.scene.desc, r.params, rs, r.wf, r.counters, I.stream, &info, tune));
	}
	CHECK_CUDA(cudaEventRecord(r.evStop, I.stream));
	TraceCounters both[2];
	CHECK_CUDA(cudaMemcpyAsync(both, r.counters, 2 * sizeof(TraceCounters), cudaMemcpyDeviceToHost, I.stream));
	unsigned bounceQueue[WF_BOUNCE_STATS] = {};
	if(!r.megakernel)
		CHECK_CUDA(cudaMemcpyAsync(bounceQueue, r.wf.counters + WF_COUNTERS - WF_BOUNCE_STATS, sizeof(bounceQueue),
		                           cudaMemcpyDeviceToHost, I.stream));
	CHECK_CUDA(cudaStreamSynchronize(I.stream));
	if(!r.megakernel) {
		// next iteration's plan: the first bounce >= wavefrontBounces whose
		// extension queue held at most tailPaths paths (none: no tail)
		const int maxB = std::max(1, r.params.maxPathLength);
		int plan = maxB;
		for(int b = std::max(0, r.wavefrontBounces); b + 1 < maxB && b < int(WF_BOUNCE_STATS); ++b)
			if(bounceQueue[b] <= unsigned(std::max(0, r.tailPaths))) { plan = b; break; }
		r.plannedTail = plan;
		r.planKey = planKey;
	}
	CHECK_CUDA(cudaEventElapsedTime(&r.lastKernelMs, r.evStart, r.evStop));
	r.lastExtend = both[0];
	r.lastShadow = both[1];
	r.lastCounters = both[0];
	r.lastCounters.rays += both[1].rays; r.lastCounters.shadowRays += both[1].shadowRays;
	r.lastCounters.nodeVisits += both[1].nodeVisits; r.lastCounters.primTests += both[1].primTests;
	r.lastCounters.instanceVisits += both[1].instanceVisits; r.lastCounters.errors += both[1].errors;
	r.lastLaunches = r.megakernel ? 1 : info.launches;
	for(float& m : r.stageMs) m = 0.0f;
	for(int i = 0; i < info.pairsUsed; ++i) {
		float ms = 0.0f;
		CHECK_CUDA(cudaEventElapsedTime(&ms, info.events[2 * i], info.events[2 * i + 1]));
		r.stageMs[info.kinds[i]] += ms;
	}
	auto t2 = clk::now();
	auto us = [](clk::duration d) { return uint64_t(std::chrono::duration_cast<std::chrono::microseconds>(d).count()); };
	if(preTime) { preTime->cycles = 0; preTime->microseconds = us(t1 - t0); }
	if(iterTime) { iterTime->cycles = 0; iterTime->microseconds = us(t2 - t1); }
	if(postTime) { postTime->cycles = 0; postTime->microseconds = 0; }
	check_traversal(r.lastCounters.errors, I.scene.desc.maxSteps);
	return true;
	CATCH_ALL(false)
}

uint32_t render_get_current_iteration(ConstMufflonInstanceHdl h) {
	if(!h) return 0;
	const MufflonInstance& I = *static_cast<const MufflonInstance*>(h);
	return uint32_t(I.renderer.iteration + 1);
}
Boolean render_reset(MufflonInstanceHdl h) {
	TRY MufflonInstance& I = minst(h); std::lock_guard<std::recursive_mutex> lock(I.iterationMutex); I.renderer.needsReset = true; return true; CATCH_ALL(false)
}

// PFM screenshot of a target (render_save_screenshot, interface.cpp:3704)
Boolean render_save_screenshot(MufflonInstanceHdl h, const char* filename, const char* target, Boolean variance) {
	TRY
	MufflonInstance& I = minst(h);
	CHECK(filename && target, "filename and target are required");
	const float* px = nullptr;
	CHECK(mufflon_get_target_image(h, target, variance, &px), s_lastError);
	CHECK(px != nullptr, "no image yet");
	const int ch = I.renderer.screenChannels;
	FILE* f = std::fopen(filename, "wb");
	CHECK(f != nullptr, "cannot open output file");
	std::fprintf(f, "PF\n%u %u\n-1.0\n", I.renderer.width, I.renderer.height);
	for(size_t p = 0; p < size_t(I.renderer.width) * I.renderer.height; ++p) {
		float rgb[3] = { 0, 0, 0 };
		for(int c = 0; c < ch && c < 3; ++c) rgb[c] = px[p * ch + c];
		std::fwrite(rgb, sizeof(float), 3, f);
	}
	std::fclose(f);
	return true;
	CATCH_ALL(false)
}

static uint32_t target_count(int32_t kind) { return kind == 1 ? 3u : kind == 3 || kind == 4 ? 2u : kind == 2 ? 1u : 8u; }
uint32_t render_get_render_target_count(MufflonInstanceHdl h) { TRY return target_count(minst(h).renderer.kind); CATCH_ALL(0u) }
const char* render_get_render_target_name(MufflonInstanceHdl h, uint32_t index) {
	TRY
	const int32_t kind = minst(h).renderer.kind;
	CHECK(index < target_count(kind), "render target index out of bounds");
	return kind == 2 ? "Border" : kind != 0 ? LT_TARGETS[index] : TARGETS[index];
	CATCH_ALL(nullptr)
}
// The record / record-variance flags of a target implemented by the CUDA
// renderers (null for other names).
static std::pair<bool*, bool*> target_flags(RendererState& r, const char* name) {
	static const char* AUX_NAMES[5] = { "Position", "Depth", "Normal", "UV", "Albedo" };
	for(int a = 0; a < 5; ++a)
		if(!std::strcmp(name, AUX_NAMES[a])) return { &r.auxTarget[a], &r.auxVarOn[a] };
	if(!std::strcmp(name, "Radiance")) return { &r.targetRadiance, &r.varRadiance };
	if(!std::strcmp(name, "Hit ID")) return { &r.targetHitId, &r.varHitId };
	if(!std::strcmp(name, "Lightness")) return { &r.targetLightness, &r.varLightness };
	if(!std::strcmp(name, "Density")) return { &r.targetDensity, &r.varDensity };
	if(!std::strcmp(name, "Border")) return { &r.targetBorder, &r.varBorder };
	return { nullptr, nullptr };
}

// output_handler.hpp:391-431: enabling records the target and, with
// `variance`, its variance too; disabling with `variance` stops only the
// variance, without it both.
Boolean render_enable_render_target(MufflonInstanceHdl h, const char* target, Boolean variance) {
	TRY
	MufflonInstance& I = minst(h);
	std::lock_guard<std::recursive_mutex> lock(I.iterationMutex);
	CHECK(target, "target name is null");
	const auto f = target_flags(I.renderer, target);
	if(!f.first) throw ApiError(std::string("render target '") + target + "' is not produced by the CUDA renderers");
	*f.first = true;
	if(variance) *f.second = true;
	I.renderer.needsReset = true;
	return true;
	CATCH_ALL(false)
}
Boolean render_disable_render_target(MufflonInstanceHdl h, const char* target, Boolean variance) {
	TRY
	MufflonInstance& I = minst(h);
	std::lock_guard<std::recursive_mutex> lock(I.iterationMutex);
	CHECK(target, "target name is null");
	const auto f = target_flags(I.renderer, target);
	if(f.first) {
		*f.second = false;
		if(!variance) *f.first = false;
	}
	I.renderer.needsReset = true;
	return true;
	CATCH_ALL(false)
}
Boolean render_is_render_target_enabled(MufflonInstanceHdl h, const char* name, Boolean variance) {
	TRY
	MufflonInstance& I = minst(h);
	if(!name) return false;
	const auto f = target_flags(I.renderer, name);
	if(!f.first) return false;
	return variance ? *f.second : *f.first;
	CATCH_ALL(false)
}

uint32_t renderer_get_num_parameters(MufflonInstanceHdl h) {
	TRY
	const int32_t kind = minst(h).renderer.kind;
	if(kind == 2) return uint32_t(sizeof(WIRE_PARAMS) / sizeof(WIRE_PARAMS[0]));
	if(kind == 4) return uint32_t(sizeof(VCM_PARAMS) / sizeof(VCM_PARAMS[0]));
	return kind != 0 ? uint32_t(sizeof(LT_PARAMS) / sizeof(LT_PARAMS[0])) : uint32_t(sizeof(PT_PARAMS) / sizeof(PT_PARAMS[0]));
	CATCH_ALL(0u)
}
const char* renderer_get_parameter_desc(MufflonInstanceHdl h, uint32_t idx, ParameterType* type) {
	TRY
	const int32_t kind = minst(h).renderer.kind;
	const ParamDesc* table = kind == 2 ? WIRE_PARAMS : kind == 4 ? VCM_PARAMS : kind != 0 ? LT_PARAMS : PT_PARAMS;
	const size_t count = kind == 2 ? sizeof(WIRE_PARAMS) / sizeof(WIRE_PARAMS[0])
	                   : kind == 4 ? sizeof(VCM_PARAMS) / sizeof(VCM_PARAMS[0])
	                   : kind != 0 ? sizeof(LT_PARAMS) / sizeof(LT_PARAMS[0]) : sizeof(PT_PARAMS) / sizeof(PT_PARAMS[0]);
	CHECK(idx < count, "parameter index out of bounds");
	if(type) *type = table[idx].type;
	return table[idx].name;
	CATCH_ALL(nullptr)
}
Boolean renderer_set_parameter_int(MufflonInstanceHdl h, const char* name, int32_t value) {
	TRY
	MufflonInstance& I = minst(h);
	std::lock_guard<std::recursive_mutex> lock(I.iterationMutex);
	CHECK(name, "parameter name is null");
	int32_t* p = param_ptr(I.renderer, name);
	CHECK(p != nullptr, std::string("unknown parameter '") + name + "'");
	if(!std::strcmp(name, "NEE count")) CHECK(value >= 0, "NEE count must be non-negative");
	if(!std::strcmp(name, "Max. path length")) CHECK(value >= 1, "Max. path length must be at least 1");
	if(!std::strcmp(name, "Ray sort bits")) CHECK(value >= 0 && value <= WF_SORT_MAX_BITS, "Ray sort bits must be in 0..16");
	if(!std::strcmp(name, "Ray sort direction bits")) CHECK(value == 0 || value == 3 || value == 6, "Ray sort direction bits must be 0, 3 or 6");
	*p = value;
	I.renderer.needsReset = true; // ResetEvent::PARAMETER (renderer.hpp:19-48)
	return true;
	CATCH_ALL(false)
}
Boolean renderer_get_parameter_int(MufflonInstanceHdl h, const char* name, int32_t* value) {
	TRY
	MufflonInstance& I = minst(h);
	CHECK(name && value, "invalid arguments");
	int32_t* p = param_ptr(I.renderer, name);
	CHECK(p != nullptr, std::string("unknown parameter '") + name + "'");
	*value = *p;
	return true;
	CATCH_ALL(false)
}
Boolean renderer_set_parameter_float(MufflonInstanceHdl h, const char* name, float value) {
	TRY
	MufflonInstance& I = minst(h);
	std::lock_guard<std::recursive_mutex> lock(I.iterationMutex);
	CHECK(name, "parameter name is null");
	if(I.renderer.kind == 4 && !std::strcmp(name, "Relative merge radius")) {
		CHECK(value > 0.0f, "Relative merge radius must be positive");
		I.renderer.vcmMergeRadius = value;
		I.renderer.needsReset = true;
		return true;
	}
	CHECK(I.renderer.kind == 2 && !std::strcmp(name, "Line width"), std::string("unknown float parameter '") + name + "'");
	I.renderer.wireParams.lineWidth = value;
	I.renderer.needsReset = true;
	return true;
	CATCH_ALL(false)
}
Boolean renderer_get_parameter_float(MufflonInstanceHdl h, const char* name, float* value) {
	TRY
	MufflonInstance& I = minst(h);
	CHECK(name && value, "invalid arguments");
	if(I.renderer.kind == 4 && !std::strcmp(name, "Relative merge radius")) {
		*value = I.renderer.vcmMergeRadius;
		return true;
	}
	CHECK(I.renderer.kind == 2 && !std::strcmp(name, "Line width"), std::string("unknown float parameter '") + name + "'");
	*value = I.renderer.wireParams.lineWidth;
	return true;
	CATCH_ALL(false)
}
Boolean renderer_set_parameter_bool(MufflonInstanceHdl h, const char* name, Boolean value) {
	TRY
	MufflonInstance& I = minst(h);
	std::lock_guard<std::recursive_mutex> lock(I.iterationMutex);
	if(name && I.renderer.kind == 4 && !std::strcmp(name, "Progressive")) {
		I.renderer.vcmProgressive = value ? 1 : 0;
		I.renderer.needsReset = true;
		return true;
	}
	CHECK(name && !std::strcmp(name, "NEE position guide"), std::string("unknown bool parameter '") + (name ? name : "") + "'");
	CHECK(!value, "NEE position guide is not implemented by the CUDA path tracer");
	return true;
	CATCH_ALL(false)
}
Boolean renderer_get_parameter_bool(MufflonInstanceHdl h, const char* name, Boolean* value) {
	TRY
	MufflonInstance& I = minst(h);
	if(name && value && I.renderer.kind == 4 && !std::strcmp(name, "Progressive")) {
		*value = I.renderer.vcmProgressive ? 1 : 0;
		return true;
	}
	CHECK(name && !std::strcmp(name, "NEE position guide") && value, "unknown bool parameter");
	*value = 0;
	return true;
	CATCH_ALL(false)
}
Boolean renderer_set_parameter_enum(MufflonInstanceHdl h, const char* name, int) {
	TRY (void)minst(h); throw ApiError(std::string("unknown enum parameter '") + (name ? name : "") + "'"); CATCH_ALL(false)
}
Boolean renderer_get_parameter_enum(MufflonInstanceHdl h, const char* name, int*) {
	TRY (void)minst(h); throw ApiError(std::string("unknown enum parameter '") + (name ? name : "") + "'"); CATCH_ALL(false)
}

// ---------------------------------------------------------------- extensions
Boolean mufflon_get_render_stats(MufflonInstanceHdl h, MufflonRenderStats* s) {
	TRY
	MufflonInstance& I = minst(h);
	CHECK(s, "stats pointer is null");
	const TraceCounters& c = I.renderer.lastCounters;
	s->rays = c.rays; s->shadowRays = c.shadowRays; s->nodeVisits = c.nodeVisits; s->primTests = c.primTests;
	s->instanceVisits = c.instanceVisits; s->errors = c.errors; s->kernelMs = I.renderer.lastKernelMs;
	return true;
	CATCH_ALL(false)
}

Boolean mufflon_get_stage_stats(MufflonInstanceHdl h, MufflonStageStats* s) {
	TRY
	MufflonInstance& I = minst(h);
	CHECK(s, "stats pointer is null");
	const RendererState& r = I.renderer;
	const TraceCounters &e = r.lastExtend, &sh = r.lastShadow;
	s->extensionRays = e.rays; s->extendNodeVisits = e.nodeVisits; s->extendPrimTests = e.primTests;
	s->extendInstanceVisits = e.instanceVisits;
	s->shadowRays = sh.rays; s->shadowNodeVisits = sh.nodeVisits; s->shadowPrimTests = sh.primTests;
	s->shadowInstanceVisits = sh.instanceVisits;
	s->cameraMs = r.stageMs[WF_CAMERA]; s->extendMs = r.stageMs[WF_EXTEND]; s->tailMs = r.stageMs[WF_TAIL];
	s->shadeMs = r.stageMs[WF_SHADE]; s->finalizeMs = r.stageMs[WF_FINALIZE]; s->binMs = r.stageMs[WF_BIN];
	s->launches = uint32_t(r.lastLaunches);
	s->wavefront = r.megakernel ? 0u : 1u;
	return true;
	CATCH_ALL(false)
}

Boolean mufflon_get_lt_records(MufflonInstanceHdl h, int32_t* pixels, float* values, uint64_t slots) {
	TRY
	MufflonInstance& I = minst(h);
	std::lock_guard<std::recursive_mutex> lock(I.iterationMutex);
	const RendererState& r = I.renderer;
	CHECK((r.kind == 1 || r.kind == 3 || r.kind == 4) && r.ltRecSlots > 0 && r.iteration >= 0,
	      "no recorded light-tracer, bidirectional or vertex connection and merging iteration");
	CHECK(pixels && values && slots == r.ltRecSlots, "the record buffers must hold the renderer's number of slots");
	CHECK_CUDA(cudaMemcpyAsync(pixels, r.ltRecPixel, slots * sizeof(int32_t), cudaMemcpyDeviceToHost, I.stream));
	CHECK_CUDA(cudaMemcpyAsync(values, r.ltRecValue, r.ltRecFloats * sizeof(float), cudaMemcpyDeviceToHost, I.stream));
	CHECK_CUDA(cudaStreamSynchronize(I.stream));
	return true;
	CATCH_ALL(false)
}

// ---------------------------------------------------------------- batches
namespace {
// Grow-only device buffers of mufflon_render_batch (one batch at a time).
struct BatchState {
	std::mutex mutex;
	int device = -1;
	cudaStream_t stream = nullptr;
	void* wf = nullptr;
	size_t wfBytes = 0;
	void* buf = nullptr;
	size_t bufBytes = 0;
	DJob* dJobs = nullptr;
	size_t jobsCap = 0;
	std::vector<cudaEvent_t> events;
};
BatchState& batch_state() {
	static BatchState* b = new BatchState(); // lives until process exit
	return *b;
}
size_t align256(size_t b) { return (b + 255) / 256 * 256; }
} // namespace

Boolean mufflon_render_batch(const MufflonBatchJob* jobs, uint32_t count, int32_t useGraph, float* const* radiance,
                             float* const* hitId, float* jobDoneMs, MufflonBatchStats* stats) {
	TRY
	CHECK(jobs && count > 0 && count <= 65535, "a batch needs 1 to 65535 jobs");
	BatchState& B = batch_state();
	std::lock_guard<std::mutex> batchLock(B.mutex);
	// every instance used by the batch is locked (in address order) and loaded
	std::vector<MufflonInstance*> insts;
	for(uint32_t j = 0; j < count; ++j) insts.push_back(&minst(jobs[j].instance));
	std::vector<MufflonInstance*> uniq(insts);
	std::sort(uniq.begin(), uniq.end());
	uniq.erase(std::unique(uniq.begin(), uniq.end()), uniq.end());
	std::vector<std::unique_lock<std::recursive_mutex>> locks;
	for(MufflonInstance* I : uniq) locks.emplace_back(I->iterationMutex);
	const int dev = uniq[0]->device;
	for(MufflonInstance* I : uniq) {
		CHECK(I->device == dev, "all jobs of a batch must use instances on the same device");
		CHECK(I->current != nullptr, "a job's instance has no loaded scenario");
		load_scene_if_needed(*I);
	}
	CHECK_CUDA(cudaSetDevice(dev));
	if(B.device != dev) {
		CHECK(B.device < 0, "batches on more than one device per process are not supported");
		CHECK_CUDA(cudaStreamCreateWithFlags(&B.stream, cudaStreamNonBlocking));
		B.device = dev;
	}
	cudaStream_t st = B.stream;
	// host job table
	const int nee = jobs[0].neeCount > 0 ? jobs[0].neeCount : 1;
	std::vector<DJob> hj(count);
	uint64_t pixels = 0;
	int maxSpp = 0, maxBounces = 1;
	for(uint32_t j = 0; j < count; ++j) {
		const MufflonBatchJob& in = jobs[j];
		const MufflonInstance& I = *insts[j];
		const uint32_t w = in.width ? in.width : I.current->width;
		const uint32_t h = in.height ? in.height : I.current->height;
		CHECK(w > 0 && h > 0 && w <= 65535 && h <= 65535, "job resolution out of range");
		CHECK(in.spp >= 1, "a job needs at least one sample");
		CHECK(in.maxPathLength >= 1, "Max. path length must be at least 1");
		CHECK((in.neeCount > 0 ? in.neeCount : 1) == nee, "all jobs of a batch must use the same NEE count");
		DJob& d = hj[j];
		d.scene = I.scene.desc;
		d.sceneGroup = uint32_t(std::lower_bound(uniq.begin(), uniq.end(), insts[j]) - uniq.begin());
		d.scene.maxSteps = step_limit(I.renderer);
		d.scene.camera.resX = uint16_t(w);
		d.scene.camera.resY = uint16_t(h);
		d.params = PtParams{ in.seed, in.minPathLength, in.maxPathLength, nee, in.rrStartDepth };
		d.width = w; d.height = h; d.spp = in.spp;
		d.pixelOffset = uint32_t(pixels);
		pixels += uint64_t(w) * h;
		maxSpp = std::max(maxSpp, int(in.spp));
		maxBounces = std::max(maxBounces, int(in.maxPathLength));
	}
	CHECK(pixels < (1ull << 31), "a batch holds at most 2^31 - 1 pixels");
	const size_t n = size_t(pixels);
	// device buffers (grow-only)
	const size_t need = align256(n * 8) + align256(n * 2) + align256(n * 12) + align256(n * 8) + align256(2 * sizeof(TraceCounters));
	if(B.bufBytes < need) {
		if(B.buf) cudaFree(B.buf);
		B.buf = nullptr; B.bufBytes = 0;
		CHECK_CUDA(cudaMalloc(&B.buf, need));
		B.bufBytes = need;
	}
	const size_t wfNeed = wavefront_bytes(n, nee);
	if(B.wfBytes < wfNeed) {
		if(B.wf) cudaFree(B.wf);
		B.wf = nullptr; B.wfBytes = 0;
		CHECK_CUDA(cudaMalloc(&B.wf, wfNeed));
		B.wfBytes = wfNeed;
	}
	if(B.jobsCap < count) {
		if(B.dJobs) cudaFree(B.dJobs);
		B.dJobs = nullptr; B.jobsCap = 0;
		CHECK_CUDA(cudaMalloc(&B.dJobs, sizeof(DJob) * count));
		B.jobsCap = count;
	}
	char* m = static_cast<char*>(B.buf);
	auto take = [&](size_t b) { char* p = m; m += align256(b); return p; };
	uint64_t* rng = reinterpret_cast<uint64_t*>(take(n * 8));
	uint16_t* pathJob = reinterpret_cast<uint16_t*>(take(n * 2));
	float* rad = reinterpret_cast<float*>(take(n * 12));
	float* hit = reinterpret_cast<float*>(take(n * 8));
	TraceCounters* counters = reinterpret_cast<TraceCounters*>(take(2 * sizeof(TraceCounters)));
	WfState W{};
	wavefront_carve(B.wf, n, nee, W);
	W.rng = rng;
	std::vector<uint16_t> pj(n);
	for(uint32_t j = 0; j < count; ++j) {
		std::fill(pj.begin() + hj[j].pixelOffset, pj.begin() + hj[j].pixelOffset + size_t(hj[j].width) * hj[j].height, uint16_t(j));
		hj[j].radiance = rad + 3 * size_t(hj[j].pixelOffset);
		hj[j].hitId = hit + 2 * size_t(hj[j].pixelOffset);
	}
	CHECK_CUDA(cudaMemcpyAsync(pathJob, pj.data(), n * 2, cudaMemcpyHostToDevice, st));
	CHECK_CUDA(cudaMemcpyAsync(B.dJobs, hj.data(), sizeof(DJob) * count, cudaMemcpyHostToDevice, st));
	CHECK_CUDA(cudaMemsetAsync(rad, 0, n * 12, st));
	CHECK_CUDA(cudaMemsetAsync(hit, 0, n * 8, st));
	CHECK_CUDA(cudaMemsetAsync(counters, 0, 2 * sizeof(TraceCounters), st));
	for(uint32_t j = 0; j < count; ++j)
		CHECK_CUDA(launch_seed_rng(rng + hj[j].pixelOffset, hj[j].width * hj[j].height, hj[j].params.seed, st));
	const RendererState& r0 = uniq[0]->renderer;
	WfTuning tune;
	tune.traceBlocksPerSm = r0.traceBlocksPerSm;
	tune.wavefrontBounces = r0.wavefrontBounces;
	tune.refillLanes = r0.refillLanes;
	tune.tailPaths = r0.tailPaths;
	tune.sortBits = r0.sortBits;
	tune.sortDirBits = r0.sortDirBits;
	tune.counters = false;
	// binning keeps the rays of different scenes apart: the scene's index among the batch's instances
	while((size_t(1) << tune.sortGroupBits) < uniq.size()) ++tune.sortGroupBits;
	for(const auto* u : uniq) tune.alpha = tune.alpha || u->scene.desc.hasAlpha != 0;
	prepare_batch_kernels(tune);
	while(B.events.size() < size_t(maxSpp) + 1) {
		cudaEvent_t e;
		CHECK_CUDA(cudaEventCreate(&e));
		B.events.push_back(e);
	}
	CHECK_CUDA(cudaStreamSynchronize(st));
	uint32_t launches = 0;
	auto body = [&]() -> cudaError_t {
		for(int it = 0; it < maxSpp; ++it) {
			WfLaunchInfo info;
			const cudaError_t e = launch_pt_batch(B.dJobs, pathJob, uint32_t(n), it, maxBounces, nee, W, counters, st, tune, &info);
			if(e != cudaSuccess) return e;
			launches += uint32_t(info.launches);
			// inside a capture only an "external" record becomes a timing record of the graph
			const cudaError_t er = useGraph ? cudaEventRecordWithFlags(B.events[size_t(it) + 1], st, cudaEventRecordExternal)
			                                : cudaEventRecord(B.events[size_t(it) + 1], st);
			if(er != cudaSuccess) return er;
		}
		return cudaSuccess;
	};
	cudaGraph_t graph = nullptr;
	cudaGraphExec_t exec = nullptr;
	if(useGraph) {
		CHECK_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
		const cudaError_t e = body();
		const cudaError_t e2 = cudaStreamEndCapture(st, &graph);
		CHECK_CUDA(e);
		CHECK_CUDA(e2);
		CHECK_CUDA(cudaGraphInstantiate(&exec, graph, 0));
		CHECK_CUDA(cudaEventRecord(B.events[0], st));
		CHECK_CUDA(cudaGraphLaunch(exec, st));
	} else {
		CHECK_CUDA(cudaEventRecord(B.events[0], st));
		CHECK_CUDA(body());
	}
	const cudaError_t se = cudaStreamSynchronize(st);
	if(exec) cudaGraphExecDestroy(exec);
	if(graph) cudaGraphDestroy(graph);
	CHECK_CUDA(se);
	CHECK_CUDA(cudaGetLastError());
	{
		TraceCounters tc[2];
		CHECK_CUDA(cudaMemcpy(tc, counters, sizeof(tc), cudaMemcpyDeviceToHost));
		check_traversal(tc[0].errors + tc[1].errors, hj[0].scene.maxSteps);
	}
	if(jobDoneMs)
		for(uint32_t j = 0; j < count; ++j) {
			float ms = 0.0f;
			CHECK_CUDA(cudaEventElapsedTime(&ms, B.events[0], B.events[hj[j].spp]));
			jobDoneMs[j] = ms;
		}
	if(stats) {
		CHECK_CUDA(cudaEventElapsedTime(&stats->deviceMs, B.events[0], B.events[size_t(maxSpp)]));
		stats->launches = launches;
		stats->usedGraph = useGraph ? 1u : 0u;
		stats->pixels = uint32_t(n);
	}
	for(uint32_t j = 0; j < count; ++j) {
		const size_t np = size_t(hj[j].width) * hj[j].height;
		if(radiance && radiance[j]) CHECK_CUDA(cudaMemcpy(radiance[j], hj[j].radiance, np * 12, cudaMemcpyDeviceToHost));
		if(hitId && hitId[j]) CHECK_CUDA(cudaMemcpy(hitId[j], hj[j].hitId, np * 8, cudaMemcpyDeviceToHost));
	}
	return true;
	CATCH_ALL(false)
}

// ---------------------------------------------------------------- differentiable rendering
Boolean mufflon_texture_update(MufflonInstanceHdl h, TextureHdl texHdl, const float* rgba) {
	TRY
	MufflonInstance& I = minst(h);
	std::lock_guard<std::recursive_mutex> lock(I.iterationMutex);
	CHECK(texHdl && rgba, "texture and texel data are required");
	HostTexture* t = static_cast<HostTexture*>(texHdl);
	const size_t n = size_t(t->width) * t->height * 4;
	CHECK(t->texels.size() == n, "texture has no texel storage");
	std::copy(rgba, rgba + n, t->texels.begin());
	for(size_t k = 0; k < I.scene.textureSources.size(); ++k)
		if(I.scene.textureSources[k] == t && I.scene.valid)
			CHECK_CUDA(cudaMemcpyAsync(I.scene.textureBuffers[k], t->texels.data(), n * sizeof(float), cudaMemcpyHostToDevice, I.stream));
	CHECK_CUDA(cudaStreamSynchronize(I.stream));
	I.renderer.needsReset = true;
	return true;
	CATCH_ALL(false)
}

// The path-replay adjoint of the loaded scenario: spp samples of every pixel,
// replayed from generators seeded as for a reset render, differentiating an
// albedo texture (texIndex >= 0, gradient texGradOut of nt texels) and/or the
// emitted radiance of the material slots flagged in emitTarget (3 floats to
// emisGradOut).
static void run_adjoint(MufflonInstance& I, uint32_t spp, const float* imageGrad, int texIndex, size_t nt,
                        float* texGradOut, const std::vector<unsigned char>* emitTarget, float* emisGradOut,
                        float* deviceMs) {
	const RendererState& r = I.renderer;
	CHECK(r.params.maxPathLength <= ADJOINT_MAX_PATH, "the adjoint supports paths of at most 32 vertices");
	const uint32_t w = I.current->width, hgt = I.current->height;
	const size_t n = size_t(w) * hgt;
	DScene desc = I.scene.desc;
	desc.maxSteps = step_limit(r);
	desc.camera.resX = uint16_t(w);
	desc.camera.resY = uint16_t(hgt);
	uint64_t* rng = nullptr;
	float *dImg = nullptr, *dGrad = nullptr, *dEmis = nullptr;
	unsigned char* dTarget = nullptr;
	void* adjMem = nullptr;
	cudaEvent_t a = nullptr, b = nullptr;
	auto cleanup = [&]() {
		cudaFree(rng); cudaFree(dImg); cudaFree(dGrad); cudaFree(dEmis); cudaFree(dTarget); cudaFree(adjMem);
		if(a) cudaEventDestroy(a);
		if(b) cudaEventDestroy(b);
	};
	const bool wavefront = !r.megakernel;
	if(wavefront) {
		ensure_render_buffers(I);
		ensure_wavefront_buffers(I);
	}
	try {
		if(wavefront) CHECK_CUDA(cudaMalloc(&adjMem, adjoint_bytes(n, r.params.maxPathLength)));
		CHECK_CUDA(cudaMalloc(&rng, n * 8));
		CHECK_CUDA(cudaMalloc(&dImg, n * 12));
		AdjointTargets T;
		if(texIndex >= 0) {
			CHECK_CUDA(cudaMalloc(&dGrad, nt * 12));
			CHECK_CUDA(cudaMemsetAsync(dGrad, 0, nt * 12, I.stream));
			T.texIndex = texIndex;
			T.texGrad = dGrad;
		}
		if(emitTarget) {
			CHECK_CUDA(cudaMalloc(&dEmis, 12));
			CHECK_CUDA(cudaMalloc(&dTarget, emitTarget->size()));
			CHECK_CUDA(cudaMemsetAsync(dEmis, 0, 12, I.stream));
			CHECK_CUDA(cudaMemcpyAsync(dTarget, emitTarget->data(), emitTarget->size(), cudaMemcpyHostToDevice, I.stream));
			T.emitTarget = dTarget;
			T.emisGrad = dEmis;
		}
		CHECK_CUDA(cudaEventCreate(&a));
		CHECK_CUDA(cudaEventCreate(&b));
		CHECK_CUDA(cudaMemcpyAsync(dImg, imageGrad, n * 12, cudaMemcpyHostToDevice, I.stream));
		CHECK_CUDA(launch_seed_rng(rng, uint32_t(n), r.params.seed, I.stream));
		CHECK_CUDA(cudaEventRecord(a, I.stream));
		WfTuning tune;
		tune.traceBlocksPerSm = r.traceBlocksPerSm;
		tune.wavefrontBounces = r.wavefrontBounces;
		tune.refillLanes = r.refillLanes;
		tune.tailPaths = r.tailPaths;
		tune.sortBits = r.sortBits;
		tune.sortDirBits = r.sortDirBits;
		tune.counters = false;
		if(wavefront) CHECK_CUDA(cudaMemsetAsync(r.counters, 0, 2 * sizeof(TraceCounters), I.stream));
		for(uint32_t s = 0; s < spp; ++s) {
			if(wavefront)
				CHECK_CUDA(launch_adjoint_wavefront(desc, r.params, rng, w, hgt, r.wf, adjMem, r.params.maxPathLength, T,
				                                    dImg, 1.0f / float(spp), r.counters, I.stream, tune));
			else
				CHECK_CUDA(launch_adjoint_albedo(desc, r.params, rng, w, hgt, T, dImg, 1.0f / float(spp), I.stream));
		}
		CHECK_CUDA(cudaEventRecord(b, I.stream));
		if(texIndex >= 0) CHECK_CUDA(cudaMemcpyAsync(texGradOut, dGrad, nt * 12, cudaMemcpyDeviceToHost, I.stream));
		if(emitTarget) CHECK_CUDA(cudaMemcpyAsync(emisGradOut, dEmis, 12, cudaMemcpyDeviceToHost, I.stream));
		TraceCounters tc[2] = {};
		if(wavefront) CHECK_CUDA(cudaMemcpyAsync(tc, r.counters, sizeof(tc), cudaMemcpyDeviceToHost, I.stream));
		CHECK_CUDA(cudaStreamSynchronize(I.stream));
		if(deviceMs) CHECK_CUDA(cudaEventElapsedTime(deviceMs, a, b));
		check_traversal(tc[0].errors + tc[1].errors, desc.maxSteps);
	} catch(...) {
		cleanup();
		throw;
	}
	cleanup();
}

Boolean mufflon_albedo_gradient(MufflonInstanceHdl h, TextureHdl texHdl, uint32_t spp, const float* imageGrad,
                                float* textureGrad, float* deviceMs) {
	TRY
	MufflonInstance& I = minst(h);
	std::lock_guard<std::recursive_mutex> lock(I.iterationMutex);
	CHECK(texHdl && imageGrad && textureGrad && spp >= 1, "invalid arguments");
	CHECK(I.current != nullptr, "no scenario loaded");
	load_scene_if_needed(I);
	const RendererState& r = I.renderer;
	CHECK(r.params.rrStartDepth >= r.params.maxPathLength,
	      "the albedo adjoint needs Russian roulette off: RR start depth >= Max. path length");
	const HostTexture* t = static_cast<const HostTexture*>(texHdl);
	int texIndex = -1;
	for(size_t k = 0; k < I.scene.textureSources.size(); ++k)
		if(I.scene.textureSources[k] == t) texIndex = int(k);
	CHECK(texIndex >= 0, "the texture is not an albedo texture of the loaded scenario");
	run_adjoint(I, spp, imageGrad, texIndex, size_t(t->width) * t->height, textureGrad, nullptr, nullptr, deviceMs);
	return true;
	CATCH_ALL(false)
}

// dLoss/dL for the emitted radiance L = radiance x scale of an emissive
// material, over every material slot of the loaded scenario that uses it.
Boolean mufflon_emission_gradient(MufflonInstanceHdl h, MaterialHdl material, uint32_t spp, const float* imageGrad,
                                  float* radianceGrad, float* deviceMs) {
	TRY
	MufflonInstance& I = minst(h);
	std::lock_guard<std::recursive_mutex> lock(I.iterationMutex);
	CHECK(material && imageGrad && radianceGrad && spp >= 1, "invalid arguments");
	CHECK(I.current != nullptr, "no scenario loaded");
	const HostMaterial* m = static_cast<const HostMaterial*>(material);
	CHECK(m->type == MAT_EMISSIVE, "the material is not emissive");
	load_scene_if_needed(I);
	const auto& slots = I.current->slotMaterials;
	std::vector<unsigned char> target(std::max<size_t>(slots.size(), 1), 0);
	bool used = false;
	for(size_t k = 0; k < slots.size(); ++k)
		if(slots[k] == m) { target[k] = 1; used = true; }
	CHECK(used, "the material is not used by the loaded scenario");
	run_adjoint(I, spp, imageGrad, -1, 0, nullptr, &target, radianceGrad, deviceMs);
	return true;
	CATCH_ALL(false)
}

// Replaces the emitted radiance (radiance x scale) of an emissive material;
// the scene (its light list and tree, whose fluxes depend on it) is rebuilt
// before the next render.
Boolean mufflon_set_emitted_radiance(MufflonInstanceHdl h, MaterialHdl material, const float* rgb) {
	TRY
	MufflonInstance& I = minst(h);
	std::lock_guard<std::recursive_mutex> lock(I.iterationMutex);
	CHECK(material && rgb, "invalid arguments");
	HostMaterial* m = static_cast<HostMaterial*>(material);
	CHECK(m->type == MAT_EMISSIVE, "the material is not emissive");
	m->emissionOverride = true;
	for(int c = 0; c < 3; ++c) m->emission[c] = rgb[c];
	I.sceneDirty = true;
	I.renderer.needsReset = true;
	return true;
	CATCH_ALL(false)
}

Boolean mufflon_get_light_tree(MufflonInstanceHdl h, uint32_t* numLights, uint32_t* numNodes, uint32_t* numAreaLights,
                               void* lights, void* nodes, uint64_t* primKeys, uint32_t* primCodes, float* rootFlux) {
	TRY
	MufflonInstance& I = minst(h);
	std::lock_guard<std::recursive_mutex> lock(I.iterationMutex);
	load_scene_if_needed(I);
	const DeviceScene& D = I.scene;
	const uint32_t nArea = D.desc.numLightPrims;
	if(numLights) *numLights = D.numLights;
	if(numNodes) *numNodes = D.numLightNodes;
	if(numAreaLights) *numAreaLights = nArea;
	if(rootFlux) *rootFlux = D.desc.rootFlux;
	static_assert(sizeof(DLight) == 112 && sizeof(DLightNode) == 20, "light layouts");
	if(lights && D.numLights) CHECK_CUDA(cudaMemcpy(lights, D.dLights, sizeof(DLight) * D.numLights, cudaMemcpyDeviceToHost));
	if(nodes && D.numLightNodes) CHECK_CUDA(cudaMemcpy(nodes, D.dLightNodes, sizeof(DLightNode) * D.numLightNodes, cudaMemcpyDeviceToHost));
	if(primKeys && nArea) CHECK_CUDA(cudaMemcpy(primKeys, D.dLightKeys, sizeof(uint64_t) * nArea, cudaMemcpyDeviceToHost));
	if(primCodes && nArea) CHECK_CUDA(cudaMemcpy(primCodes, D.dLightCodes, sizeof(uint32_t) * nArea, cudaMemcpyDeviceToHost));
	return true;
	CATCH_ALL(false)
}

Boolean mufflon_get_load_stats(MufflonInstanceHdl h, MufflonLoadStats* s) {
	TRY
	MufflonInstance& I = minst(h);
	CHECK(s, "stats pointer is null");
	const DeviceScene& D = I.scene;
	s->totalMs = D.loadMs[0]; s->uploadMs = D.loadMs[1]; s->bvhMs = D.loadMs[2];
	s->instanceBvhMs = D.loadMs[3]; s->otherMs = D.loadMs[4];
	s->pad = 0;
	s->h2dBytes = D.loadH2dBytes;
	return true;
	CATCH_ALL(false)
}

Boolean mufflon_trace_rays(MufflonInstanceHdl h, const float* rays, const float* geo, float tmax, uint32_t n,
                           float* t, int32_t* inst, int32_t* prim, float* sp) {
	TRY
	MufflonInstance& I = minst(h);
	std::lock_guard<std::recursive_mutex> lock(I.iterationMutex);
	CHECK(rays && t && inst && prim, "invalid arguments");
	load_scene_if_needed(I);
	if(n == 0) return true;
	float *dr = nullptr, *dg = nullptr, *dt = nullptr, *dsp = nullptr;
	int32_t *di = nullptr, *dp = nullptr;
	CHECK_CUDA(cudaMalloc(&dr, size_t(n) * 24));
	CHECK_CUDA(cudaMalloc(&dt, size_t(n) * 4));
	CHECK_CUDA(cudaMalloc(&di, size_t(n) * 4));
	CHECK_CUDA(cudaMalloc(&dp, size_t(n) * 4));
	CHECK_CUDA(cudaMalloc(&dsp, size_t(n) * 8));
	if(geo) CHECK_CUDA(cudaMalloc(&dg, size_t(n) * 12));
	CHECK_CUDA(cudaMemcpyAsync(dr, rays, size_t(n) * 24, cudaMemcpyHostToDevice, I.stream));
	if(geo) CHECK_CUDA(cudaMemcpyAsync(dg, geo, size_t(n) * 12, cudaMemcpyHostToDevice, I.stream));
	if(I.renderer.megakernel) CHECK_CUDA(launch_trace_rays(I.scene.desc, dr, dg, tmax, n, dt, di, dp, dsp, I.stream));
	else CHECK_CUDA(launch_trace_rays_wide(I.scene.desc, dr, dg, tmax, n, dt, di, dp, dsp, I.stream));
	CHECK_CUDA(cudaMemcpyAsync(t, dt, size_t(n) * 4, cudaMemcpyDeviceToHost, I.stream));
	CHECK_CUDA(cudaMemcpyAsync(inst, di, size_t(n) * 4, cudaMemcpyDeviceToHost, I.stream));
	CHECK_CUDA(cudaMemcpyAsync(prim, dp, size_t(n) * 4, cudaMemcpyDeviceToHost, I.stream));
	if(sp) CHECK_CUDA(cudaMemcpyAsync(sp, dsp, size_t(n) * 8, cudaMemcpyDeviceToHost, I.stream));
	CHECK_CUDA(cudaStreamSynchronize(I.stream));
	cudaFree(dr); cudaFree(dg); cudaFree(dt); cudaFree(di); cudaFree(dp); cudaFree(dsp);
	return true;
	CATCH_ALL(false)
}

Boolean mufflon_trace_occlusion(MufflonInstanceHdl h, const float* a, const float* b, uint32_t n, uint8_t* occ) {
	TRY
	MufflonInstance& I = minst(h);
	std::lock_guard<std::recursive_mutex> lock(I.iterationMutex);
	CHECK(a && b && occ, "invalid arguments");
	load_scene_if_needed(I);
	if(n == 0) return true;
	float *da = nullptr, *db = nullptr;
	uint8_t* dout = nullptr;
	CHECK_CUDA(cudaMalloc(&da, size_t(n) * 12));
	CHECK_CUDA(cudaMalloc(&db, size_t(n) * 12));
	CHECK_CUDA(cudaMalloc(&dout, n));
	CHECK_CUDA(cudaMemcpyAsync(da, a, size_t(n) * 12, cudaMemcpyHostToDevice, I.stream));
	CHECK_CUDA(cudaMemcpyAsync(db, b, size_t(n) * 12, cudaMemcpyHostToDevice, I.stream));
	if(I.renderer.megakernel) CHECK_CUDA(launch_occlusion(I.scene.desc, da, db, n, dout, I.stream));
	else CHECK_CUDA(launch_occlusion_wide(I.scene.desc, da, db, n, dout, I.stream));
	CHECK_CUDA(cudaMemcpyAsync(occ, dout, n, cudaMemcpyDeviceToHost, I.stream));
	CHECK_CUDA(cudaStreamSynchronize(I.stream));
	cudaFree(da); cudaFree(db); cudaFree(dout);
	return true;
	CATCH_ALL(false)
}

Boolean mufflon_get_bvh(MufflonInstanceHdl h, int32_t which, int32_t* numPrims, int32_t* numInternal, void* nodes, int32_t* primIds) {
	TRY
	MufflonInstance& I = minst(h);
	std::lock_guard<std::recursive_mutex> lock(I.iterationMutex);
	load_scene_if_needed(I);
	const BvhBuffers* b = nullptr;
	if(which < 0) b = &I.scene.tlas;
	else { CHECK(size_t(which) < I.scene.lods.size(), "LoD index out of range"); b = &I.scene.lods[which].bvh; }
	if(numPrims) *numPrims = b->numPrims;
	if(numInternal) *numInternal = b->numInternal;
	if(nodes && b->numInternal > 0) CHECK_CUDA(cudaMemcpy(nodes, b->nodes, sizeof(BvhNode) * 2 * size_t(b->numInternal), cudaMemcpyDeviceToHost));
	if(primIds && b->numPrims > 0) CHECK_CUDA(cudaMemcpy(primIds, b->primIds, sizeof(int32_t) * size_t(b->numPrims), cudaMemcpyDeviceToHost));
	return true;
	CATCH_ALL(false)
}

Boolean mufflon_lbvh_build(const float* vertices, uint32_t numVertices, const uint32_t* indices, uint32_t numTriangles,
                           uint32_t numQuads, const float* spheres, uint32_t numSpheres, uint64_t* mortonSorted,
                           int32_t* parents, void* nodes, int32_t* primIds, int32_t* numInternal, float* stageMs) {
	return mufflon_lbvh_build_ex(vertices, numVertices, indices, numTriangles, numQuads, spheres, numSpheres, 63,
	                             mortonSorted, parents, nodes, primIds, numInternal, stageMs);
}

Boolean mufflon_lbvh_build_ex(const float* vertices, uint32_t numVertices, const uint32_t* indices, uint32_t numTriangles,
                              uint32_t numQuads, const float* spheres, uint32_t numSpheres, int32_t mortonBits,
                              uint64_t* mortonSorted, int32_t* parents, void* nodes, int32_t* primIds,
                              int32_t* numInternal, float* stageMs) {
	TRY
	CHECK(mufflon_is_cuda_available(), "no CUDA device");
	CHECK(mortonBits == 63 || mortonBits == 30, "Morton codes have 63 or 30 bits");
	HostLod L;
	L.vertices.assign(vertices, vertices + 3 * size_t(numVertices));
	L.triIdx.assign(indices, indices + 3 * size_t(numTriangles));
	L.quadIdx.assign(indices + 3 * size_t(numTriangles), indices + 3 * size_t(numTriangles) + 4 * size_t(numQuads));
	L.triMat.assign(numTriangles, 0); L.quadMat.assign(numQuads, 0);
	if(numSpheres) L.spheres.assign(spheres, spheres + 4 * size_t(numSpheres));
	L.sphereMat.assign(numSpheres, 0);
	const uint32_t n = numTriangles + numQuads + numSpheres;
	float *dv = nullptr; uint32_t* di = nullptr; float4* ds = nullptr;
	CHECK_CUDA(cudaMalloc(&dv, std::max<size_t>(1, L.vertices.size()) * 4));
	CHECK_CUDA(cudaMalloc(&di, std::max<size_t>(1, 3 * size_t(numTriangles) + 4 * size_t(numQuads)) * 4));
	CHECK_CUDA(cudaMalloc(&ds, std::max<size_t>(1, numSpheres) * 16));
	if(!L.vertices.empty()) CHECK_CUDA(cudaMemcpy(dv, L.vertices.data(), L.vertices.size() * 4, cudaMemcpyHostToDevice));
	if(numTriangles + numQuads) CHECK_CUDA(cudaMemcpy(di, indices, (3 * size_t(numTriangles) + 4 * size_t(numQuads)) * 4, cudaMemcpyHostToDevice));
	if(numSpheres) CHECK_CUDA(cudaMemcpy(ds, spheres, size_t(numSpheres) * 16, cudaMemcpyHostToDevice));
	LodBuildInput in{};
	in.numTriangles = numTriangles; in.numQuads = numQuads; in.numSpheres = numSpheres;
	in.vertices = dv; in.indices = di; in.spheres = ds;
	L.bounds(in.aabbMin, in.aabbMax);
	LbvhBuilder builder;
	builder.enable_timing(stageMs != nullptr);
	builder.set_morton_bits(mortonBits);
	BvhBuffers out;
	cudaStream_t s;
	CHECK_CUDA(cudaStreamCreate(&s));
	const cudaError_t e = builder.build_lod(in, out, s);
	if(e == cudaSuccess && n > 1) {
		if(mortonSorted) cudaMemcpy(mortonSorted, builder.sorted_keys(), sizeof(uint64_t) * n, cudaMemcpyDeviceToHost);
		if(parents) cudaMemcpy(parents, builder.parents(), sizeof(int32_t) * (2 * size_t(n) - 1), cudaMemcpyDeviceToHost);
	}
	if(e == cudaSuccess) {
		if(nodes && out.numInternal > 0) cudaMemcpy(nodes, out.nodes, sizeof(BvhNode) * 2 * size_t(out.numInternal), cudaMemcpyDeviceToHost);
		if(primIds && n > 0) cudaMemcpy(primIds, out.primIds, sizeof(int32_t) * n, cudaMemcpyDeviceToHost);
		if(numInternal) *numInternal = out.numInternal;
		if(stageMs) { const StageTimes t = builder.last_times(); const float v[9] = { t.morton, t.sort, t.emit, t.merge, t.mark, t.scan, t.compact, t.soup, t.wide }; std::memcpy(stageMs, v, sizeof(v)); }
	}
	out.release();
	cudaStreamDestroy(s);
	cudaFree(dv); cudaFree(di); cudaFree(ds);
	CHECK_CUDA(e);
	CHECK_CUDA(cudaGetLastError());
	return true;
	CATCH_ALL(false)
}

Boolean mufflon_lbvh_build_device(const float* dVertices, const uint32_t* dIndices, uint32_t numTriangles, uint32_t numQuads,
                                  const float* dSpheres, uint32_t numSpheres, const float* aabb6, int32_t* numInternal,
                                  float* buildMs, float* stageMs) {
	TRY
	CHECK(aabb6, "aabb is required");
	LodBuildInput in{};
	in.numTriangles = numTriangles; in.numQuads = numQuads; in.numSpheres = numSpheres;
	in.vertices = dVertices; in.indices = dIndices; in.spheres = reinterpret_cast<const float4*>(dSpheres);
	std::memcpy(in.aabbMin, aabb6, 12); std::memcpy(in.aabbMax, aabb6 + 3, 12);
	static LbvhBuilder* builder = new LbvhBuilder();
	static BvhBuffers* out = new BvhBuffers();
	builder->enable_timing(stageMs != nullptr);
	cudaEvent_t a, b;
	CHECK_CUDA(cudaEventCreate(&a)); CHECK_CUDA(cudaEventCreate(&b));
	CHECK_CUDA(cudaEventRecord(a, 0));
	CHECK_CUDA(builder->build_lod(in, *out, 0));
	CHECK_CUDA(cudaEventRecord(b, 0));
	CHECK_CUDA(cudaEventSynchronize(b));
	float ms = 0.0f;
	cudaEventElapsedTime(&ms, a, b);
	cudaEventDestroy(a); cudaEventDestroy(b);
	if(buildMs) *buildMs = ms;
	if(numInternal) *numInternal = out->numInternal;
	if(stageMs) { const StageTimes t = builder->last_times(); const float v[9] = { t.morton, t.sort, t.emit, t.merge, t.mark, t.scan, t.compact, t.soup, t.wide }; std::memcpy(stageMs, v, sizeof(v)); }
	return true;
	CATCH_ALL(false)
}

Boolean mufflon_measure_l2_bandwidth(uint64_t bytes, int32_t reps, float* gbs) {
	TRY
	CHECK(gbs && bytes >= (1u << 20) && reps > 0, "invalid arguments");
	CHECK_CUDA(measure_l2_bandwidth(size_t(bytes), reps, gbs));
	return true;
	CATCH_ALL(false)
}

// Allocation-free sort: launches and memsets only (sort_noalloc.cu).
static_assert(NOALLOC_MAX_PAIRS == MUFFLON_SORT_NOALLOC_MAX_PAIRS, "the public limit is the implementation's");
Boolean mufflon_sort_pairs_device_noalloc(uint64_t* keys, int32_t* values, uint32_t n, void* stream) {
	TRY
	CHECK(n <= NOALLOC_MAX_PAIRS, "n = " + std::to_string(n) + " exceeds the maximum of " +
	      std::to_string(NOALLOC_MAX_PAIRS) + " pairs of the allocation-free sort");
	CHECK(n == 0 || (keys && values), "keys and values must be device pointers");
	bool expired = false;
	const cudaError_t e = sort_pairs_noalloc(keys, values, n, static_cast<cudaStream_t>(stream), &expired);
	CHECK(!expired, "a bounded wait of the sort expired; the result is incomplete");
	CHECK_CUDA(e);
	return true;
	CATCH_ALL(false)
}

Boolean mufflon_sort_pairs(uint64_t* keys, int32_t* values, uint32_t n) {
	TRY
	CHECK(keys && values, "invalid arguments");
	if(n == 0) return true;
	LbvhBuilder builder;
	uint64_t* dk = nullptr; int32_t* dv = nullptr;
	CHECK_CUDA(cudaMalloc(&dk, size_t(n) * 8));
	CHECK_CUDA(cudaMalloc(&dv, size_t(n) * 4));
	CHECK_CUDA(cudaMemcpy(dk, keys, size_t(n) * 8, cudaMemcpyHostToDevice));
	CHECK_CUDA(cudaMemcpy(dv, values, size_t(n) * 4, cudaMemcpyHostToDevice));
	CHECK_CUDA(builder.sort_pairs(dk, dv, n, 0));
	CHECK_CUDA(cudaDeviceSynchronize());
	CHECK_CUDA(cudaMemcpy(keys, dk, size_t(n) * 8, cudaMemcpyDeviceToHost));
	CHECK_CUDA(cudaMemcpy(values, dv, size_t(n) * 4, cudaMemcpyDeviceToHost));
	cudaFree(dk); cudaFree(dv);
	return true;
	CATCH_ALL(false)
}

} // extern "C"
