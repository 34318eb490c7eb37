// Device state of the wavefront path tracer (see wavefront.cu).
#pragma once

#include <cuda_runtime.h>
#include "scene_types.hpp"

namespace mb {

// All arrays are sized for one path per pixel; queues are indexed by slot.
struct WfState {
	uint64_t* rng;        // per pixel (the renderer's generator state)
	float4* thrPdf;       // per path: throughput xyz, pdf of the sampled direction
	float4* rad;          // per path: radiance of this iteration
	float4* prevPos;      // per path: position of the vertex that sent its ray (scenes with sphere lights only)
	float2* hit0;         // per path: first hit (instance, primitive)
	int* qPath[2];        // extension queues (double buffered)
	float4* qOrg[2];      // ray origin (epsilon offset applied)
	float4* qDir[2];      // ray direction
	float4* qHit[2];      // t, instance bits, primitive bits, surface u
	float* qHitSpy[2];    // surface v
	int* sPath;           // shadow rays: neeCount consecutive slots per path
	float4* sOrg;         // origin, length (<= 0: empty slot)
	float4* sDir;         // direction
	float4* sContrib;     // contribution if unoccluded
	unsigned* counters;   // queue sizes and per-launch work counters (WF_COUNTERS)
	// Coherence binning of the rays a shade stage queues (see wavefront.cu):
	// the shade writes a key per queued extension ray and per shadow-ray
	// group and counts the keys; a scan and a scatter then build the order in
	// which the next trace launch takes them.
	unsigned* extKey;     // per extension-queue slot
	unsigned* shKey;      // per shadow-ray group
	unsigned* extOrder;   // trace order: the slot of the i-th extension ray
	unsigned* shOrder;    // trace order: the i-th shadow-ray group
	unsigned* binHist;    // 2 << WF_SORT_MAX_BITS key counts (extension, then shadow)
	unsigned* binCursor;  // 2 << WF_SORT_MAX_BITS scatter cursors
	int sortBits;         // key bits (0: no binning; at most WF_SORT_MAX_BITS)
	int sortDirBits;      // of those, direction bits: 0, 3 (octant) or 6 (octahedral 8 x 8)
	int sortGroupBits;    // of those, the top bits: the path's group (the scene of a batch job)
	int ordered;          // set for a trace launch whose queues were binned
	// The auxiliary targets of the path tracer (null: none recorded): per path
	// the footprint's m_a and the last vertex's guide weight, and the
	// iteration's AUX_CHANNELS values, channel-major with auxStride paths per channel.
	float2* guide;
	float* auxIter;
	uint32_t auxStride;
};
constexpr int WF_SORT_MAX_BITS = 16;

// Size of WfState::counters: queue sizes, flags and one work counter per
// persistent launch (two per bounce; longer paths recycle them), then the
// extension-queue length of each bounce (WF_BOUNCE_STATS entries at the end).
constexpr unsigned WF_COUNTERS = 4096;
constexpr unsigned WF_BOUNCE_STATS = 64;

// WF_EXTEND: the trace launches of the wavefront bounces (extension and
// shadow rays); WF_TAIL: the launch that finishes the remaining paths.
// WF_BIN: the scan and scatter launches that order queued rays by coherence.
enum WfStage { WF_CAMERA = 0, WF_EXTEND = 1, WF_TAIL = 2, WF_SHADE = 3, WF_FINALIZE = 4, WF_BIN = 5, WF_STAGES = 6 };

// Host-side launch record of one iteration. With `events` set, a pair of
// events is recorded around each stage launch (while capacity lasts) and
// `kinds` receives the stage of each pair.
struct WfLaunchInfo {
	cudaEvent_t* events = nullptr;
	unsigned char* kinds = nullptr;
	int eventPairs = 0;     // capacity in pairs
	int pairsUsed = 0;
	int launches = 0;       // kernel launches of the iteration
};

// One iteration (one sample per pixel) of the wavefront path tracer.
// counters[0] receives the extension rays' traversal counts, counters[1] the
// shadow rays'.
struct WfTuning {
	int traceBlocksPerSm = 6;  // register budget of the trace kernel: 4, 5, 6 or 8 resident blocks of 128 threads
	int wavefrontBounces = 2;  // bounces 0 .. this-1 always run as separate trace and shade launches; from
	                           // bounce this on, the first bounce with at most tailPaths queued paths
	                           // is finished by one launch that runs every remaining path in place
	int tailPaths = 98304;
	int tailBounce = -1;       // >= 0: planned schedule, the tail launch takes over at this bounce and
	                           // nothing is launched after it; -1: decided on the device per bounce
	int refillLanes = 32;      // idle lanes of a trace warp are refilled together once this many are idle (1..32)
	int sortBits = 0;          // coherence binning of the queued rays before each trace launch of bounce >= 1
	int sortDirBits = 3;       // (key bits in all, of them direction bits); 0 bits: trace in queue order
	int sortGroupBits = 0;     // extra key bits above those for the path's group (batches: the job's scene)
	bool counters = true;      // count node visits, primitive tests and instance entries (a slower kernel variant)
	bool alpha = false;        // batches: some job's scene has alpha textures (single renders take it from the scene)
};
cudaError_t launch_pt_wavefront(const DScene& scene, const PtParams& params, const RenderState& state, WfState W,
                                TraceCounters* counters, cudaStream_t stream, WfLaunchInfo* info,
                                const WfTuning& tuning = WfTuning());

// Closest hits and shadow-ray tests over the compressed 8-wide hierarchies
// (same arguments as launch_trace_rays / launch_occlusion of pt_api.hpp).
cudaError_t launch_trace_rays_wide(const DScene& scene, const float* rays, const float* geoNormals, float tmax,
                                  uint32_t n, float* t, int32_t* inst, int32_t* prim, float* sp, cudaStream_t stream);
cudaError_t launch_occlusion_wide(const DScene& scene, const float* a, const float* b, uint32_t n, uint8_t* out,
                                 cudaStream_t stream);

// Device memory of the wavefront state for n paths and nee shadow rays per
// path, and the carving of one allocation of that size into WfState.
size_t wavefront_bytes(size_t n, int nee);
void wavefront_carve(void* memory, size_t n, int nee, WfState& W);

// Resolves the trace and tail kernels' launch shapes (occupancy queries), so
// that a later stream capture does not have to.
void prepare_batch_kernels(const WfTuning& tuning);

// What a path-replay adjoint sample differentiates: an albedo texture
// (Lambert vertices that look it up; requires Russian roulette off) and/or
// the emitted radiance (radiance x scale) of flagged emissive material slots.
// Both gradients are accumulated: texGrad w * h * 3 floats, emisGrad 3 floats.
struct AdjointTargets {
	int texIndex = -1;                         // -1: no albedo gradient
	float* texGrad = nullptr;
	const unsigned char* emitTarget = nullptr; // per material slot, 1: differentiate; null: no emission gradient
	float* emisGrad = nullptr;
};

// One sample of the path-replay adjoint for every pixel: adds
// scale * dL/dI(p) * d(sample radiance)/d(parameter) to the targets'
// gradients. `rng` is the replay's per-pixel generator state, seeded as for
// a reset render and advanced one sample per launch.
constexpr int ADJOINT_MAX_PATH = 32;
cudaError_t launch_adjoint_albedo(const DScene& scene, const PtParams& params, uint64_t* rng, uint32_t width,
                                  uint32_t height, const AdjointTargets& targets, const float* imageGrad, float scale,
                                  cudaStream_t stream);

// The same adjoint sample through the wavefront kernels (one sample for
// every pixel per call): `adjointMemory` holds adjoint_bytes(width * height,
// maxEntries) bytes of per-path bookkeeping, maxEntries >= the max path length.
size_t adjoint_bytes(size_t numPaths, int maxEntries);
cudaError_t launch_adjoint_wavefront(const DScene& scene, const PtParams& params, uint64_t* rng, uint32_t width,
                                     uint32_t height, WfState W, void* adjointMemory, int maxEntries,
                                     const AdjointTargets& targets, const float* imageGrad, float scale,
                                     TraceCounters* counters, cudaStream_t stream, const WfTuning& tuning);

// One job of a batch: its scene (a loaded scene of some library instance),
// path-tracer parameters, resolution, sample count, its pixels' place in the
// batch's global pixel range, and its cumulative images.
struct DJob {
	DScene scene;
	PtParams params;
	uint32_t width, height, pixelOffset, spp;
	float* radiance;  // width * height * 3, cumulative mean
	float* hitId;     // width * height * 2, or null
	uint32_t sceneGroup; // jobs that render the same loaded scene share it (ray binning)
};

// One iteration (sample) of every job with spp > iteration, all jobs' paths
// in the same queues. pathJob[g] is the job of global pixel g; W.rng holds
// every global pixel's generator. neeCount must be the same for all jobs;
// maxBounces is the largest max path length of the batch.
cudaError_t launch_pt_batch(const DJob* jobs, const uint16_t* pathJob, uint32_t numPixels, int iteration,
                            int maxBounces, int neeCount, WfState W, TraceCounters* counters, cudaStream_t stream,
                            const WfTuning& tuning, WfLaunchInfo* info);

} // namespace mb
