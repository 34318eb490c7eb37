// Wavefront path tracer: pt_sample (src/core/renderer/pt/pt_common.hpp:75-156)
// split into stage kernels that run once per bounce over queues in HBM.
//
//   camera   one thread per pixel: consume the camera's and the first walk's
//            random numbers, write the primary ray into queue 0;
//   extend   persistent warps pull 32 rays at a time from the current queue
//            (one atomic per warp) and run closest-hit traversal only;
//   shadow   persistent warps pull shadow-ray groups, run any-hit traversal
//            and add the visible next-event contributions to the path's sum;
//   shade    one thread per queued path: hit attributes, emission with MIS,
//            then (if the path continues) next-event estimation, which
//            appends shadow rays, and the BSDF sample, Russian roulette and
//            the next ray, appended to the other queue;
//   finalize one thread per pixel: running mean of the iteration's result.
//
// Each kernel is small and does one kind of work, so it keeps its lanes
// converged, stays in the instruction cache and needs few registers. The
// per-path order of random numbers and of radiance additions is the one of
// pt_sample: the shadow kernel of bounce k runs after shade k and before
// shade k+1, so a next-event contribution is added between the emission terms
// that surround it, exactly as the sequential loop adds them.
#include "accumulate.cuh"
#include "aux_targets.cuh"
#include "shading.cuh"
#include "wide_traverse.cuh"
#include "wavefront.hpp"

#include <algorithm>
#include <cooperative_groups.h>

namespace mb {
namespace {

// counters: queue sizes, the shadow-slot count, the "paths handed to the tail"
// flag, then one work counter per persistent launch
enum { C_QUEUE0 = 0, C_QUEUE1 = 1, C_SHADOW0 = 2, C_SHADOW1 = 3, C_TAILED = 4, C_WORK = 5 };
// Threads per block of the trace and tail kernels (their shared-memory stacks are sized for it).
constexpr uint32_t WF_BLOCK = 128;
// Shade of bounce b appends its next rays to queue (b + 1) & 1 and its shadow
// rays to shadow counter C_SHADOW0 + (b & 1); the trace launch of bounce b
// reads queue b & 1 and shadow counter C_SHADOW0 + ((b - 1) & 1) and resets
// the two counters that the following shade fills.

MBD float nan_to_zero(float x) { return isnan(x) ? 0.0f : x; }
MBD f3 contribute(f3 acc, f3 c) {
	return make3(acc.x + nan_to_zero(c.x), acc.y + nan_to_zero(c.y), acc.z + nan_to_zero(c.z));
}
MBD f3 incident_direction(f3 e) {
	float t = 1.0f - e.x * e.x - e.y * e.y;
	t = fminf(fmaxf(t, 0.0f), 1.0f);
	return make3(e.x, e.y, sgn(e.z) * sqrt_(t));
}
MBD float4 pack(f3 v, float w) { return make_float4(v.x, v.y, v.z, w); }

// One atomic per group of converged lanes that each ask for `want` items.
MBD unsigned warp_reserve(unsigned* counter, unsigned want) {
	namespace cg = cooperative_groups;
	cg::coalesced_group g = cg::coalesced_threads();
	unsigned base = 0;
	if(g.thread_rank() == 0) base = atomicAdd(counter, g.size() * want);
	base = g.shfl(base, 0);
	return base + g.thread_rank() * want;
}

// ---------------------------------------------------------------- ray binning
// Rays queued by a shade stage are traced in an order that groups similar
// rays: the shade gives every extension ray and every shadow-ray group a key
// (direction cell above the Morton code of the origin's cell in the scene
// box) and counts the keys; k_bin_scan turns the counts into bin offsets and
// k_bin_scatter writes each ray's slot at its bin's next position. A warp of
// the next trace launch then takes 32 rays of one or a few bins: similar
// origins and directions, so similar node visits and step counts. Only the
// order changes; each ray's result is written to its own slot, and a
// closest hit does not depend on when the ray is traced.

// Octahedral cell (3 bits per coordinate) of a unit direction.
MBD unsigned octa_cell(f3 d) {
	const float s = fabsf(d.x) + fabsf(d.y) + fabsf(d.z);
	float u = __fdividef(d.x, s), v = __fdividef(d.y, s);
	if(d.z < 0.0f) {
		const float uu = (1.0f - fabsf(v)) * (u < 0.0f ? -1.0f : 1.0f);
		v = (1.0f - fabsf(u)) * (v < 0.0f ? -1.0f : 1.0f);
		u = uu;
	}
	const unsigned cu = min(7u, unsigned(fmaxf(0.0f, (u + 1.0f) * 4.0f)));
	const unsigned cv = min(7u, unsigned(fmaxf(0.0f, (v + 1.0f) * 4.0f)));
	return cu << 3 | cv;
}

// Coherence key of a ray: its group (W.sortGroupBits: the scene of a batch
// job) above W.sortDirBits of direction above a Morton code of the origin's
// cell in the scene box with the remaining bits (x gets the extra bit when
// they do not divide by three, then y).
MBD unsigned ray_key(const WfState& W, const DScene& S, unsigned group, f3 o, f3 d) {
	const int mb = W.sortBits - W.sortGroupBits - W.sortDirBits;
	const int bb[3] = { (mb + 2) / 3, (mb + 1) / 3, mb / 3 };
	const float oc[3] = { o.x, o.y, o.z };
	unsigned cell[3];
	for(int a = 0; a < 3; ++a) {
		const float ext = S.aabbMax[a] - S.aabbMin[a];
		const float f = ext > 0.0f ? __fdividef(oc[a] - S.aabbMin[a], ext) : 0.0f;
		const unsigned cells = 1u << bb[a];
		cell[a] = min(cells - 1u, unsigned(fmaxf(0.0f, f * float(cells))));
	}
	unsigned key = 0;
	for(int level = bb[0] - 1; level >= 0; --level)
		for(int a = 0; a < 3; ++a)
			if(level < bb[a]) key = key << 1 | ((cell[a] >> level) & 1u);
	unsigned dir = 0;
	if(W.sortDirBits == 3) dir = (d.x < 0.0f ? 4u : 0u) | (d.y < 0.0f ? 2u : 0u) | (d.z < 0.0f ? 1u : 0u);
	else if(W.sortDirBits == 6) dir = octa_cell(d);
	return (group << (W.sortBits - W.sortGroupBits)) | dir << mb | key;
}

// Records `key` for entry i and counts it (one atomic per key per warp).
MBD void bin_append(unsigned* keys, unsigned* hist, unsigned i, unsigned key) {
	keys[i] = key;
	const unsigned peers = __match_any_sync(__activemask(), key);
	if((threadIdx.x & 31u) == unsigned(__ffs(int(peers)) - 1)) atomicAdd(hist + key, unsigned(__popc(peers)));
}

// Exclusive offsets of the extension bins (block 0) and the shadow bins
// (block 1), 1 << bits each; the counts are cleared for the next shade.
__global__ void __launch_bounds__(1024) k_bin_scan(unsigned* hist, unsigned* cursor, int bits) {
	__shared__ unsigned part[1024];
	const unsigned nb = 1u << bits;
	unsigned* h = hist + blockIdx.x * nb;
	unsigned* c = cursor + blockIdx.x * nb;
	const unsigned per = (nb + 1023u) / 1024u;
	const unsigned t = threadIdx.x, b0 = t * per;
	unsigned sum = 0;
	for(unsigned k = 0; k < per && b0 + k < nb; ++k) sum += h[b0 + k];
	part[t] = sum;
	__syncthreads();
	for(unsigned off = 1; off < 1024u; off <<= 1) {
		const unsigned v = t >= off ? part[t - off] : 0u;
		__syncthreads();
		part[t] += v;
		__syncthreads();
	}
	unsigned run = part[t] - sum;
	for(unsigned k = 0; k < per && b0 + k < nb; ++k) {
		const unsigned x = h[b0 + k];
		c[b0 + k] = run;
		run += x;
		h[b0 + k] = 0u;
	}
}

// Writes the trace order of the queues the last shade filled: extension
// queue qNext and the shadow groups of shadow counter C_SHADOW0 + (qNext ^ 1).
__global__ void k_bin_scatter(WfState W, int qNext, int neeCount, unsigned capacity) {
	const unsigned nb = 1u << W.sortBits;
	const unsigned nExt = W.counters[qNext];
	const unsigned nGroups = W.counters[C_SHADOW0 + (qNext ^ 1)] / unsigned(neeCount);
	const unsigned lane = threadIdx.x & 31u;
	for(unsigned i0 = blockIdx.x * blockDim.x; i0 < nExt + nGroups; i0 += gridDim.x * blockDim.x) {
		const unsigned i = i0 + threadIdx.x;
		const bool ext = i < nExt;
		const bool valid = i < nExt + nGroups;
		const unsigned key = !valid ? 0xFFFFFFFFu : ext ? W.extKey[i] : nb + W.shKey[i - nExt];
		const unsigned peers = __match_any_sync(0xffffffffu, key);
		const int leader = __ffs(int(peers)) - 1;
		unsigned base = 0;
		if(valid && int(lane) == leader) base = atomicAdd(W.binCursor + key, unsigned(__popc(peers)));
		base = __shfl_sync(0xffffffffu, base, leader);
		if(!valid) continue;
		const unsigned pos = base + unsigned(__popc(peers & ((1u << lane) - 1u)));
		if(pos >= capacity) continue; // unreachable while the counts match the queues
		if(ext) W.extOrder[pos] = i;
		else W.shOrder[pos] = i - nExt;
	}
}

// Where a path's scene and path-tracer parameters come from: the kernel
// argument for a plain render, or the device job table of a batch, whose jobs
// share the queues (path p belongs to job pathJob[p]).
struct OneScene {
	static constexpr bool adjoint = false;
	DScene S;
	PtParams P;
	MBD const DScene& scene(int) const { return S; }
	MBD const PtParams& params(int) const { return P; }
	MBD unsigned group(int) const { return 0u; } // binning group of a path's rays
};

// Per-path bookkeeping of the albedo adjoint (path replay through the
// wavefront kernels): for every Lambert vertex that looked up albedo texture
// texIndex, its texel and albedo and the sum of the radiance terms added
// after it. Entry k of path p lives at k * numPaths + p.
//
// The same replay gives the derivative with respect to the emitted radiance
// L (radiance x scale) of the emissive materials flagged in emitTarget: each
// term such a material emits (an emitter hit, or a next-event sample of one
// of its area lights) is linear in L, so it adds term / L to the path's
// emisAcc, which k_adjoint_scatter weights by dL/dI and sums.
struct AdjointState {
	int texIndex;      // albedo texture, or -1: no albedo gradient
	uint32_t numPaths, maxEntries;
	DTexture tex;
	int* count;        // entries per path
	float4* entry;     // albedo xyz, texel index bits in w
	float4* suffix;    // suffix sum xyz
	const float* imageGrad;
	float scale;
	float* texGrad;
	const unsigned char* emitTarget; // per material slot: 1 if its emission is differentiated; null: none
	float4* emisAcc;   // per path: sum of term / L over the target's terms
	float* emisGrad;   // 3 floats: dLoss/dL
};
MBD void adjoint_add(const AdjointState& A, int p, f3 c) {
	const int n = A.count[p];
	for(int k = 0; k < n; ++k) {
		float4& s = A.suffix[size_t(k) * A.numPaths + p];
		s.x += c.x; s.y += c.y; s.z += c.z;
	}
}
// A term c emitted by material slot `mat` (-1: not an emissive material).
MBD void adjoint_emitted(const AdjointState& A, const DScene& S, int p, f3 c, int mat) {
	if(!A.emitTarget || mat < 0 || !__ldg(A.emitTarget + mat)) return;
	const f3 L = load3(S.materials[mat].radiance);
	float4& a = A.emisAcc[p];
	if(L.x > 0.0f) a.x += __fdiv_rn(c.x, L.x);
	if(L.y > 0.0f) a.y += __fdiv_rn(c.y, L.y);
	if(L.z > 0.0f) a.z += __fdiv_rn(c.z, L.z);
}
struct VertexInfo;
MBD void adjoint_vertex(const AdjointState& A, const DScene& S, int p, f3 e, bool surface, int type, int mat, f2 uv,
                        f3 albedo);

// A plain render whose paths also keep the adjoint's bookkeeping.
struct OneSceneAdjoint {
	static constexpr bool adjoint = true;
	DScene S;
	PtParams P;
	AdjointState A;
	MBD const DScene& scene(int) const { return S; }
	MBD const PtParams& params(int) const { return P; }
	MBD unsigned group(int) const { return 0u; }
};
struct JobScenes {
	static constexpr bool adjoint = false;
	const DJob* jobs;
	const uint16_t* pathJob;
	MBD const DScene& scene(int p) const { return jobs[pathJob[p]].scene; }
	MBD const PtParams& params(int p) const { return jobs[pathJob[p]].params; }
	// rays of jobs on the same scene are binned together, apart from other scenes'
	MBD unsigned group(int p) const { return jobs[pathJob[p]].sceneGroup; }
};

// Primary ray of one path (pinhole_ray, the camera's and the first walk's
// random numbers, Russian roulette at path length 0).
MBD void camera_path(const DScene& S, const PtParams& P, WfState& W, uint32_t p, int px, int py) {
	u64 rng = W.rng[p];
	(void)pcg_next(rng); // create_camera
	const u64 x0 = pcg_next(rng);
	(void)pcg_next(rng);
	const float rr = sample_uniform(uint32_t(pcg_next(rng)));
	const float ru0 = sample_uniform(uint32_t(x0)), ru1 = sample_uniform(uint32_t(x0 >> 32));
	float pdfF;
	const f3 dir = pinhole_ray(S.camera, px, py, ru0, ru1, pdfF);
	f3 thr = make3(1.0f, 1.0f, 1.0f);
	bool alive = true;
	if(0 >= P.rrStartDepth) {
		const float cp = fmin_(maxc(thr) + 0.1f, 1.0f);
		if(rr >= cp) alive = false;
		else thr = thr / cp;
	}
	W.rng[p] = rng;
	W.rad[p] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
	W.hit0[p] = make_float2(-1.0f, -1.0f);
	W.thrPdf[p] = pack(thr, pdfF);
	if(W.auxIter) {
		W.guide[p] = make_float2(0.0f, 1.0f); // the camera vertex's footprint (pChoice 1)
		for(int c = 0; c < AUX_CHANNELS; ++c) W.auxIter[size_t(c) * W.auxStride + p] = 0.0f;
	}
	if(!alive) return;
	f3 o = lv(S.camera.position);
	if(S.sphereLights) W.prevPos[p] = pack(o, 0.0f);
	add_epsilon(o, dir, make3(0.0f, 0.0f, 0.0f));
	const unsigned slot = warp_reserve(W.counters + C_QUEUE0, 1u);
	W.qPath[0][slot] = int(p);
	W.qOrg[0][slot] = pack(o, 0.0f);
	W.qDir[0][slot] = pack(dir, 0.0f);
}

// Camera stage of a batch: global pixel g of job pathJob[g]; pixels of jobs
// whose samples are all taken stay idle.
__global__ void k_camera_batch(const DJob* jobs, WfState W, const uint16_t* pathJob, uint32_t numPixels, int iteration) {
	const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
	if(g >= numPixels) return;
	const DJob& J = jobs[pathJob[g]];
	if(iteration >= int(J.spp)) return;
	const uint32_t local = g - J.pixelOffset;
	camera_path(J.scene, J.params, W, g, int(local % J.width), int(local / J.width));
}

__global__ void k_camera(const DScene S, const PtParams P, WfState W, uint32_t numPixels, uint32_t width) {
	const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
	if(p >= numPixels) return;
	camera_path(S, P, W, p, int(p % width), int(p / width));
}

// Block-wide traversal statistics in shared memory, one set per ray kind.
struct BlockStats { unsigned long long v[2][6]; };
template < class C >
MBD void stats_add(BlockStats& b, int kind, const C& c) {
	if(c.nodes) atomicAdd(&b.v[kind][0], (unsigned long long)c.nodes);
	if(c.prims) atomicAdd(&b.v[kind][1], (unsigned long long)c.prims);
	if(c.instances) atomicAdd(&b.v[kind][2], (unsigned long long)c.instances);
	atomicAdd(&b.v[kind][3], 1ull);
	if(c.errors) atomicAdd(&b.v[kind][5], (unsigned long long)c.errors);
}

// Persistent traversal of one bounce: the extension rays of queue q (closest
// hit) and the shadow-ray groups written by the previous shade (any hit; one
// lane runs a path's neeCount rays in order and adds the unoccluded
// contributions in that order). Idle lanes fetch work items with one atomic
// per warp once at least `refillLanes` of them are idle (or none is busy);
// with 32 a warp takes 32 new rays whenever all of its rays are finished,
// which measured fastest: the ray set-up then runs with all lanes at once.
// Every loop iteration runs one traversal step in every busy lane.
// Queue entries are read and written with streaming (evict-first) accesses so
// that they do not displace the hierarchies from L2.
template < int MINB, class SP, class C, int AM >
__global__ void __launch_bounds__(128, MINB) k_trace(const SP sp, WfState W, int q, int neeCount, int workIdx,
                                                     TraceCounters* counters, int refillLanes, int bounce) {
	__shared__ BlockStats stats;
	if(threadIdx.x < 12) (&stats.v[0][0])[threadIdx.x] = 0ull;
	__syncthreads();
	if(*reinterpret_cast<volatile unsigned*>(W.counters + C_TAILED)) return; // the tail launch finished the paths
	if(blockIdx.x == 0 && threadIdx.x == 0) {
		W.counters[q ^ 1] = 0u;           // filled by this bounce's shade
		W.counters[C_SHADOW0 + q] = 0u;
		if(bounce < int(WF_BOUNCE_STATS)) W.counters[WF_COUNTERS - WF_BOUNCE_STATS + bounce] = W.counters[q];
	}
	LocalStack stack;
	C cnt;
	const unsigned nExt = *reinterpret_cast<volatile unsigned*>(W.counters + q);
	const unsigned nGroups = *reinterpret_cast<volatile unsigned*>(W.counters + C_SHADOW0 + (q ^ 1)) / unsigned(neeCount);
	const unsigned total = nExt + nGroups;
	WideTracerT<AM> t;
	bool active = false, exhausted = false;
	unsigned item = 0;
	unsigned ent = 0;      // the item's extension-queue slot or shadow-ray group
	int path = 0, ray = 0; // path of the current item
	f3 radiance = make3(0.0f, 0.0f, 0.0f);
	float radW = 0.0f;
	const unsigned lane = threadIdx.x & 31u;
	for(;;) {
		bool seek = false; // look for the next shadow ray of the current group
		// Refill idle lanes together once enough of them are idle (or none is
		// busy), so that ray set-up runs with many lanes at a time.
		const unsigned busy = __ballot_sync(0xffffffffu, active);
		const unsigned idle = __ballot_sync(0xffffffffu, !active && !exhausted);
		if(idle && (__popc(idle) >= refillLanes || !busy)) {
			// One atomic per refill: the items a warp takes at a time are the
			// next ones of the queue. (Taking larger chunks per warp, to refill
			// lanes one by one without the atomic, measured 12-100 % slower:
			// the warps of an SM then trace rays from a wider window of the
			// queue and share fewer hierarchy nodes in L1.)
			unsigned base = 0;
			if(lane == unsigned(__ffs(int(idle)) - 1)) base = atomicAdd(W.counters + C_WORK + workIdx, unsigned(__popc(idle)));
			base = __shfl_sync(0xffffffffu, base, __ffs(int(idle)) - 1);
			if(idle & (1u << lane)) {
				item = base + unsigned(__popc(idle & ((1u << lane) - 1u)));
				if(item >= total) {
					exhausted = true;
				} else if(item < nExt) {
					ent = W.ordered ? __ldcs(W.extOrder + item) : item;
					const float4 o = __ldcs(W.qOrg[q] + ent), d = __ldcs(W.qDir[q] + ent);
					path = W.qPath[q][ent];
					cnt = C();
					t.init(sp.scene(path), f4to3(o), f4to3(d), MAX_SCENE_SIZE, false, cnt);
					active = true;
				} else {
					ent = W.ordered ? __ldcs(W.shOrder + (item - nExt)) : item - nExt;
					path = __ldcs(W.sPath + ent * unsigned(neeCount));
					const float4 acc = W.rad[path];
					radiance = f4to3(acc);
					radW = acc.w;
					ray = 0;
					seek = true;
				}
			}
		}
		if(__all_sync(0xffffffffu, exhausted)) break;
		if(active && t.step(sp.scene(path), cnt, stack)) {
			if(item < nExt) {
				stats_add(stats, 0, cnt);
				const HitRec& h = t.best;
				__stcs(W.qHit[q] + ent, make_float4(h.t, __int_as_float(h.has ? h.inst : -1), __int_as_float(h.has ? h.prim : -1), h.sp.x));
				__stcs(W.qHitSpy[q] + ent, h.sp.y);
				active = false;
			} else {
				stats_add(stats, 1, cnt);
				const unsigned slot = ent * unsigned(neeCount) + unsigned(ray);
				if(!t.occluded) {
					const float4 c4 = __ldcs(W.sContrib + slot);
					const f3 c = f4to3(c4);
					radiance = contribute(radiance, c);
					if(W.auxIter) {
						float* a = W.auxIter + size_t(AUX_LIGHT) * W.auxStride + size_t(path);
						*a = *a + nan_to_zero(__ldcs(W.sDir + slot).w);
					}
					if constexpr(SP::adjoint) {
						const f3 cc = contribute(make3(0.0f, 0.0f, 0.0f), c);
						adjoint_add(sp.A, path, cc);
						adjoint_emitted(sp.A, sp.scene(path), path, cc, __float_as_int(c4.w));
					}
				}
				++ray;
				seek = true;
			}
		}
		if(seek) {
			// next non-empty slot of the group, or write the group's radiance
			active = false;
			const unsigned g0 = ent * unsigned(neeCount);
			for(; ray < neeCount; ++ray) {
				const float4 o = __ldcs(W.sOrg + g0 + unsigned(ray));
				if(!(o.w > 0.0f)) continue;
				const float4 d = __ldcs(W.sDir + g0 + unsigned(ray));
				cnt = C();
				t.init(sp.scene(path), f4to3(o), f4to3(d), o.w, true, cnt);
				active = true;
				break;
			}
			if(!active) W.rad[path] = pack(radiance, radW);
		}
	}
	__syncthreads();
	if(threadIdx.x < 2) {
		TraceCounters* out = counters + threadIdx.x;
		const unsigned long long* v = stats.v[threadIdx.x];
		if(v[3]) {
			atomicAdd(&out->rays, v[3]);
			if(threadIdx.x == 1) atomicAdd(&out->shadowRays, v[3]);
			atomicAdd(&out->nodeVisits, v[0]);
			atomicAdd(&out->primTests, v[1]);
			atomicAdd(&out->instanceVisits, v[2]);
		}
		if(v[5]) atomicAdd(&out->errors, unsigned(v[5]));
	}
}

// One vertex of pt_sample (pt_common.hpp:75-156, random_walk.hpp:38-113):
// the vertex hit by (origin, dir) at bounce `bounce`, its emission with MIS,
// then (if the path continues) next-event estimation and the BSDF sample,
// Russian roulette and the next ray. Next-event samples with a non-zero
// contribution are handed to shadow(i, origin, dir, length, contribution) in
// the order i of pt_sample. Returns true and the next ray if the path goes on.
// The generator `rng` is advanced exactly as pt_sample advances it.
// What the adjoint needs to know about a vertex (see onVertex below).
struct VertexInfo {
	bool surface;
	int materialIndex;  // -1 for the background
	int materialType;
	f2 uv;
	f3 albedo;
	// for the auxiliary targets: whether the vertex contributes (path length
	// >= the minimum), its position, incident distance and shading normal (0
	// for a miss), and its emission after the MIS weight, before the throughput
	bool counts;
	f3 position;
	float depth;
	f3 normal;
	f3 emission;
};

// A vertex's auxiliary-target contributions, added to path p's iteration
// values (channel-major, W.auxStride paths per channel).
MBD void aux_vertex_path(const WfState& W, int p, float gw, const VertexInfo& v) {
	const f3 zero = make3(0.0f, 0.0f, 0.0f);
	aux_vertex([&](int c, float x) { float* a = W.auxIter + size_t(c) * W.auxStride + size_t(p); *a = *a + nan_to_zero(x); },
	           gw, v.position, v.depth, v.normal, v.surface ? v.uv : make2(0.0f, 0.0f),
	           v.surface && v.materialType != MAT_EMISSIVE ? v.albedo : zero, v.emission);
}

// The state of a shaded path vertex between the parts of shade_vertex.
struct ShadeState {
	f3 position, incident;
	TangentSpace ts;
	Params mat;
	int pathLen;
};

// shade_vertex, first part: hit attributes, the first-hit id, the emission
// term (pt_common.hpp:139-153; prevPos: the previous vertex, whose distance
// to an emissive sphere sets the sphere's next-event pdf). False when the path
// ends at this vertex (a miss, or the maximum path length).
template < class VertexFn >
MBD bool shade_begin(const DScene& S, const PtParams& P, int bounce, f3 origin, f3 dir, const HitRec& hr, f3 prevPos,
                     const f3& throughput, float pdfF, f3& radiance, float2* hit0, ShadeState& v, VertexFn&& onVertex) {
	bool surface = false;
	int matIndex = -1;
	f3 position = make3(0.0f, 0.0f, 0.0f), incidentEncoded;
	float incidentPdf;
	TangentSpace ts;
	Params mat;
	const Intersection hit = hit_attributes(S, origin, dir, hr);
	if(hit.inst < 0) {
		incidentEncoded = dir;
		incidentPdf = pdfF * 1.0f;
	} else {
		surface = true;
		position = origin + dir * hit.distance;
		ts = tangent_space(S, hit);
		incidentEncoded = make3(dir.x, dir.y, hit.distance * sgn(dir.z));
		matIndex = material_index(S, hit.inst, hit.prim);
		mat = fetch_material(S, uint16_t(matIndex), hit.uv);
		const float inCosAbs = fabsf(dot(dir, ts.shadingN));
		incidentPdf = __fdiv_rn(pdfF * fabsf(inCosAbs), hit.distance * hit.distance);
	}
	if(bounce == 0 && hit0) *hit0 = make_float2(float(surface ? hit.inst : -1), float(surface ? hit.prim : -1));
	const int pathLen = bounce + 1;
	// -- emission (pt_common.hpp:139-153)
	if(pathLen >= P.minPathLength) {
		f3 emission = make3(0.0f, 0.0f, 0.0f);
		float connectPdf = 0.0f;
		if(!surface) {
			if(S.hasBackground) {
				emission = lv(S.bgColor) * lv(S.bgScale);
				if(nonzero(emission)) {
					const float bgFlux = (S.bgFlux[0] + S.bgFlux[1]) + S.bgFlux[2];
					const float pb = __fdiv_rn(bgFlux, (S.dirFlux + S.rootFlux) + bgFlux);
					connectPdf = __fdiv_rn(1.0f, 4.0f * PI) * pb;
				}
			}
		} else if(mat.type == MAT_EMISSIVE) {
			const f3 ex = -incident_direction(incidentEncoded);
			const float cosOut = dot(ts.geoN, ex);
			if(cosOut > 0.0f) {
				emission = mat.radiance;
				if(nonzero(emission)) connectPdf = light_pdfs(S, hit.inst, hit.prim, hit.sp, prevPos).connect;
			}
		}
		if(nonzero(emission) && pathLen > 1) {
			const float misWeight = __fdiv_rn(1.0f, 1.0f + float(P.neeCount) * __fdiv_rn(connectPdf, incidentPdf));
			emission = emission * misWeight;
		}
		const f3 eterm = throughput * emission;
		radiance = contribute(radiance, eterm);
		onVertex(contribute(make3(0.0f, 0.0f, 0.0f), eterm), VertexInfo{ surface, matIndex, surface ? mat.type : -1, hit.uv,
		                                                            surface ? mat.albedo : make3(0.0f, 0.0f, 0.0f),
		                                                            true, position, surface ? hit.distance : 0.0f,
		                                                            surface ? ts.shadingN : make3(0.0f, 0.0f, 0.0f), emission });
	} else {
		onVertex(make3(0.0f, 0.0f, 0.0f), VertexInfo{ surface, matIndex, surface ? mat.type : -1, hit.uv,
		                                            surface ? mat.albedo : make3(0.0f, 0.0f, 0.0f),
		                                            false, position, 0.0f, make3(0.0f, 0.0f, 0.0f), make3(0.0f, 0.0f, 0.0f) });
	}
	if(!surface || !(pathLen < P.maxPathLength)) return false;
	v.position = position;
	v.incident = incident_direction(incidentEncoded);
	v.ts = ts;
	v.mat = mat;
	v.pathLen = pathLen;
	return true;
}

// Whether the next loop iteration of pt_sample estimates direct light.
MBD bool shade_has_nee(const PtParams& P, const ShadeState& v) {
	return v.pathLen + 1 >= P.minPathLength && v.pathLen + 1 <= P.maxPathLength;
}

// Next-event sample i at v (pt_common.hpp:105-124): draws its number; true
// with the shadow ray and the term it adds when it can contribute.
MBD bool shade_nee(const DScene& S, const PtParams& P, const ShadeState& v, const f3& throughput, u64& rng, u64 neeSeed,
                   int i, f3& so, f3& sd, float& stmax, f3& c, int& emitMat, float& cosOut) {
	const u64 r = pcg_next(rng);
	const float nu0 = sample_uniform(uint32_t(r)), nu1 = sample_uniform(uint32_t(r >> 32));
	const Nee nee = lights_connect(S, u64(i), u64(P.neeCount), neeSeed, v.position, nu0, nu1);
	if(!nee.valid) return false;
	EvalValue val = material_evaluate(v.ts, v.mat, v.incident, nee.dir);
	if(nee.cosOut != 0.0f) val.cosOut *= nee.cosOut;
	const f3 rad = val.value * nee.diffIrradiance;
	if(!(any_pos(rad) && val.cosOut > 0.0f)) return false;
	const float hitPdf = __fdiv_rn(val.pdfF * fabsf(nee.cosOut), nee.distSq);
	const float mis = __fdiv_rn(1.0f, float(P.neeCount) + __fdiv_rn(hitPdf, nee.creationPdf));
	c = ((throughput * val.cosOut) * rad) * mis;
	emitMat = nee.emitMat;
	cosOut = val.cosOut;
	shadow_ray(v.position, nee.position, v.ts.geoN, nee.geoNormal, nee.dir, so, sd, stmax);
	return true;
}

// The walk (random_walk.hpp:38-86): BSDF sample, throughput, Russian
// roulette; false when the path ends. nextO is already offset.
MBD bool shade_walk(const PtParams& P, const ShadeState& v, f3& throughput, float& pdfF, u64& rng, f3& nextO, f3& nextD) {
	const u64 x0 = pcg_next(rng), x1 = pcg_next(rng);
	const float ru0 = sample_uniform(uint32_t(x0)), ru1 = sample_uniform(uint32_t(x0 >> 32));
	const float rr = sample_uniform(uint32_t(pcg_next(rng)));
	const PathSample smp = material_sample(v.ts, v.mat, v.incident, ru0, ru1, x1);
	if(!smp.valid) return false;
	throughput = throughput * smp.throughput;
	if(v.pathLen >= P.rrStartDepth) {
		const float cp = fmin_(maxc(throughput) + 0.1f, 1.0f);
		if(rr >= cp) return false;
		throughput = throughput / cp;
	}
	pdfF = smp.pdfF;
	nextO = v.position;
	add_epsilon(nextO, smp.excident, v.ts.geoN);
	nextD = smp.excident;
	return true;
}

// One vertex of pt_sample: emission, next-event estimation (each shadow ray
// handed to `shadow` in order) and the walk to the next ray. prevPos: the
// previous vertex's position on entry, this vertex's on return.
template < class ShadowFn, class VertexFn >
MBD bool shade_vertex(const DScene& S, const PtParams& P, int bounce, f3 origin, f3 dir, const HitRec& hr, f3& prevPos,
                      f3& throughput, float& pdfF, f3& radiance, u64& rng, float2* hit0, f3& nextO, f3& nextD,
                      ShadowFn&& shadow, VertexFn&& onVertex) {
	ShadeState v;
	if(!shade_begin(S, P, bounce, origin, dir, hr, prevPos, throughput, pdfF, radiance, hit0, v, onVertex)) return false;
	prevPos = v.position; // the previous vertex of the next one
	if(shade_has_nee(P, v)) {
		const u64 neeSeed = pcg_next(rng);
		for(int i = 0; i < P.neeCount; ++i) {
			f3 so, sd, c;
			float stmax;
			int emitMat = -1;
			float cosOut = 0.0f;
			if(shade_nee(S, P, v, throughput, rng, neeSeed, i, so, sd, stmax, c, emitMat, cosOut))
				shadow(i, so, sd, stmax, c, emitMat, cosOut);
		}
	}
	return shade_walk(P, v, throughput, pdfF, rng, nextO, nextD);
}

// Shade stage of the wavefront: one thread per queued path. Next-event rays go
// to the shadow queue (neeCount consecutive slots per path, allocated when
// the first one is needed), the next ray to the other extension queue.
template < class SP >
MBD void shade_slot(const SP& sp, WfState& W, int q, int bounce, unsigned slot) {
	const int p = __ldcs(W.qPath[q] + slot);
	const DScene& S = sp.scene(p);
	const PtParams& P = sp.params(p);
	const f3 origin = f4to3(__ldcs(W.qOrg[q] + slot));
	const f3 dir = f4to3(__ldcs(W.qDir[q] + slot));
	const float4 hh = __ldcs(W.qHit[q] + slot);
	HitRec hr;
	hr.t = hh.x; hr.inst = __float_as_int(hh.y); hr.prim = __float_as_int(hh.z);
	hr.sp = make2(hh.w, __ldcs(W.qHitSpy[q] + slot));
	hr.has = hr.inst >= 0;
	const float4 tp = W.thrPdf[p];
	f3 throughput = f4to3(tp);
	float pdfF = tp.w;
	const float4 ra = W.rad[p];
	f3 radiance = f4to3(ra);
	u64 rng = W.rng[p];
	const u64 rng0 = rng;
	unsigned base = 0xFFFFFFFFu;
	float gw = 0.0f; // the vertex's guide weight (auxiliary targets)
	f3 nextO, nextD;
	f3 prevPos = S.sphereLights ? f4to3(W.prevPos[p]) : origin;
	const bool cont = shade_vertex(S, P, bounce, origin, dir, hr, prevPos, throughput, pdfF, radiance, rng, W.hit0 + p,
		nextO, nextD, [&](int i, f3 so, f3 sd, float stmax, f3 c, int emitMat, float cosOut) {
			if(base == 0xFFFFFFFFu) {
				base = atomicAdd(W.counters + C_SHADOW0 + q, unsigned(P.neeCount));
				for(int k = 0; k < P.neeCount; ++k) { W.sPath[base + k] = p; W.sOrg[base + k] = make_float4(0, 0, 0, -1.0f); }
				if(W.sortBits)
					bin_append(W.shKey, W.binHist + (1u << W.sortBits), base / unsigned(P.neeCount), ray_key(W, S, sp.group(p), so, sd));
			}
			W.sOrg[base + i] = pack(so, stmax);
			W.sDir[base + i] = pack(sd, W.auxIter ? __fmul_rn(gw, cosOut) : 0.0f); // w: its Lightness term
			W.sContrib[base + i] = pack(c, __int_as_float(emitMat)); // w: the emitter's material (adjoint)
		}, [&](f3 e, const VertexInfo& v) {
			if constexpr(SP::adjoint) adjoint_vertex(sp.A, S, p, e, v.surface, v.materialType, v.materialIndex, v.uv, v.albedo);
			if(W.auxIter) {
				float ma = W.guide[p].x;
				gw = guide_after_segment(ma, pdfF); // pdfF: the pdf of the segment that reached this vertex
				W.guide[p] = make_float2(ma, gw);
				if(v.counts) aux_vertex_path(W, p, gw, v);
			}
		});
	W.rad[p] = pack(radiance, ra.w);
	if(rng != rng0) W.rng[p] = rng;
	if(!cont) return;
	W.thrPdf[p] = pack(throughput, pdfF);
	if(S.sphereLights) W.prevPos[p] = pack(prevPos, 0.0f);
	const int out = q ^ 1;
	const unsigned nslot = warp_reserve(W.counters + out, 1u);
	W.qPath[out][nslot] = p;
	W.qOrg[out][nslot] = pack(nextO, 0.0f);
	W.qDir[out][nslot] = pack(nextD, 0.0f);
	if(W.sortBits) bin_append(W.extKey, W.binHist, nslot, ray_key(W, S, sp.group(p), nextO, nextD));
}

// Shade stage of the wavefront over queue q, grid-stride over its entries
// (a fixed grid, so that a launch over a short or empty queue costs little).
// Register budget: 8 resident blocks of 128 threads; the shade is bound by
// the latency of scattered vertex-attribute reads, and the higher occupancy
// made the stage 14 % faster than the unbounded 126-register build (0.44 vs
// 0.52 ms per 1080p iteration).
template < class SP >
__global__ void __launch_bounds__(128, 8) k_shade(const SP sp, WfState W, int q, int bounce, unsigned tailMax, int tailAllowed) {
	const unsigned count = *reinterpret_cast<volatile unsigned*>(W.counters + q);
	if(*reinterpret_cast<volatile unsigned*>(W.counters + C_TAILED)) return;
	if(tailAllowed && count <= tailMax) {
		// the tail launch of this bounce took the paths; later launches skip
		if(blockIdx.x == 0 && threadIdx.x == 0) W.counters[C_TAILED] = 1u;
		return;
	}
	for(unsigned slot = blockIdx.x * blockDim.x + threadIdx.x; slot < count; slot += gridDim.x * blockDim.x)
		shade_slot(sp, W, q, bounce, slot);
}

// Tail of an iteration: persistent threads take the paths of extension queue
// q (already traced, bounce `bounce`) and finish each of them in place:
// shade, trace the next-event rays one by one and add their contributions in
// order, trace the next extension ray, and so on until the path ends. Used
// once few paths are left, where a separate launch per bounce would be
// dominated by launch and drain latency.
//
// The lanes run a state machine: a lane takes a new path as soon as its own
// ends (the warp claims all idle lanes' paths with one atomic), and every pass
// of the loop traces at most one ray per lane (a shadow ray or the next
// extension ray) in one traversal loop shared by the warp. A path's random
// numbers, terms and their order are those of shade_vertex.
template < int MINB, class SP, class C, int AM >
__global__ void __launch_bounds__(128, MINB) k_tail(const SP sp, WfState W, int q, int bounce,
                                                    int workIdx, TraceCounters* counters, unsigned tailMax) {
	__shared__ BlockStats stats;
	if(threadIdx.x < 12) (&stats.v[0][0])[threadIdx.x] = 0ull;
	__syncthreads();
	const unsigned count = *reinterpret_cast<volatile unsigned*>(W.counters + q);
	// takes over only the first bounce whose queue holds at most tailMax paths
	if(*reinterpret_cast<volatile unsigned*>(W.counters + C_TAILED) || count > tailMax) return;
	enum { T_IDLE = 0, T_NEE, T_WALK, T_EXIT };
	LocalStack stack;
	const unsigned lane = threadIdx.x & 31u;
	int phase = T_IDLE;
	int p = 0, b = 0, i = 0;
	int emitMat = -1; // emitter material of the current shadow ray (adjoint)
	float guideA = 0.0f, gw = 0.0f, lightTerm = 0.0f; // auxiliary targets: footprint, guide weight, shadow ray's term
	f3 throughput = make3(0.0f, 0.0f, 0.0f), radiance = make3(0.0f, 0.0f, 0.0f), c = make3(0.0f, 0.0f, 0.0f);
	float pdfF = 0.0f, radW = 0.0f;
	u64 rng = 0, neeSeed = 0;
	ShadeState v;
	auto on_vertex = [&](f3 e, const VertexInfo& vi) {
		if constexpr(SP::adjoint) adjoint_vertex(sp.A, sp.scene(p), p, e, vi.surface, vi.materialType, vi.materialIndex, vi.uv, vi.albedo);
		if(W.auxIter) {
			gw = guide_after_segment(guideA, pdfF); // pdfF: the pdf of the segment that reached this vertex
			if(vi.counts) aux_vertex_path(W, p, gw, vi);
		}
	};
	// shades the vertex a traced extension ray reached; sets the next phase
	auto begin_vertex = [&](f3 origin, f3 dir, const HitRec& hr, f3 prevPos) {
		const DScene& S = sp.scene(p);
		const PtParams& P = sp.params(p);
		if(!shade_begin(S, P, b, origin, dir, hr, prevPos, throughput, pdfF, radiance, W.hit0 + p, v, on_vertex)) {
			W.rad[p] = pack(radiance, radW);
			W.rng[p] = rng;
			phase = T_IDLE;
			return;
		}
		i = 0;
		if(shade_has_nee(P, v)) { neeSeed = pcg_next(rng); phase = T_NEE; }
		else phase = T_WALK;
	};
	for(;;) {
		const unsigned idle = __ballot_sync(0xffffffffu, phase == T_IDLE);
		if(idle) {
			const int leader = __ffs(idle) - 1;
			unsigned base = 0;
			if(int(lane) == leader) base = atomicAdd(W.counters + C_WORK + workIdx, unsigned(__popc(idle)));
			base = __shfl_sync(0xffffffffu, base, leader);
			if(phase == T_IDLE) {
				const unsigned item = base + unsigned(__popc(idle & ((1u << lane) - 1u)));
				if(item >= count) phase = T_EXIT;
				else {
					p = W.qPath[q][item];
					const float4 hh = W.qHit[q][item];
					HitRec hr;
					hr.t = hh.x; hr.inst = __float_as_int(hh.y); hr.prim = __float_as_int(hh.z);
					hr.sp = make2(hh.w, W.qHitSpy[q][item]);
					hr.has = hr.inst >= 0;
					const float4 tp = W.thrPdf[p];
					throughput = f4to3(tp);
					pdfF = tp.w;
					const float4 ra = W.rad[p];
					radiance = f4to3(ra);
					radW = ra.w;
					rng = W.rng[p];
					if(W.auxIter) guideA = W.guide[p].x;
					b = bounce;
					const f3 o = f4to3(W.qOrg[q][item]);
					begin_vertex(o, f4to3(W.qDir[q][item]), hr, sp.scene(p).sphereLights ? f4to3(W.prevPos[p]) : o);
				}
			}
		}
		if(__all_sync(0xffffffffu, phase == T_EXIT)) break;
		bool trace = false, shadow = false;
		f3 ro = make3(0.0f, 0.0f, 0.0f), rd = make3(0.0f, 0.0f, 1.0f);
		float tmax = MAX_SCENE_SIZE;
		if(phase == T_NEE) {
			const DScene& S = sp.scene(p);
			const PtParams& P = sp.params(p);
			while(i < P.neeCount) {
				if(shade_nee(S, P, v, throughput, rng, neeSeed, i, ro, rd, tmax, c, emitMat, lightTerm)) { trace = shadow = true; break; }
				++i;
			}
			if(!trace) phase = T_WALK;
		}
		if(!trace && phase == T_WALK) {
			if(shade_walk(sp.params(p), v, throughput, pdfF, rng, ro, rd)) { trace = true; tmax = MAX_SCENE_SIZE; }
			else {
				W.rad[p] = pack(radiance, radW);
				W.rng[p] = rng;
				phase = T_IDLE;
			}
		}
		if(!trace) continue;
		const DScene& S = sp.scene(p);
		C cnt;
		WideTracerT<AM> t;
		t.init(S, ro, rd, tmax, shadow, cnt);
		while(!t.step(S, cnt, stack)) {}
		stats_add(stats, shadow ? 1 : 0, cnt);
		if(shadow) {
			if(!t.occluded) {
				radiance = contribute(radiance, c);
				if constexpr(SP::adjoint) {
					const f3 cc = contribute(make3(0.0f, 0.0f, 0.0f), c);
					adjoint_add(sp.A, p, cc);
					adjoint_emitted(sp.A, S, p, cc, emitMat);
				}
				if(W.auxIter) {
					float* a = W.auxIter + size_t(AUX_LIGHT) * W.auxStride + size_t(p);
					*a = *a + nan_to_zero(__fmul_rn(gw, lightTerm));
				}
			}
			++i;
		} else {
			++b;
			begin_vertex(ro, rd, t.best, v.position);
		}
	}
	__syncthreads();
	if(threadIdx.x < 2) {
		TraceCounters* out = counters + threadIdx.x;
		const unsigned long long* v2 = stats.v[threadIdx.x];
		if(v2[3]) {
			atomicAdd(&out->rays, v2[3]);
			if(threadIdx.x == 1) atomicAdd(&out->shadowRays, v2[3]);
			atomicAdd(&out->nodeVisits, v2[0]);
			atomicAdd(&out->primTests, v2[1]);
			atomicAdd(&out->instanceVisits, v2[2]);
		}
		if(v2[5]) atomicAdd(&out->errors, unsigned(v2[5]));
	}
}

__global__ void k_finalize(WfState W, RenderState R, uint32_t numPixels) {
	const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
	if(p >= numPixels) return;
	const int iteration = R.dIteration ? *R.dIteration : R.iteration;
	const float4 rad = W.rad[p];
	if(R.radiance) {
		float* cr = R.radiance + 3 * size_t(p);
		float* vr = R.radianceVar ? R.radianceVar + 3 * size_t(p) : nullptr;
		const float it[3] = { rad.x, rad.y, rad.z };
		for(int c = 0; c < 3; ++c) update_moments(it[c], cr + c, vr ? vr + c : nullptr, iteration);
	}
	if(R.hitId) {
		const float2 h = W.hit0[p];
		float* ch = R.hitId + 2 * size_t(p);
		float* vh = R.hitIdVar ? R.hitIdVar + 2 * size_t(p) : nullptr;
		const float it[2] = { h.x, h.y };
		for(int c = 0; c < 2; ++c) update_moments(it[c], ch + c, vh ? vh + c : nullptr, iteration);
	}
	if(R.iterRadiance) {
		float* o = R.iterRadiance + 3 * size_t(p);
		o[0] = rad.x; o[1] = rad.y; o[2] = rad.z;
	}
	if(R.auxOn && W.auxIter)
		for(int a = 0; a < AUX_TARGETS; ++a) {
			if(!R.aux[a]) continue;
			float* cum = R.aux[a] + size_t(aux_count(a)) * p;
			float* var = R.auxVar[a] ? R.auxVar[a] + size_t(aux_count(a)) * p : nullptr;
			for(int c = 0; c < aux_count(a); ++c)
				update_moments(W.auxIter[size_t(aux_first(a) + c) * W.auxStride + p], cum + c, var ? var + c : nullptr, iteration);
		}
}

MBD void adjoint_vertex(const AdjointState& A, const DScene& S, int p, f3 e, bool surface, int type, int mat, f2 uv,
                        f3 albedo) {
	adjoint_add(A, p, e);
	if(surface && type == MAT_EMISSIVE) adjoint_emitted(A, S, p, e, mat);
	if(A.texIndex < 0 || !surface || type != MAT_LAMBERT || __ldg(&S.materials[mat].albedoTex) != A.texIndex) return;
	const int k = A.count[p];
	if(k >= int(A.maxEntries)) return;
	const float fx = uv.x - floorf(uv.x), fy = uv.y - floorf(uv.y);
	int x = int(fx * float(A.tex.width)), y = int(fy * float(A.tex.height));
	if(x >= int(A.tex.width)) x = int(A.tex.width) - 1;
	if(y >= int(A.tex.height)) y = int(A.tex.height) - 1;
	A.entry[size_t(k) * A.numPaths + p] = make_float4(albedo.x, albedo.y, albedo.z, __int_as_float(y * int(A.tex.width) + x));
	A.suffix[size_t(k) * A.numPaths + p] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
	A.count[p] = k + 1;
}

// End of an adjoint sample: d(sample)/d(a_k) = suffix_k / a_k, weighted by
// scale * dL/dI of the pixel, added to the texel gradient.
// The emission derivative: sum over paths of scale * dL/dI * emisAcc, reduced
// per warp before the atomics.
__global__ void k_adjoint_scatter(AdjointState A) {
	const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
	if(A.emitTarget) {
		float3 e = make_float3(0.0f, 0.0f, 0.0f);
		if(p < A.numPaths) {
			const float4 a = A.emisAcc[p];
			e = make_float3(A.imageGrad[3 * size_t(p)] * A.scale * a.x, A.imageGrad[3 * size_t(p) + 1] * A.scale * a.y,
			                A.imageGrad[3 * size_t(p) + 2] * A.scale * a.z);
		}
		for(int off = 16; off > 0; off >>= 1) {
			e.x += __shfl_down_sync(0xffffffffu, e.x, off);
			e.y += __shfl_down_sync(0xffffffffu, e.y, off);
			e.z += __shfl_down_sync(0xffffffffu, e.z, off);
		}
		if((threadIdx.x & 31u) == 0) {
			if(e.x != 0.0f) atomicAdd(A.emisGrad, e.x);
			if(e.y != 0.0f) atomicAdd(A.emisGrad + 1, e.y);
			if(e.z != 0.0f) atomicAdd(A.emisGrad + 2, e.z);
		}
	}
	if(p >= A.numPaths) return;
	const int n = A.count[p];
	if(n == 0) return;
	const f3 g = make3(A.imageGrad[3 * size_t(p)] * A.scale, A.imageGrad[3 * size_t(p) + 1] * A.scale,
	                   A.imageGrad[3 * size_t(p) + 2] * A.scale);
	for(int k = 0; k < n; ++k) {
		const float4 a = A.entry[size_t(k) * A.numPaths + p];
		const float4 sf = A.suffix[size_t(k) * A.numPaths + p];
		float* t = A.texGrad + 3 * size_t(__float_as_int(a.w));
		if(a.x > 0.0f && sf.x != 0.0f) atomicAdd(t, g.x * __fdiv_rn(sf.x, a.x));
		if(a.y > 0.0f && sf.y != 0.0f) atomicAdd(t + 1, g.y * __fdiv_rn(sf.y, a.y));
		if(a.z > 0.0f && sf.z != 0.0f) atomicAdd(t + 2, g.z * __fdiv_rn(sf.z, a.z));
	}
}

// Path-replay adjoint of the radiance with respect to one albedo texture
// (no counterpart in the reference). One launch replays one sample of every
// pixel with the generator state `rng` (seeded as for a reset render, so that
// sample s replays iteration s of the forward render) through the same code
// as the forward path tracer. With Russian roulette off (rrStartDepth >=
// maxPathLength), the sample's radiance is a sum of terms that are products
// of the Lambert albedos of the vertices before them; each term after vertex
// k contains vertex k's albedo a_k once, so d(radiance)/d(a_k) = (sum of the
// terms added after vertex k, its own next-event terms included) / a_k. The
// suffix sums are kept per textured vertex (no subtraction of running sums),
// and `scale * imageGrad[p] * suffix / a_k` is added to the gradient of the
// texel the vertex looked up (nearest texel, as sample_texture). With
// emission targets, each term emitted by a flagged material adds term / L to
// d(radiance)/dL, weighted the same way and reduced per warp at the end.
constexpr int ADJOINT_MAX_VERTICES = 32;

__global__ void __launch_bounds__(128, 4) k_adjoint_albedo(const DScene S, const PtParams P, uint64_t* rng,
                                                            uint32_t numPixels, uint32_t width, AdjointTargets T,
                                                            const float* __restrict__ imageGrad, float scale) {
	LocalStack stack;
	const int texIndex = T.texIndex;
	const DTexture tex = texIndex >= 0 ? S.textures[texIndex] : DTexture{ 0, 0, nullptr };
	f3 emisSum = make3(0.0f, 0.0f, 0.0f); // this thread's share of dLoss/dL
	auto emitted = [&](f3 c, int mat, f3& acc) {
		if(!T.emitTarget || mat < 0 || !__ldg(T.emitTarget + mat)) return;
		const f3 L = load3(S.materials[mat].radiance);
		if(L.x > 0.0f) acc.x += __fdiv_rn(c.x, L.x);
		if(L.y > 0.0f) acc.y += __fdiv_rn(c.y, L.y);
		if(L.z > 0.0f) acc.z += __fdiv_rn(c.z, L.z);
	};
	for(uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < numPixels; p += gridDim.x * blockDim.x) {
		u64 r = rng[p];
		(void)pcg_next(r); // create_camera
		const u64 x0 = pcg_next(r);
		(void)pcg_next(r);
		const float rr = sample_uniform(uint32_t(pcg_next(r)));
		const float ru0 = sample_uniform(uint32_t(x0)), ru1 = sample_uniform(uint32_t(x0 >> 32));
		float pdfF;
		f3 dir = pinhole_ray(S.camera, int(p % width), int(p / width), ru0, ru1, pdfF);
		f3 throughput = make3(1.0f, 1.0f, 1.0f);
		bool alive = true;
		if(0 >= P.rrStartDepth) {
			const float cp = fmin_(maxc(throughput) + 0.1f, 1.0f);
			if(rr >= cp) alive = false;
			else throughput = throughput / cp;
		}
		int texel[ADJOINT_MAX_VERTICES];
		f3 alb[ADJOINT_MAX_VERTICES], suf[ADJOINT_MAX_VERTICES];
		int n = 0;
		f3 em = make3(0.0f, 0.0f, 0.0f);
		f3 radiance = make3(0.0f, 0.0f, 0.0f);
		f3 origin = lv(S.camera.position);
		f3 prevPos = origin;
		add_epsilon(origin, dir, make3(0.0f, 0.0f, 0.0f));
		for(int b = 0; alive; ++b) {
			LocalCounters cnt;
			const HitRec hr = closest_hit_wide(S, origin, dir, MAX_SCENE_SIZE, cnt, stack);
			f3 nextO, nextD;
			const bool cont = shade_vertex(S, P, b, origin, dir, hr, prevPos, throughput, pdfF, radiance, r, nullptr, nextO, nextD,
				[&](int, f3 so, f3 sd, float stmax, f3 c, int emitMat, float) {
					LocalCounters sc;
					if(occluded_wide(S, so, sd, stmax, sc, stack)) return;
					const f3 cc = contribute(make3(0.0f, 0.0f, 0.0f), c);
					radiance = radiance + cc;
					for(int k = 0; k < n; ++k) suf[k] = suf[k] + cc;
					emitted(cc, emitMat, em);
				},
				[&](f3 e, const VertexInfo& v) {
					for(int k = 0; k < n; ++k) suf[k] = suf[k] + e;
					if(v.surface && v.materialType == MAT_EMISSIVE) emitted(e, v.materialIndex, em);
					if(texIndex >= 0 && v.surface && v.materialType == MAT_LAMBERT && n < ADJOINT_MAX_VERTICES &&
					   __ldg(&S.materials[v.materialIndex].albedoTex) == texIndex) {
						const float fx = v.uv.x - floorf(v.uv.x), fy = v.uv.y - floorf(v.uv.y);
						int x = int(fx * float(tex.width)), y = int(fy * float(tex.height));
						if(x >= int(tex.width)) x = int(tex.width) - 1;
						if(y >= int(tex.height)) y = int(tex.height) - 1;
						texel[n] = y * int(tex.width) + x;
						alb[n] = v.albedo;
						suf[n] = make3(0.0f, 0.0f, 0.0f);
						++n;
					}
				});
			if(!cont) break;
			origin = nextO;
			dir = nextD;
		}
		rng[p] = r;
		const f3 g = make3(imageGrad[3 * size_t(p)] * scale, imageGrad[3 * size_t(p) + 1] * scale,
		                   imageGrad[3 * size_t(p) + 2] * scale);
		for(int k = 0; k < n; ++k) {
			float* t = T.texGrad + 3 * size_t(texel[k]);
			if(alb[k].x > 0.0f && suf[k].x != 0.0f) atomicAdd(t, g.x * __fdiv_rn(suf[k].x, alb[k].x));
			if(alb[k].y > 0.0f && suf[k].y != 0.0f) atomicAdd(t + 1, g.y * __fdiv_rn(suf[k].y, alb[k].y));
			if(alb[k].z > 0.0f && suf[k].z != 0.0f) atomicAdd(t + 2, g.z * __fdiv_rn(suf[k].z, alb[k].z));
		}
		emisSum = emisSum + make3(g.x * em.x, g.y * em.y, g.z * em.z);
	}
	if(T.emitTarget) {
		for(int off = 16; off > 0; off >>= 1) {
			emisSum.x += __shfl_down_sync(0xffffffffu, emisSum.x, off);
			emisSum.y += __shfl_down_sync(0xffffffffu, emisSum.y, off);
			emisSum.z += __shfl_down_sync(0xffffffffu, emisSum.z, off);
		}
		if((threadIdx.x & 31u) == 0) {
			if(emisSum.x != 0.0f) atomicAdd(T.emisGrad, emisSum.x);
			if(emisSum.y != 0.0f) atomicAdd(T.emisGrad + 1, emisSum.y);
			if(emisSum.z != 0.0f) atomicAdd(T.emisGrad + 2, emisSum.z);
		}
	}
}

// Accumulation of a batch iteration into each job's image (jobs whose
// samples are all taken are left alone).
__global__ void k_finalize_batch(const DJob* jobs, WfState W, const uint16_t* pathJob, uint32_t numPixels, int iteration) {
	const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
	if(g >= numPixels) return;
	const DJob& J = jobs[pathJob[g]];
	if(iteration >= int(J.spp)) return;
	const size_t local = g - J.pixelOffset;
	const float den = fmaxf(1.0f, float(iteration) + 1.0f);
	const float4 rad = W.rad[g];
	float* cr = J.radiance + 3 * local;
	const float it[3] = { rad.x, rad.y, rad.z };
	for(int c = 0; c < 3; ++c) { const float diff = it[c] - cr[c]; cr[c] += __fdiv_rn(diff, den); }
	if(J.hitId) {
		const float2 h = W.hit0[g];
		float* ch = J.hitId + 2 * local;
		const float ih[2] = { h.x, h.y };
		for(int c = 0; c < 2; ++c) { const float diff = ih[c] - ch[c]; ch[c] += __fdiv_rn(diff, den); }
	}
}

// Closest hits / shadow-ray tests of caller-provided rays over the wide
// hierarchies (the parity and measurement entry points).
__global__ void k_trace_rays_wide(const DScene S, const float* rays, const float* geoNormals, float tmax, uint32_t n,
                                  float* tOut, int32_t* instOut, int32_t* primOut, float* spOut) {
	LocalStack stack;
	LocalCounters cnt;
	for(uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
		f3 o = make3(rays[6 * i], rays[6 * i + 1], rays[6 * i + 2]);
		const f3 d = make3(rays[6 * i + 3], rays[6 * i + 4], rays[6 * i + 5]);
		const f3 g = geoNormals ? make3(geoNormals[3 * i], geoNormals[3 * i + 1], geoNormals[3 * i + 2]) : make3(0, 0, 0);
		add_epsilon(o, d, g);
		const HitRec hr = closest_hit_wide(S, o, d, tmax, cnt, stack);
		const Intersection h = hit_attributes(S, o, d, hr);
		tOut[i] = h.distance; instOut[i] = h.inst; primOut[i] = h.prim;
		if(spOut) { spOut[2 * i] = h.sp.x; spOut[2 * i + 1] = h.sp.y; }
	}
}

__global__ void k_occlusion_wide(const DScene S, const float* a, const float* b, uint32_t n, uint8_t* out) {
	LocalStack stack;
	LocalCounters cnt;
	for(uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
		const f3 pa = make3(a[3 * i], a[3 * i + 1], a[3 * i + 2]);
		const f3 pb = make3(b[3 * i], b[3 * i + 1], b[3 * i + 2]);
		const f3 dv = pb - pa;
		const f3 dir = dv / len(dv);
		f3 so, sd;
		float stmax;
		shadow_ray(pa, pb, make3(0, 0, 0), make3(0, 0, 0), dir, so, sd, stmax);
		out[i] = occluded_wide(S, so, sd, stmax, cnt, stack) ? 1 : 0;
	}
}

int persistent_blocks(const void* fn, int threads);

template < class SP > struct TraceKernel {
	using Fn = void (*)(const SP, WfState, int, int, int, TraceCounters*, int, int);
	Fn fn;
	int blocks;
};
// The trace kernel compiled for `perSm` resident blocks of 128 threads
// (register budget 65536 / (128 * perSm)); other values pick 6. With
// `counting`, the variant that counts node visits, primitive tests and
// instance entries per ray kind (it decides on alpha textures per step);
// otherwise the variant for scenes with (`alpha`) or without alpha textures.
template < class SP > TraceKernel<SP> trace_kernel(int perSm, bool counting, bool alpha) {
	static TraceKernel<SP> table[3][4] = {};
	static const typename TraceKernel<SP>::Fn fns[3][4] = {
		{ k_trace<4, SP, NoCounters, ALPHA_NEVER>, k_trace<5, SP, NoCounters, ALPHA_NEVER>,
		  k_trace<6, SP, NoCounters, ALPHA_NEVER>, k_trace<8, SP, NoCounters, ALPHA_NEVER> },
		{ k_trace<4, SP, NoCounters, ALPHA_ALWAYS>, k_trace<5, SP, NoCounters, ALPHA_ALWAYS>,
		  k_trace<6, SP, NoCounters, ALPHA_ALWAYS>, k_trace<8, SP, NoCounters, ALPHA_ALWAYS> },
		{ k_trace<4, SP, LocalCounters, ALPHA_SCENE>, k_trace<5, SP, LocalCounters, ALPHA_SCENE>,
		  k_trace<6, SP, LocalCounters, ALPHA_SCENE>, k_trace<8, SP, LocalCounters, ALPHA_SCENE> } };
	static const int occ[4] = { 4, 5, 6, 8 };
	int idx = 2;
	for(int i = 0; i < 4; ++i) if(occ[i] == perSm) idx = i;
	const int c = counting ? 2 : (alpha ? 1 : 0);
	if(!table[c][idx].fn)
		table[c][idx] = { fns[c][idx], persistent_blocks(reinterpret_cast<const void*>(fns[c][idx]), int(WF_BLOCK)) };
	return table[c][idx];
}

template < class SP > struct TailKernel {
	using Fn = void (*)(const SP, WfState, int, int, int, TraceCounters*, unsigned);
	Fn fn;
	int blocks;
};
template < class SP > TailKernel<SP> tail_kernel(bool counting, bool alpha) {
	static TailKernel<SP> k[3] = {};
	const typename TailKernel<SP>::Fn fn = counting ? k_tail<4, SP, LocalCounters, ALPHA_SCENE>
	                                     : alpha ? k_tail<4, SP, NoCounters, ALPHA_ALWAYS> : k_tail<4, SP, NoCounters, ALPHA_NEVER>;
	const int c = counting ? 2 : (alpha ? 1 : 0);
	if(!k[c].fn) k[c] = { fn, persistent_blocks(reinterpret_cast<const void*>(fn), int(WF_BLOCK)) };
	return k[c];
}

// Stage timing and launch counting of one iteration.
struct LaunchLog {
	WfLaunchInfo& L;
	cudaStream_t stream;
	void begin(WfStage k) {
		++L.launches;
		if(L.events && L.pairsUsed < L.eventPairs) {
			L.kinds[L.pairsUsed] = (unsigned char)k;
			cudaEventRecord(L.events[2 * L.pairsUsed], stream);
		}
	}
	void end() {
		if(L.events && L.pairsUsed < L.eventPairs) cudaEventRecord(L.events[2 * L.pairsUsed++ + 1], stream);
	}
};

// The bounces of one iteration after the camera stage: per-bounce trace and
// shade launches for bounces 0 .. wavefrontBounces, then one launch that
// finishes the remaining paths. `numPaths` bounds the queue lengths.
template < class SP >
void run_bounces(const SP& sp, WfState W, TraceCounters* counters, uint32_t numPaths, int maxBounces, int neeCount,
                 const WfTuning& tuning, LaunchLog& log, cudaStream_t stream) {
	const int refillLanes = tuning.refillLanes < 1 ? 1 : (tuning.refillLanes > 32 ? 32 : tuning.refillLanes);
	const TraceKernel<SP> tk = trace_kernel<SP>(tuning.traceBlocksPerSm, tuning.counters, tuning.alpha);
	const unsigned workSlots = WF_COUNTERS - WF_BOUNCE_STATS - C_WORK;
	static int sms = 0;
	if(!sms) { int dev = 0; cudaGetDevice(&dev); cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev); }
	const unsigned shadeGrid = std::max(1u, std::min((numPaths + 127) / 128, unsigned(sms) * 16u));
	const unsigned tailMax = unsigned(tuning.tailPaths < 0 ? 0 : tuning.tailPaths);
	const bool binning = tuning.sortBits > 0 && W.extKey != nullptr;
	// key bits: the group's above the direction and origin bits, at most WF_SORT_MAX_BITS in all
	W.sortGroupBits = binning ? std::min(tuning.sortGroupBits, WF_SORT_MAX_BITS - 1) : 0;
	W.sortBits = binning ? std::min(tuning.sortBits + W.sortGroupBits, WF_SORT_MAX_BITS) : 0;
	W.sortDirBits = std::min(tuning.sortDirBits == 3 || tuning.sortDirBits == 6 ? tuning.sortDirBits : 0,
	                         W.sortBits - W.sortGroupBits);
	// After the shade of bounce b, the rays it queued are binned for the
	// trace launch of bounce b + 1.
	// every shade's counts are consumed by the scan that follows it, except
	// those of an iteration's last shade: start each iteration from zero
	if(binning) cudaMemsetAsync(W.binHist, 0, (size_t(2) << W.sortBits) * sizeof(unsigned), stream);
	auto bin = [&](int b) {
		if(!binning || b + 1 >= maxBounces) return;
		log.begin(WF_BIN);
		k_bin_scan<<<2, 1024, 0, stream>>>(W.binHist, W.binCursor, W.sortBits);
		++log.L.launches; // the scatter: two launches in one timed stage
		k_bin_scatter<<<unsigned(sms) * 8u, 256, 0, stream>>>(W, (b & 1) ^ 1, neeCount, numPaths);
		log.end();
	};
	unsigned work = 0;
	for(int b = 0; b < maxBounces; ++b) {
		const int q = b & 1;
		if(work + 2 > workSlots) { // very long paths: recycle the work counters (stream ordered)
			cudaMemsetAsync(W.counters + C_WORK, 0, sizeof(unsigned) * workSlots, stream);
			work = 0;
		}
		WfState Wt = W;
		Wt.ordered = binning && b >= 1 ? 1 : 0;
		log.begin(WF_EXTEND);
		tk.fn<<<tk.blocks, WF_BLOCK, 0, stream>>>(sp, Wt, q, neeCount, int(work++), counters, refillLanes, b);
		log.end();
		if(tuning.tailBounce >= 0) {
			// planned schedule: the tail takes over at tailBounce, nothing follows
			if(b == tuning.tailBounce && b + 1 < maxBounces) {
				const TailKernel<SP> tl = tail_kernel<SP>(tuning.counters, tuning.alpha);
				log.begin(WF_TAIL);
				tl.fn<<<tl.blocks, WF_BLOCK, 0, stream>>>(sp, W, q, b, int(work++), counters, 0xFFFFFFFFu);
				log.end();
				break;
			}
			log.begin(WF_SHADE);
			k_shade<SP><<<(numPaths + 127) / 128, 128, 0, stream>>>(sp, W, q, b, 0u, 0); // one thread per entry
			log.end();
			bin(b);
			continue;
		}
		// From bounce wavefrontBounces on, the first bounce whose queue holds
		// at most tailMax paths is finished by one launch (decided on the
		// device from the queue length); the later launches return at once.
		const bool tailAllowed = b >= tuning.wavefrontBounces && b + 1 < maxBounces;
		if(tailAllowed) {
			const TailKernel<SP> tl = tail_kernel<SP>(tuning.counters, tuning.alpha);
			log.begin(WF_TAIL);
			tl.fn<<<tl.blocks, WF_BLOCK, 0, stream>>>(sp, W, q, b, int(work++), counters, tailMax);
			log.end();
		}
		// the shade of this bounce appends to the other queue and to the shadow
		// queue (the trace launch above reset both counters)
		log.begin(WF_SHADE);
		k_shade<SP><<<shadeGrid, 128, 0, stream>>>(sp, W, q, b, tailMax, tailAllowed ? 1 : 0);
		log.end();
		bin(b);
	}
}

int persistent_blocks(const void* fn, int threads) {
	int dev = 0, sms = 148, perSm = 4;
	cudaGetDevice(&dev);
	cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
	cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, fn, threads, 0);
	return sms * (perSm > 0 ? perSm : 1);
}

} // namespace

namespace {
constexpr size_t WF_ALIGN = 256;
size_t wf_align(size_t b) { return (b + WF_ALIGN - 1) / WF_ALIGN * WF_ALIGN; }
} // namespace

size_t wavefront_bytes(size_t n, int nee) {
	if(nee < 1) nee = 1;
	return wf_align(n * 16) * 3 + wf_align(n * 8) + 2 * (wf_align(n * 4) + 3 * wf_align(n * 16) + wf_align(n * 4)) +
	       wf_align(n * nee * 4) + 3 * wf_align(n * nee * 16) + wf_align(WF_COUNTERS * 4) +
	       4 * wf_align(n * 4) + 2 * wf_align((size_t(2) << WF_SORT_MAX_BITS) * 4);
}

void wavefront_carve(void* memory, size_t n, int nee, WfState& W) {
	if(nee < 1) nee = 1;
	char* m = static_cast<char*>(memory);
	auto take = [&](size_t b) { char* p = m; m += wf_align(b); return p; };
	W.thrPdf = reinterpret_cast<float4*>(take(n * 16));
	W.rad = reinterpret_cast<float4*>(take(n * 16));
	W.prevPos = reinterpret_cast<float4*>(take(n * 16));
	W.hit0 = reinterpret_cast<float2*>(take(n * 8));
	for(int q = 0; q < 2; ++q) {
		W.qPath[q] = reinterpret_cast<int*>(take(n * 4));
		W.qOrg[q] = reinterpret_cast<float4*>(take(n * 16));
		W.qDir[q] = reinterpret_cast<float4*>(take(n * 16));
		W.qHit[q] = reinterpret_cast<float4*>(take(n * 16));
		W.qHitSpy[q] = reinterpret_cast<float*>(take(n * 4));
	}
	W.sPath = reinterpret_cast<int*>(take(n * nee * 4));
	W.sOrg = reinterpret_cast<float4*>(take(n * nee * 16));
	W.sDir = reinterpret_cast<float4*>(take(n * nee * 16));
	W.sContrib = reinterpret_cast<float4*>(take(n * nee * 16));
	W.counters = reinterpret_cast<unsigned*>(take(WF_COUNTERS * 4));
	W.extKey = reinterpret_cast<unsigned*>(take(n * 4));
	W.shKey = reinterpret_cast<unsigned*>(take(n * 4));
	W.extOrder = reinterpret_cast<unsigned*>(take(n * 4));
	W.shOrder = reinterpret_cast<unsigned*>(take(n * 4));
	W.binHist = reinterpret_cast<unsigned*>(take((size_t(2) << WF_SORT_MAX_BITS) * 4));
	W.binCursor = reinterpret_cast<unsigned*>(take((size_t(2) << WF_SORT_MAX_BITS) * 4));
	W.sortBits = 0;
	W.sortDirBits = 0;
	W.sortGroupBits = 0;
	W.ordered = 0;
	W.guide = nullptr;
	W.auxIter = nullptr;
	W.auxStride = 0;
}

cudaError_t launch_adjoint_albedo(const DScene& S, const PtParams& P, uint64_t* rng, uint32_t width, uint32_t height,
                                  const AdjointTargets& T, const float* imageGrad, float scale, cudaStream_t stream) {
	const uint32_t n = width * height;
	if(n == 0) return cudaSuccess;
	static int sms = 0;
	if(!sms) { int dev = 0; cudaGetDevice(&dev); cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev); }
	const unsigned blocks = std::min<unsigned>((n + 127) / 128, unsigned(sms) * 8u);
	k_adjoint_albedo<<<blocks, 128, 0, stream>>>(S, P, rng, n, width, T, imageGrad, scale);
	return cudaGetLastError();
}

size_t adjoint_bytes(size_t numPaths, int maxEntries) {
	return wf_align(numPaths * 4) + 2 * wf_align(numPaths * size_t(maxEntries) * 16) + wf_align(numPaths * 16);
}

cudaError_t launch_adjoint_wavefront(const DScene& S, const PtParams& P, uint64_t* rng, uint32_t width, uint32_t height,
                                     WfState W, void* adjointMemory, int maxEntries, const AdjointTargets& T,
                                     const float* imageGrad, float scale, TraceCounters* counters, cudaStream_t stream,
                                     const WfTuning& tuning) {
	const uint32_t n = width * height;
	if(n == 0) return cudaSuccess;
	AdjointState A;
	A.texIndex = T.texIndex;
	A.numPaths = n;
	A.maxEntries = uint32_t(maxEntries);
	char* m = static_cast<char*>(adjointMemory);
	A.count = reinterpret_cast<int*>(m);
	m += wf_align(size_t(n) * 4);
	A.entry = reinterpret_cast<float4*>(m);
	m += wf_align(size_t(n) * maxEntries * 16);
	A.suffix = reinterpret_cast<float4*>(m);
	m += wf_align(size_t(n) * maxEntries * 16);
	A.emisAcc = reinterpret_cast<float4*>(m);
	A.imageGrad = imageGrad;
	A.scale = scale;
	A.texGrad = T.texGrad;
	A.emitTarget = T.emitTarget;
	A.emisGrad = T.emisGrad;
	A.tex = DTexture{ 0, 0, nullptr };
	W.auxIter = nullptr; // no auxiliary targets in a replay
	W.guide = nullptr;
	cudaError_t e = cudaSuccess;
	if(T.texIndex >= 0) {
		e = cudaMemcpyAsync(&A.tex, S.textures + T.texIndex, sizeof(DTexture), cudaMemcpyDeviceToHost, stream);
		if(e == cudaSuccess) e = cudaStreamSynchronize(stream);
	}
	if(e == cudaSuccess) e = cudaMemsetAsync(A.count, 0, size_t(n) * 4, stream);
	if(e == cudaSuccess && T.emitTarget) e = cudaMemsetAsync(A.emisAcc, 0, size_t(n) * 16, stream);
	if(e != cudaSuccess) return e;
	const int neeCount = P.neeCount > 0 ? P.neeCount : 1;
	const int maxBounces = P.maxPathLength < 1 ? 1 : P.maxPathLength;
	const unsigned workSlots = WF_COUNTERS - WF_BOUNCE_STATS - C_WORK;
	const unsigned firstClear = unsigned(2 * maxBounces) < workSlots ? unsigned(2 * maxBounces) : workSlots;
	if((e = cudaMemsetAsync(W.counters, 0, sizeof(unsigned) * (C_WORK + firstClear), stream)) != cudaSuccess) return e;
	W.rng = rng;
	const unsigned grid = (n + 127) / 128;
	k_camera<<<grid, 128, 0, stream>>>(S, P, W, n, width);
	OneSceneAdjoint one;
	one.S = S;
	one.P = P;
	one.A = A;
	WfLaunchInfo none;
	LaunchLog log{ none, stream };
	WfTuning t = tuning;
	t.tailBounce = -1;
	t.alpha = S.hasAlpha != 0;
	run_bounces(one, W, counters, n, maxBounces, neeCount, t, log, stream);
	k_adjoint_scatter<<<grid, 128, 0, stream>>>(A);
	return cudaGetLastError();
}

void prepare_batch_kernels(const WfTuning& tuning) {
	(void)trace_kernel<JobScenes>(tuning.traceBlocksPerSm, tuning.counters, tuning.alpha);
	(void)tail_kernel<JobScenes>(tuning.counters, tuning.alpha);
	(void)trace_kernel<OneScene>(tuning.traceBlocksPerSm, tuning.counters, tuning.alpha);
	(void)tail_kernel<OneScene>(tuning.counters, tuning.alpha);
}

cudaError_t launch_trace_rays_wide(const DScene& S, const float* rays, const float* geoNormals, float tmax, uint32_t n,
                                  float* t, int32_t* inst, int32_t* prim, float* sp, cudaStream_t stream) {
	if(n == 0) return cudaSuccess;
	const unsigned blocks = unsigned(std::min<uint32_t>((n + 127) / 128, 148u * 16u));
	k_trace_rays_wide<<<blocks, 128, 0, stream>>>(S, rays, geoNormals, tmax, n, t, inst, prim, sp);
	return cudaGetLastError();
}

cudaError_t launch_occlusion_wide(const DScene& S, const float* a, const float* b, uint32_t n, uint8_t* out,
                                 cudaStream_t stream) {
	if(n == 0) return cudaSuccess;
	const unsigned blocks = unsigned(std::min<uint32_t>((n + 127) / 128, 148u * 16u));
	k_occlusion_wide<<<blocks, 128, 0, stream>>>(S, a, b, n, out);
	return cudaGetLastError();
}

cudaError_t launch_pt_wavefront(const DScene& S, const PtParams& P, const RenderState& R, WfState W,
                                TraceCounters* counters, cudaStream_t stream, WfLaunchInfo* info, const WfTuning& tuning) {
	WfLaunchInfo none;
	WfLaunchInfo& L = info ? *info : none;
	L.pairsUsed = 0;
	L.launches = 0;
	LaunchLog log{ L, stream };
	const uint32_t n = R.width * R.height;
	if(n == 0) return cudaSuccess;
	const int neeCount = P.neeCount > 0 ? P.neeCount : 1;
	const int maxBounces = P.maxPathLength < 1 ? 1 : P.maxPathLength;
	const unsigned workSlots = WF_COUNTERS - WF_BOUNCE_STATS - C_WORK;
	const unsigned firstClear = unsigned(2 * maxBounces) < workSlots ? unsigned(2 * maxBounces) : workSlots;
	cudaError_t e = cudaMemsetAsync(W.counters, 0, sizeof(unsigned) * (C_WORK + firstClear), stream);
	if(e == cudaSuccess)
		e = cudaMemsetAsync(W.counters + WF_COUNTERS - WF_BOUNCE_STATS, 0, sizeof(unsigned) * WF_BOUNCE_STATS, stream);
	if(e != cudaSuccess) return e;
	W.rng = R.rngState;
	const unsigned grid = (n + 127) / 128;
	log.begin(WF_CAMERA);
	k_camera<<<grid, 128, 0, stream>>>(S, P, W, n, R.width);
	log.end();
	OneScene one;
	one.S = S;
	one.P = P;
	WfTuning t = tuning;
	t.alpha = S.hasAlpha != 0;
	run_bounces(one, W, counters, n, maxBounces, neeCount, t, log, stream);
	log.begin(WF_FINALIZE);
	k_finalize<<<grid, 128, 0, stream>>>(W, R, n);
	log.end();
	return cudaGetLastError();
}

cudaError_t launch_pt_batch(const DJob* jobs, const uint16_t* pathJob, uint32_t numPixels, int iteration,
                            int maxBounces, int neeCount, WfState W, TraceCounters* counters, cudaStream_t stream,
                            const WfTuning& tuning, WfLaunchInfo* info) {
	WfLaunchInfo none;
	WfLaunchInfo& L = info ? *info : none;
	L.pairsUsed = 0;
	L.launches = 0;
	LaunchLog log{ L, stream };
	if(numPixels == 0) return cudaSuccess;
	if(neeCount < 1) neeCount = 1;
	if(maxBounces < 1) maxBounces = 1;
	W.auxIter = nullptr; // batches render Radiance and Hit ID only
	W.guide = nullptr;
	const unsigned workSlots = WF_COUNTERS - WF_BOUNCE_STATS - C_WORK;
	const unsigned firstClear = unsigned(2 * maxBounces) < workSlots ? unsigned(2 * maxBounces) : workSlots;
	cudaError_t e = cudaMemsetAsync(W.counters, 0, sizeof(unsigned) * (C_WORK + firstClear), stream);
	if(e == cudaSuccess)
		e = cudaMemsetAsync(W.counters + WF_COUNTERS - WF_BOUNCE_STATS, 0, sizeof(unsigned) * WF_BOUNCE_STATS, stream);
	if(e != cudaSuccess) return e;
	const unsigned grid = (numPixels + 127) / 128;
	log.begin(WF_CAMERA);
	k_camera_batch<<<grid, 128, 0, stream>>>(jobs, W, pathJob, numPixels, iteration);
	log.end();
	JobScenes js;
	js.jobs = jobs;
	js.pathJob = pathJob;
	run_bounces(js, W, counters, numPixels, maxBounces, neeCount, tuning, log, stream);
	log.begin(WF_FINALIZE);
	k_finalize_batch<<<grid, 128, 0, stream>>>(jobs, W, pathJob, numPixels, iteration);
	log.end();
	return cudaGetLastError();
}

} // namespace mb
