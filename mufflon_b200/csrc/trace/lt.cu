// Light tracer (the CUDA "Lighttracer" of the C API).
//
// One thread follows one photon per iteration, as lt_sample does
// (src/core/renderer/lt/lt_common.hpp:19-77): a start point on a light is
// drawn from the light tree by flux, every vertex of the random walk (the
// light vertex included) is connected to the pinhole camera with a shadow ray,
// and a visible connection adds its radiance to the pixel the camera sees it
// in. Photons are handed out to persistent warps from an atomic counter (the
// reference's gpu_lt.cu:20-67 hands out 8x4 tiles to whole warps); here a
// lane takes a new photon as soon as its own ends. Closest-hit and shadow
// rays use the 8-wide hierarchies with the local-memory stack of the
// wavefront path tracer. The contributions go to an
// iteration buffer with vector atomics (radiance and lightness in one float4),
// and a second kernel folds that buffer into the running means.
#include "accumulate.cuh"
#include "shading.cuh"
#include "wide_traverse.cuh"
#include "ray_queue.cuh"
#include "emit.cuh"
#include "lt_api.hpp"

#include <algorithm>

namespace mb {
namespace {

enum LtPhase { PH_IDLE = 0, PH_CONNECT = 1, PH_EXTEND = 2, PH_EXIT = 3 };

// The state of one photon's current path vertex.
struct Photon {
	f3 throughput, position, normal, intensity, incEnc;
	TangentSpace ts;
	Params mat;
	int kind, pathLen;
	uint32_t photon;
	u64 rng;
};

// lt_common.hpp:19-37: the start vertex on a light. The generator draws, in
// order, the position numbers, the light-tree seed and the camera's number.
static __device__ __noinline__ bool lt_emit(const DScene& S, Photon& ph, uint32_t numPhotons) {
	ph.throughput = make3(1.0f, 1.0f, 1.0f);
	const u64 r0 = pcg_next(ph.rng);
	const float su0 = sample_uniform(uint32_t(r0)), su1 = sample_uniform(uint32_t(r0 >> 32));
	const u64 treeSeed = pcg_next(ph.rng);
	const Emitter em = lights_emit(S, ph.photon, numPhotons, treeSeed, su0, su1);
	(void)pcg_next(ph.rng); // create_camera consumes one number (unused by the pinhole camera)
	ph.kind = em.kind;
	ph.position = em.position;
	ph.normal = em.normal;
	ph.intensity = em.intensity;
	ph.incEnc = make3(0.0f, 0.0f, 0.0f);
	ph.pathLen = 0;
	return em.valid;
}

MBD f3 vertex_geo_normal(const Photon& ph) {
	return ph.kind == LV_SURFACE ? ph.ts.geoN : (ph.kind == LV_AREA ? ph.normal : make3(0.0f, 0.0f, 0.0f));
}


// lt_common.hpp:39-72: the connection of the current vertex to the camera.
// Returns true with the shadow ray and the terms it adds when it needs an
// occlusion test.
static __device__ __noinline__ bool lt_connect(const DScene& S, const LtTargets& T, const Photon& ph, f3& so, f3& sd, float& stmax,
                    uint32_t& pix, float4& add, float& dens) {
	const f3 camPos = lv(S.camera.position);
	// get_connection(camera, vertex) (path_util.hpp:384-403); an environment
	// vertex has no position: the connection is its direction at distance 1
	f3 dir;
	float distSq;
	if(ph.kind == LV_ENV) {
		dir = -ph.normal;
		distSq = 1.0f;
	} else {
		const f3 c = ph.position - camPos;
		distSq = lensq(c);
		const float dist = sqrt_(distSq);
		dir = make3(sdiv(c.x, dist), sdiv(c.y, dist), sdiv(c.z, dist));
	}
	int px, py;
	float w;
	if(!pinhole_project(S.camera, dir, px, py, w)) return false;
	// vertex.evaluate(-dir, adjoint) (path_util.hpp:245-293, lights.hpp:263-293)
	const f3 ex = -dir;
	f3 lvalue = make3(0.0f, 0.0f, 0.0f);
	float lcos = 0.0f;
	if(ph.kind == LV_POINT || ph.kind == LV_ENV) { lvalue = ph.intensity; lcos = 1.0f; }
	else if(ph.kind == LV_AREA) { const float co = dot(ph.normal, ex); if(co > 0.0f) { lvalue = ph.intensity; lcos = co; } }
	else { const EvalValue ev = material_evaluate(ph.ts, ph.mat, decode_incident(ph.incEnc), ex, true); lvalue = ev.value; lcos = ev.cosOut; }
	f3 bxdfProd = make3(w, w, w) * lvalue;
	const float cosProd = 1.0f * lcos;
	if(!(T.density || (any_pos(bxdfProd) && cosProd > 0.0f))) return false;
	// the environment vertex is placed the maximum scene size away (path_util.hpp:130-137)
	const f3 vpos = ph.kind == LV_ENV ? camPos - decode_incident(ph.normal) * MAX_SCENE_SIZE : ph.position;
	shadow_ray(camPos, vpos, make3(0.0f, 0.0f, 0.0f), vertex_geo_normal(ph), dir, so, sd, stmax);
	bxdfProd = bxdfProd / distSq;
	const f3 rad = (ph.throughput * cosProd) * bxdfProd;
	const float light = __fdiv_rn((ph.throughput.x + ph.throughput.y) + ph.throughput.z, 3.0f) * cosProd;
	dens = 0.0f;
	if(T.density) {
		dens = __fdiv_rn(w * 1.0f, distSq);
		const float gf = ph.kind == LV_SURFACE ? dot(dir, ph.ts.shadingN)
		               : ph.kind == LV_AREA ? dot(dir, ph.normal) : ph.kind == LV_ENV ? 1.0f : 0.0f;
		dens *= fabsf(gf);
	}
	add = make_float4(nan_to_zero(rad.x), nan_to_zero(rad.y), nan_to_zero(rad.z), nan_to_zero(light));
	dens = nan_to_zero(dens);
	pix = uint32_t(py) * T.width + uint32_t(px);
	return true;
}

// random_walk.hpp:38-75 (Russian roulette always on): the next direction
// and throughput; false when the path ends here. The ray origin is offset.
static __device__ __noinline__ bool lt_walk(const DScene& S, Photon& ph, f3& origin, f3& excident) {
	const u64 x0 = pcg_next(ph.rng), x1 = pcg_next(ph.rng);
	const float ru0 = sample_uniform(uint32_t(x0)), ru1 = sample_uniform(uint32_t(x0 >> 32));
	const float rr = sample_uniform(uint32_t(pcg_next(ph.rng)));
	f3 sThroughput;
	f3 start = ph.position;
	if(ph.kind == LV_POINT) {
		// sample_light_dir_point (light_sampling.hpp:85-89)
		excident = sample_dir_sphere_uniform(ru0, ru1);
		sThroughput = (ph.intensity * 4.0f) * PI;
	} else if(ph.kind == LV_AREA) {
		// sample_light_dir_area (light_sampling.hpp:197-210)
		const f3 d = sample_dir_cosine(ru0, ru1);
		const f3 tx = normalize(perpendicular(ph.normal));
		const f3 ty = cross(ph.normal, tx);
		excident = (d.x * tx + d.y * ty) + d.z * ph.normal;
		sThroughput = ph.intensity * PI;
	} else if(ph.kind == LV_ENV) {
		// path_util.hpp:312-320: a start point on the scene box, travelling along the photon's direction
		float pdf;
		start = sample_position(S, ph.normal, ru0, ru1, pdf);
		excident = ph.normal;
		sThroughput = ph.intensity / pdf;
	} else {
		const PathSample smp = material_sample(ph.ts, ph.mat, decode_incident(ph.incEnc), ru0, ru1, x1, true);
		if(!smp.valid) return false;
		excident = smp.excident;
		sThroughput = smp.throughput;
	}
	ph.throughput = ph.throughput * sThroughput;
	const float cp = fmin_(maxc(ph.throughput) + 0.1f, 1.0f);
	if(rr >= cp) return false;
	ph.throughput = ph.throughput / cp;
	origin = start;
	add_epsilon(origin, excident, vertex_geo_normal(ph));
	return true;
}

// (lt_emit, lt_connect and lt_walk are out of line: once per vertex, they
// would otherwise crowd the traversal loop out of the instruction cache; 3 %
// faster on the instanced scene.)
// lt_common.hpp:19-77 as a per-lane state machine: a lane takes a new photon
// as soon as its photon ends (the warp claims all its idle lanes' photons with
// one atomic), and every pass of the loop traces at most one ray per lane
// (the camera connection's shadow ray or the walk's extension ray) in one
// traversal loop shared by the warp. Each photon still draws its random
// numbers in lt_sample's order. Register budget: 6 resident blocks of 128
// threads (80 registers, some spilled to L1) measured fastest on the 1080p
// headline scene: 616 Mrays/s against 588 with 5 blocks, 559 with 4, and 3
// blocks without spills slower still.
template < int AM >
__global__ void __launch_bounds__(128, 6) k_lt(const DScene S, const LtParams P, const LtTargets T,
                                            unsigned int* workCounter, TraceCounters* counters) {
	LocalStack stack;
	LocalCounters cnt;
	const unsigned lane = threadIdx.x & 31u;
	const uint32_t n = T.width * T.height;
	const uint32_t maxL = uint32_t(P.maxPathLength > 0 ? P.maxPathLength : 1);
	Photon ph;
	ph.photon = 0; ph.rng = 0; ph.pathLen = 0; ph.kind = LV_POINT;
	int phase = PH_IDLE;
	for(;;) {
		const unsigned idle = __ballot_sync(0xffffffffu, phase == PH_IDLE);
		if(idle) {
			const int leader = __ffs(idle) - 1;
			unsigned base = 0;
			if(int(lane) == leader) base = atomicAdd(workCounter, unsigned(__popc(idle)));
			base = __shfl_sync(0xffffffffu, base, leader);
			if(phase == PH_IDLE) {
				const uint32_t photon = base + unsigned(__popc(idle & ((1u << lane) - 1u)));
				if(photon >= n) phase = PH_EXIT;
				else {
					ph.photon = photon;
					ph.rng = T.rngState[photon];
					if(lt_emit(S, ph, n)) phase = PH_CONNECT;
					else T.rngState[photon] = ph.rng;
				}
			}
		}
		if(__all_sync(0xffffffffu, phase == PH_EXIT)) break;
		// one ray per lane: the camera connection, else the walk's next segment
		bool trace = false, shadow = false;
		f3 ro = make3(0.0f, 0.0f, 0.0f), rd = make3(0.0f, 0.0f, 1.0f);
		float tmax = 0.0f;
		uint32_t pix = 0;
		float4 add = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
		float dens = 0.0f;
		if(phase == PH_CONNECT) {
			if(ph.pathLen + 1 >= P.minPathLength && ph.pathLen + 1 <= P.maxPathLength)
				trace = shadow = lt_connect(S, T, ph, ro, rd, tmax, pix, add, dens);
			phase = PH_EXTEND;
		}
		if(!trace && phase == PH_EXTEND) {
			if(lt_walk(S, ph, ro, rd)) { trace = true; tmax = MAX_SCENE_SIZE; }
			else { T.rngState[ph.photon] = ph.rng; phase = PH_IDLE; }
		}
		if(trace) {
			++cnt.rays;
			if(shadow) ++cnt.shadow;
			WideTracerT<AM> t;
			t.init(S, ro, rd, tmax, shadow, cnt);
			while(!t.step(S, cnt, stack)) {}
			if(shadow) {
				if(!t.occluded) {
					atomicAdd(T.iter + pix, add);
					if(T.density) atomicAdd(T.iterDensity + pix, dens);
					if(T.recPixel) {
						const size_t slot = size_t(ph.photon) * maxL + size_t(ph.pathLen);
						T.recPixel[slot] = int(pix);
						float* o = T.recValue + 5 * slot;
						o[0] = add.x; o[1] = add.y; o[2] = add.z; o[3] = add.w; o[4] = dens;
					}
				}
			} else if(!t.best.has) {
				T.rngState[ph.photon] = ph.rng;
				phase = PH_IDLE;
			} else {
				const Intersection hit = hit_attributes(S, ro, rd, t.best);
				ph.position = ro + rd * hit.distance;
				ph.ts = tangent_space(S, hit);
				ph.mat = fetch_material(S, material_index(S, hit.inst, hit.prim), hit.uv);
				ph.incEnc = make3(rd.x, rd.y, hit.distance * sgn(rd.z));
				ph.kind = LV_SURFACE;
				++ph.pathLen;
				if(ph.pathLen < P.maxPathLength) phase = PH_CONNECT;
				else { T.rngState[ph.photon] = ph.rng; phase = PH_IDLE; }
			}
		}
	}
	unsigned long long rays = cnt.rays, shadowRays = cnt.shadow, nodes = cnt.nodes, prims = cnt.prims, inst = cnt.instances;
	unsigned errs = cnt.errors;
	for(int o = 16; o > 0; o >>= 1) {
		rays += __shfl_down_sync(0xffffffffu, rays, o);
		shadowRays += __shfl_down_sync(0xffffffffu, shadowRays, o);
		nodes += __shfl_down_sync(0xffffffffu, nodes, o);
		prims += __shfl_down_sync(0xffffffffu, prims, o);
		inst += __shfl_down_sync(0xffffffffu, inst, o);
		errs += __shfl_down_sync(0xffffffffu, errs, o);
	}
	if(lane == 0) {
		atomicAdd(&counters->rays, rays);
		atomicAdd(&counters->shadowRays, shadowRays);
		atomicAdd(&counters->nodeVisits, nodes);
		atomicAdd(&counters->primTests, prims);
		atomicAdd(&counters->instanceVisits, inst);
		if(errs) atomicAdd(&counters->errors, errs);
	}
}

// ---------------------------------------------------------------- wavefront schedule
// The light tracer in stages, like the path tracer's wavefront: a start
// launch emits every photon, connects its light vertex to the camera and
// queues the first segment of its walk; then, per path length, a trace launch
// runs the queued segments (closest hit) and camera connections (any hit,
// adding visible ones to their pixels) and a shade launch turns each hit into
// the next vertex: its camera connection and the next segment. Every photon
// draws its random numbers in lt_sample's order, so the connections (their
// pixels and values, and the records) are the single kernel's bit for bit;
// only the order of the atomic additions into the image differs.
//
// Queue state (LtwState) lives in one device allocation carved by ltw_carve.
enum { LTW_EXT0 = 0, LTW_SH0 = 2, LTW_WORK = 4 };
// Resident blocks of 128 threads per SM the trace stage is compiled for: 5
// measured fastest on the 1080p headline scene (1 063 Mrays/s; 6: 1 048,
// 8: 975).
constexpr int LTW_TRACE_BLOCKS = 5;
// ... and the shade stage (its grid is this many blocks per SM): 8 (64
// registers, no spills) measured 1 059 Mrays/s, 12 (42 registers) 992.
constexpr int LTW_SHADE_BLOCKS = 8;
constexpr int LTW_COUNTERS = 4 + 2 * LTW_MAX_LAUNCHES;

struct LtwState {
	float4* thr;        // per photon: throughput xyz, path length (int bits) in w
	int* qPhoton[2];    // segment queues (double buffered by path length)
	float4* qOrg[2];    // origin (offset)
	float4* qDir[2];    // direction
	float4* qHit[2];    // t, instance bits, primitive bits, surface u
	float* qHitV[2];    // surface v
	float4* sOrg;       // camera connections: origin, length
	float4* sDir;       // direction, density
	float4* sAdd;       // radiance rgb, lightness
	uint2* sMeta;       // pixel, record slot
	unsigned* counters; // LTW_COUNTERS
};

MBD void ltw_queue_connection(const LtwState& W, int gen, f3 so, f3 sd, float stmax, uint32_t pix, float4 add, float dens,
                              uint32_t slot) {
	const unsigned i = queue_reserve(W.counters + LTW_SH0 + (gen & 1));
	W.sOrg[i] = make_float4(so.x, so.y, so.z, stmax);
	W.sDir[i] = make_float4(sd.x, sd.y, sd.z, dens);
	W.sAdd[i] = add;
	W.sMeta[i] = make_uint2(pix, slot);
}

MBD void ltw_queue_segment(const LtwState& W, int gen, uint32_t photon, f3 o, f3 d) {
	const int q = gen & 1;
	const unsigned i = queue_reserve(W.counters + LTW_EXT0 + q);
	W.qPhoton[q][i] = int(photon);
	W.qOrg[q][i] = make_float4(o.x, o.y, o.z, 0.0f);
	W.qDir[q][i] = make_float4(d.x, d.y, d.z, 0.0f);
}

// connection and walk of vertex ph (generation gen: the queues its rays go to)
MBD void ltw_vertex(const DScene& S, const LtParams& P, const LtTargets& T, const LtwState& W, Photon& ph, int gen,
                    uint32_t maxL) {
	if(ph.pathLen + 1 >= P.minPathLength && ph.pathLen + 1 <= P.maxPathLength) {
		f3 so, sd;
		float stmax, dens;
		uint32_t pix;
		float4 add;
		if(lt_connect(S, T, ph, so, sd, stmax, pix, add, dens))
			ltw_queue_connection(W, gen, so, sd, stmax, pix, add, dens, ph.photon * maxL + uint32_t(ph.pathLen));
	}
	f3 o, d;
	if(lt_walk(S, ph, o, d)) {
		ltw_queue_segment(W, gen, ph.photon, o, d);
		W.thr[ph.photon] = make_float4(ph.throughput.x, ph.throughput.y, ph.throughput.z, __int_as_float(ph.pathLen));
	}
	T.rngState[ph.photon] = ph.rng;
}

// Every photon: emission, the light vertex's connection and first segment
// (generation 0).
__global__ void k_ltw_start(const DScene S, const LtParams P, const LtTargets T, LtwState W) {
	const uint32_t n = T.width * T.height;
	const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
	if(p >= n) return;
	const uint32_t maxL = uint32_t(P.maxPathLength > 0 ? P.maxPathLength : 1);
	Photon ph;
	ph.photon = p;
	ph.rng = T.rngState[p];
	if(!lt_emit(S, ph, n)) { T.rngState[p] = ph.rng; return; }
	ltw_vertex(S, P, T, W, ph, 0, maxL);
}

// Generation gen: the segments of queue gen & 1 (closest hit) and the camera
// connections counted in LTW_SH0 + (gen & 1) (any hit), taken by persistent
// warps 32 items at a time once all their lanes are idle.
template < int AM >
__global__ void __launch_bounds__(128, LTW_TRACE_BLOCKS) k_ltw_trace(const DScene S, const LtParams P, const LtTargets T, LtwState W,
                                                   int gen, TraceCounters* counters) {
	const int q = gen & 1;
	if(blockIdx.x == 0 && threadIdx.x == 0) {
		W.counters[LTW_EXT0 + (q ^ 1)] = 0u; // filled by this generation's shade
		W.counters[LTW_SH0 + (q ^ 1)] = 0u;
	}
	RayQueue Q;
	Q.org = W.qOrg[q]; Q.dir = W.qDir[q]; Q.hit = W.qHit[q]; Q.hitV = W.qHitV[q];
	Q.sOrg = W.sOrg; Q.sDir = W.sDir;
	Q.nExt = *reinterpret_cast<volatile unsigned*>(W.counters + LTW_EXT0 + q);
	Q.nSh = *reinterpret_cast<volatile unsigned*>(W.counters + LTW_SH0 + q);
	Q.work = W.counters + LTW_WORK + gen;
	trace_ray_queue<AM>(S, Q, counters, [&](unsigned s, bool occluded) {
		if(occluded) return;
		const float4 add = __ldcs(W.sAdd + s);
		const uint2 meta = __ldcs(W.sMeta + s);
		atomicAdd(T.iter + meta.x, add);
		const float dens = __ldcs(W.sDir + s).w;
		if(T.density) atomicAdd(T.iterDensity + meta.x, dens);
		if(T.recPixel) {
			T.recPixel[meta.y] = int(meta.x);
			float* o = T.recValue + 5 * size_t(meta.y);
			o[0] = add.x; o[1] = add.y; o[2] = add.z; o[3] = add.w; o[4] = dens;
		}
	});
}

// Generation gen: each traced segment of queue gen & 1 that hit a surface
// becomes the photon's next vertex (lt_sample's loop body); its connection
// and next segment go to generation gen + 1.
__global__ void __launch_bounds__(128, LTW_SHADE_BLOCKS) k_ltw_shade(const DScene S, const LtParams P, const LtTargets T, LtwState W, int gen) {
	const int q = gen & 1;
	const unsigned count = *reinterpret_cast<volatile unsigned*>(W.counters + LTW_EXT0 + q);
	const uint32_t maxL = uint32_t(P.maxPathLength > 0 ? P.maxPathLength : 1);
	for(unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
		const float4 hh = __ldcs(W.qHit[q] + i);
		const int hitInst = __float_as_int(hh.y);
		if(hitInst < 0) continue; // the photon left the scene (its generator is stored)
		const uint32_t p = uint32_t(__ldcs(W.qPhoton[q] + i));
		const f3 ro = f4to3(__ldcs(W.qOrg[q] + i)), rd = f4to3(__ldcs(W.qDir[q] + i));
		HitRec hr;
		hr.t = hh.x; hr.inst = hitInst; hr.prim = __float_as_int(hh.z);
		hr.sp = make2(hh.w, __ldcs(W.qHitV[q] + i));
		hr.has = true;
		const float4 tp = W.thr[p];
		Photon ph;
		ph.photon = p;
		ph.rng = T.rngState[p];
		ph.throughput = f4to3(tp);
		ph.pathLen = __float_as_int(tp.w);
		const Intersection hit = hit_attributes(S, ro, rd, hr);
		ph.position = ro + rd * hit.distance;
		ph.ts = tangent_space(S, hit);
		ph.mat = fetch_material(S, material_index(S, hit.inst, hit.prim), hit.uv);
		ph.incEnc = make3(rd.x, rd.y, hit.distance * sgn(rd.z));
		ph.kind = LV_SURFACE;
		ph.normal = make3(0.0f, 0.0f, 0.0f);
		ph.intensity = make3(0.0f, 0.0f, 0.0f);
		++ph.pathLen;
		if(ph.pathLen < P.maxPathLength) ltw_vertex(S, P, T, W, ph, gen + 1, maxL);
	}
}

int ltw_trace_blocks() {
	static int blocks = 0;
	if(blocks == 0) {
		int dev = 0, sms = 148, a = 0, b = 0;
		cudaGetDevice(&dev);
		cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
		cudaOccupancyMaxActiveBlocksPerMultiprocessor(&a, k_ltw_trace<ALPHA_NEVER>, 128, 0);
		cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_ltw_trace<ALPHA_ALWAYS>, 128, 0);
		blocks = sms * std::max(1, std::min(a, b));
	}
	return blocks;
}

size_t ltw_size(size_t n) {
	auto al = [](size_t b) { return (b + 255) & ~size_t(255); };
	return al(n * 16) + 2 * (al(n * 4) + 3 * al(n * 16) + al(n * 4)) + 3 * al(n * 16) + al(n * 8) +
	       al(LTW_COUNTERS * sizeof(unsigned));
}

LtwState ltw_carve(void* memory, size_t n) {
	auto al = [](size_t b) { return (b + 255) & ~size_t(255); };
	char* m = static_cast<char*>(memory);
	auto take = [&](size_t b) { char* r = m; m += al(b); return r; };
	LtwState W;
	W.thr = reinterpret_cast<float4*>(take(n * 16));
	for(int q = 0; q < 2; ++q) {
		W.qPhoton[q] = reinterpret_cast<int*>(take(n * 4));
		W.qOrg[q] = reinterpret_cast<float4*>(take(n * 16));
		W.qDir[q] = reinterpret_cast<float4*>(take(n * 16));
		W.qHit[q] = reinterpret_cast<float4*>(take(n * 16));
		W.qHitV[q] = reinterpret_cast<float*>(take(n * 4));
	}
	W.sOrg = reinterpret_cast<float4*>(take(n * 16));
	W.sDir = reinterpret_cast<float4*>(take(n * 16));
	W.sAdd = reinterpret_cast<float4*>(take(n * 16));
	W.sMeta = reinterpret_cast<uint2*>(take(n * 8));
	W.counters = reinterpret_cast<unsigned*>(take(LTW_COUNTERS * sizeof(unsigned)));
	return W;
}

// output_handler_variance.hpp:7-31: running means and variances; Density
// reduces moments (render_targets.hpp:68-74): its target holds the
// iteration's value and its variance slot the running mean.
__global__ void k_lt_finalize(LtTargets T) {
	const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
	if(p >= T.width * T.height) return;
	const float4 it = T.iter[p];
	if(T.radiance) {
		float* cr = T.radiance + 3 * size_t(p);
		float* vr = T.radianceVar ? T.radianceVar + 3 * size_t(p) : nullptr;
		const float v[3] = { it.x, it.y, it.z };
		for(int c = 0; c < 3; ++c) update_moments(v[c], cr + c, vr ? vr + c : nullptr, T.iteration);
	}
	if(T.lightness) update_moments(it.w, T.lightness + p, T.lightnessVar ? T.lightnessVar + p : nullptr, T.iteration);
	if(T.density) update_reduced(T.iterDensity[p], T.density + p, T.densityMean ? T.densityMean + p : nullptr, T.iteration);
}

int lt_blocks() {
	static int blocks = 0;
	if(blocks == 0) {
		int dev = 0, sms = 148, perSm = 0;
		cudaGetDevice(&dev);
		cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
		// both variants (scenes with and without alpha textures) fit as many blocks
		int perSmAlpha = 0;
		cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, k_lt<ALPHA_NEVER>, 128, 0);
		cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSmAlpha, k_lt<ALPHA_ALWAYS>, 128, 0);
		if(perSmAlpha > perSm) perSm = perSmAlpha;
		blocks = sms * (perSm > 0 ? perSm : 1);
	}
	return blocks;
}

} // namespace

size_t ltw_bytes(size_t numPhotons) { return ltw_size(numPhotons); }

cudaError_t launch_lt(const DScene& S, const LtParams& P, const LtTargets& T, unsigned int* workCounter,
                      TraceCounters* counters, cudaStream_t stream, void* wavefront) {
	const uint32_t n = T.width * T.height;
	if(n == 0) return cudaSuccess;
	cudaError_t e;
	if((e = cudaMemsetAsync(T.iter, 0, size_t(n) * sizeof(float4), stream)) != cudaSuccess) return e;
	if(T.density && (e = cudaMemsetAsync(T.iterDensity, 0, size_t(n) * sizeof(float), stream)) != cudaSuccess) return e;
	if(T.recPixel) {
		const size_t slots = size_t(n) * size_t(P.maxPathLength > 0 ? P.maxPathLength : 1);
		if((e = cudaMemsetAsync(T.recPixel, 0xFF, slots * sizeof(int32_t), stream)) != cudaSuccess) return e;
		if((e = cudaMemsetAsync(T.recValue, 0, slots * 5 * sizeof(float), stream)) != cudaSuccess) return e;
	}
	if(wavefront) {
		const LtwState W = ltw_carve(wavefront, n);
		const int gens = P.maxPathLength > 0 ? P.maxPathLength : 1;
		if(gens > LTW_MAX_LAUNCHES) return cudaErrorInvalidValue;
		if((e = cudaMemsetAsync(W.counters, 0, LTW_COUNTERS * sizeof(unsigned), stream)) != cudaSuccess) return e;
		k_ltw_start<<<(n + 127) / 128, 128, 0, stream>>>(S, P, T, W);
		const int tb = ltw_trace_blocks();
		int dev = 0, sms = 148;
		cudaGetDevice(&dev);
		cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
		// generation g: the connections of path length g and the segments reaching path length g + 1
		for(int g = 0; g < gens; ++g) {
			if(S.hasAlpha) k_ltw_trace<ALPHA_ALWAYS><<<tb, 128, 0, stream>>>(S, P, T, W, g, counters);
			else k_ltw_trace<ALPHA_NEVER><<<tb, 128, 0, stream>>>(S, P, T, W, g, counters);
			if(g + 1 < gens) k_ltw_shade<<<sms * LTW_SHADE_BLOCKS, 128, 0, stream>>>(S, P, T, W, g);
		}
	} else {
		if((e = cudaMemsetAsync(workCounter, 0, sizeof(unsigned int), stream)) != cudaSuccess) return e;
		// the variant for the scene: alpha textures or none (no alpha code in the loop)
		if(S.hasAlpha) k_lt<ALPHA_ALWAYS><<<lt_blocks(), 128, 0, stream>>>(S, P, T, workCounter, counters);
		else k_lt<ALPHA_NEVER><<<lt_blocks(), 128, 0, stream>>>(S, P, T, workCounter, counters);
	}
	if((e = cudaGetLastError()) != cudaSuccess) return e;
	k_lt_finalize<<<(n + 255) / 256, 256, 0, stream>>>(T);
	return cudaGetLastError();
}

} // namespace mb
