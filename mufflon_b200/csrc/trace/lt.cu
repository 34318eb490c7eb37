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
#include "shading.cuh"
#include "wide_traverse.cuh"
#include "lt_api.hpp"

namespace mb {
namespace {

enum LtKind { LV_POINT = 0, LV_AREA = 1, LV_SURFACE = 2, LV_ENV = 3 };

// A photon's start on a light (light_sampling.hpp:20-49 Emitter): the
// position, the intensity divided by the probability of choosing the light
// (light_tree_sampling.hpp:12-16) and, for an area light, its normal; for
// the environment, the direction the photon travels (in `normal`) and the
// irradiance.
struct Emitter { f3 position, intensity, normal; int kind; bool valid; };

// render_target.hpp:64-75: a NaN channel of a contribution is added as 0
MBD float nan_to_zero(float x) { return isnan(x) ? 0.0f : x; }

// A vector perpendicular to n (not normalised): n crossed with the coordinate
// axis of n's smallest component. The reference takes `perpendicular` from
// its math library (epsilon, absent); the emission lobe it orients is
// rotationally symmetric about n, so the choice of axis changes which
// direction a random number pair maps to, not the image's expectation.
MBD f3 perpendicular(f3 n) {
	const float ax = fabsf(n.x), ay = fabsf(n.y), az = fabsf(n.z);
	if(ax <= ay && ax <= az) return make3(0.0f, n.z, -n.y);
	if(ay <= az) return make3(-n.z, 0.0f, n.x);
	return make3(n.y, -n.x, 0.0f);
}

// light_sampling.hpp:80-84 (point), 117-140 (triangle), 143-171 (quad)
MBD Emitter sample_light_pos(const DScene& S, const DLight& l, float u0, float u1, float lightProb) {
	Emitter e;
	e.valid = true;
	if(l.type == LT_POINT) {
		e.position = lv(l.position);
		e.intensity = lv(l.intensity) / lightProb;
		e.normal = make3(0.0f, 0.0f, 0.0f);
		e.kind = LV_POINT;
		return e;
	}
	const DMaterial& m = S.materials[l.material];
	const f3 radiance = m.type == MAT_EMISSIVE ? load3(m.radiance) : make3(0, 0, 0);
	f3 normal, position;
	float area;
	if(l.type == LT_TRI) {
		normal = cross(lv(l.posV[1]), lv(l.posV[2]));
		const float area2 = len(normal);
		normal = normal / area2;
		area = area2 * 0.5f;
		const float bs = 1.0f - sqrt_(1.0f - u0);
		const float bt = (1.0f - bs) * u1;
		position = (lv(l.posV[0]) + lv(l.posV[1]) * bs) + lv(l.posV[2]) * bt;
	} else {
		const f3 tx = lv(l.posV[1]) + u0 * lv(l.posV[3]);
		const f3 ty = lv(l.posV[2]) + u1 * lv(l.posV[3]);
		normal = cross(ty, tx);
		area = len(normal);
		normal = normal / area;
		position = (lv(l.posV[0]) + tx * u1) + lv(l.posV[2]) * u0;
	}
	e.position = position;
	e.intensity = (radiance * area) / lightProb;
	e.normal = normal;
	e.kind = LV_AREA;
	return e;
}

// light_sampling.hpp:226-232 and 292-306 (a colored background), scaled by
// the environment's choice probability (light_tree_sampling.hpp:158-167): a
// direction drawn uniformly on the sphere; the photon travels against it.
MBD Emitter sample_background(const DScene& S, float u0, float u1, float envProb) {
	const f3 dir = sample_dir_sphere_uniform(u0, u1);
	const float dirPdf = __fdiv_rn(1.0f, 4.0f * PI);
	const f3 irradiance = (lv(S.bgColor) * lv(S.bgScale)) / dirPdf;
	Emitter e;
	e.valid = true;
	e.kind = LV_ENV;
	e.position = make3(0.0f, 0.0f, 0.0f);
	e.normal = -dir;
	e.intensity = irradiance / envProb;
	return e;
}

// light_tree_sampling.hpp:141-188 with the sub-tree descent of :81-131: the
// photon index spreads the photons evenly over the flux interval before the
// seed's random offset. There are no directional lights.
MBD Emitter lights_emit(const DScene& S, u64 index, u64 numIndices, u64 seed, float u0, float u1) {
	u64 rndChoice = numIndices > 0 ? seed + index * (~0ull / numIndices) : seed;
	if(rndChoice == ~0ull) --rndChoice;
	const float bgSum = (S.bgFlux[0] + S.bgFlux[1]) + S.bgFlux[2];
	const float fluxSum = (bgSum + S.dirFlux) + S.rootFlux;
	Emitter none;
	none.valid = false;
	if(!(fluxSum > 0.0f)) return none;
	const float envProb = __fdiv_rn(bgSum, fluxSum);
	const float dirProb = __fdiv_rn(S.dirFlux, fluxSum);
	const float posProb = __fdiv_rn(S.rootFlux, fluxSum);
	if(rndChoice < percentage_of(~0ull, envProb)) return sample_background(S, u0, u1, envProb);
	const u64 right = percentage_of(~0ull, envProb + dirProb);
	if(rndChoice < right) return none;
	u64 iL = right, iR = ~0ull;
	float lightProb = posProb;
	uint16_t type = S.rootType;
	int idx = S.rootIndex;
	int nodeIdx = 0;
	while(type == LT_INTERNAL) {
		const DLightNode& nd = S.lightNodes[nodeIdx];
		const float probLeft = __fdiv_rn(nd.leftFlux, nd.leftFlux + nd.rightFlux);
		const u64 boundary = iL + percentage_of(iR - iL, probLeft);
		if(rndChoice < boundary) { type = nd.leftType; idx = nd.leftIndex; iR = boundary; lightProb *= probLeft; }
		else { type = nd.rightType; idx = nd.rightIndex; iL = boundary; lightProb *= (1.0f - probLeft); }
		nodeIdx = idx;
	}
	return sample_light_pos(S, S.lights[idx], u0, u1, lightProb);
}

// pinhole.hpp:86-116: the pixel a direction leaving the camera falls in and
// the sensor response w (equal to the sampling pdf); false when the direction
// points behind the camera or off the image.
MBD bool pinhole_project(const DCamera& c, f3 excident, int& px, int& py, float& w) {
	const f3 view = lv(c.viewDir), up = lv(c.up);
	const float cosOut = dot(view, excident);
	if(cosOut < 0.0f) return false;
	const f3 xAxis = cross(view, up);
	const float d = cosOut * c.tanVFov;
	float ux = __fdiv_rn(dot(xAxis, excident), d);
	const float uy = __fdiv_rn(dot(up, excident), d);
	const float aspect = __fdiv_rn(float(c.resX), float(c.resY));
	ux = __fdiv_rn(ux, aspect);
	if(!(ux > -1.0f && ux <= 1.0f && uy > -1.0f && uy <= 1.0f)) return false;
	px = int(floorf((ux * 0.5f + 0.5f) * float(c.resX)));
	py = int(floorf((uy * 0.5f + 0.5f) * float(c.resY)));
	if(px >= int(c.resX)) px = int(c.resX) - 1;
	if(py >= int(c.resY)) py = int(c.resY) - 1;
	const float t2 = 2.0f * c.tanVFov;
	const float pixelArea = (t2 * t2) * aspect;
	w = __fdiv_rn(1.0f, ((pixelArea * cosOut) * cosOut) * cosOut);
	return true;
}

MBD f3 decode_incident(f3 e) {
	float t = 1.0f - e.x * e.x - e.y * e.y;
	t = fminf(fmaxf(t, 0.0f), 1.0f);
	return make3(e.x, e.y, sgn(e.z) * sqrt_(t));
}

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

// math/sampling.hpp:132-158: a start point for a photon of direction dir on
// the faces of the scene box it enters through, and the inverse of the
// box's projected area (the position pdf).
MBD f3 sample_position(const DScene& S, f3 dir, float u0, float u1, float& pdf) {
	const f3 mn = lv(S.aabbMin);
	const f3 sides = lv(S.aabbMax) - mn;
	const float projAx = (sides.y * sides.z) * fabsf(dir.x);
	const float projAy = (sides.x * sides.z) * fabsf(dir.y);
	const float projAz = (sides.x * sides.y) * fabsf(dir.z);
	const float area = (projAx + projAy) + projAz;
	float x = u0 * area;
	f3 p;
	if(x < projAx) {
		x = __fdiv_rn(x - 0.0f, projAx - 0.0f);
		p = make3(dir.x < 0.0f ? 1.0f : 0.0f, u1, x);
	} else if(x < projAx + projAy) {
		x = __fdiv_rn(x - projAx, (projAx + projAy) - projAx);
		p = make3(u1, dir.y < 0.0f ? 1.0f : 0.0f, x);
	} else {
		x = __fdiv_rn(x - (projAx + projAy), area - (projAx + projAy));
		p = make3(u1, x, dir.z < 0.0f ? 1.0f : 0.0f);
	}
	pdf = __fdiv_rn(1.0f, area);
	return (mn + p * sides) - dir * 1e-3f;
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
// numbers in lt_sample's order. Register budget: 5 resident blocks of 128
// threads (96 registers, some spilled to L1) measured faster than 3 blocks
// without spills (4.60 vs 4.95 ms per 1080p iteration).
__global__ void __launch_bounds__(128, 5) k_lt(const DScene S, const LtParams P, const LtTargets T,
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
			WideTracer t;
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

// output_handler_variance.hpp:7-31 (mean only): cum += (iter - cum) / (it + 1)
__global__ void k_lt_finalize(LtTargets T) {
	const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
	if(p >= T.width * T.height) return;
	const float den = fmaxf(1.0f, float(T.iteration) + 1.0f);
	const float4 it = T.iter[p];
	if(T.radiance) {
		float* cr = T.radiance + 3 * size_t(p);
		const float v[3] = { it.x, it.y, it.z };
		for(int c = 0; c < 3; ++c) { const float diff = v[c] - cr[c]; cr[c] += __fdiv_rn(diff, den); }
	}
	if(T.lightness) { const float diff = it.w - T.lightness[p]; T.lightness[p] += __fdiv_rn(diff, den); }
	if(T.density) { const float diff = T.iterDensity[p] - T.density[p]; T.density[p] += __fdiv_rn(diff, den); }
}

int lt_blocks() {
	static int blocks = 0;
	if(blocks == 0) {
		int dev = 0, sms = 148, perSm = 0;
		cudaGetDevice(&dev);
		cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
		cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, k_lt, 128, 0);
		blocks = sms * (perSm > 0 ? perSm : 1);
	}
	return blocks;
}

} // namespace

cudaError_t launch_lt(const DScene& S, const LtParams& P, const LtTargets& T, unsigned int* workCounter,
                      TraceCounters* counters, cudaStream_t stream) {
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
	if((e = cudaMemsetAsync(workCounter, 0, sizeof(unsigned int), stream)) != cudaSuccess) return e;
	k_lt<<<lt_blocks(), 128, 0, stream>>>(S, P, T, workCounter, counters);
	if((e = cudaGetLastError()) != cudaSuccess) return e;
	k_lt_finalize<<<(n + 255) / 256, 256, 0, stream>>>(T);
	return cudaGetLastError();
}

} // namespace mb
