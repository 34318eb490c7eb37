// Light tracer (the CUDA "Lighttracer" of the C API).
//
// One thread follows one photon per iteration, as lt_sample does
// (src/core/renderer/lt/lt_common.hpp:19-77): a start point on a light is
// drawn from the light tree by flux, every vertex of the random walk (the
// light vertex included) is connected to the pinhole camera with a shadow ray,
// and a visible connection adds its radiance to the pixel the camera sees it
// in. Photons are handed out to persistent warps 32 at a time from an atomic
// counter (the reference's gpu_lt.cu:20-67 hands out 8x4 tiles the same
// way). Closest-hit and shadow rays use the 8-wide hierarchies with the
// local-memory stack of the wavefront path tracer. The contributions go to an
// iteration buffer with vector atomics (radiance and lightness in one float4),
// and a second kernel folds that buffer into the running means.
#include "shading.cuh"
#include "wide_traverse.cuh"
#include "lt_api.hpp"

namespace mb {
namespace {

// A photon's start on a light (light_sampling.hpp:20-49 Emitter): the
// position, the intensity divided by the probability of choosing the light
// (light_tree_sampling.hpp:12-16) and, for an area light, its normal.
struct Emitter { f3 position, intensity, normal; bool area, valid; };

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
		e.area = false;
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
	e.area = true;
	return e;
}

// light_tree_sampling.hpp:141-188 with the sub-tree descent of :81-131: the
// photon index spreads the photons evenly over the flux interval before the
// seed's random offset. Scenes with environment light are refused by the
// renderer before launch; there are no directional lights.
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
	if(rndChoice < percentage_of(~0ull, envProb)) return none;
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

enum LtKind { LV_POINT = 0, LV_AREA = 1, LV_SURFACE = 2 };

// lt_common.hpp:19-77: one photon's random walk from a light, every vertex
// connected to the camera.
template < class Stack >
MBD void lt_sample(const DScene& S, const LtParams& P, const LtTargets& T, uint32_t photon, uint32_t numPhotons,
                   u64& rng, LocalCounters& cnt, Stack& stack) {
	f3 throughput = make3(1.0f, 1.0f, 1.0f);
	const u64 r0 = pcg_next(rng);
	const float su0 = sample_uniform(uint32_t(r0)), su1 = sample_uniform(uint32_t(r0 >> 32));
	const u64 treeSeed = pcg_next(rng);
	const Emitter em = lights_emit(S, photon, numPhotons, treeSeed, su0, su1);
	(void)pcg_next(rng); // create_camera consumes one number (unused by the pinhole camera)
	if(!em.valid) return;
	int kind = em.area ? LV_AREA : LV_POINT;
	f3 position = em.position;
	const f3 normal = em.normal, intensity = em.intensity;
	TangentSpace ts;
	Params mat;
	f3 incEnc = make3(0.0f, 0.0f, 0.0f);
	const f3 camPos = lv(S.camera.position);
	const size_t rec = size_t(photon) * size_t(P.maxPathLength > 0 ? P.maxPathLength : 1);
	int pathLen = 0;
	do {
		if(pathLen + 1 >= P.minPathLength && pathLen + 1 <= P.maxPathLength) {
			// get_connection(camera, vertex) (path_util.hpp:384-403)
			const f3 c = position - camPos;
			const float distSq = lensq(c);
			const float dist = sqrt_(distSq);
			const f3 dir = make3(sdiv(c.x, dist), sdiv(c.y, dist), sdiv(c.z, dist));
			int px, py;
			float w;
			if(pinhole_project(S.camera, dir, px, py, w)) {
				// vertex.evaluate(-dir, adjoint) (path_util.hpp:245-293, lights.hpp:263-293)
				const f3 ex = -dir;
				f3 lvalue = make3(0.0f, 0.0f, 0.0f);
				float lcos = 0.0f;
				if(kind == LV_POINT) { lvalue = intensity; lcos = 1.0f; }
				else if(kind == LV_AREA) { const float co = dot(normal, ex); if(co > 0.0f) { lvalue = intensity; lcos = co; } }
				else { const EvalValue ev = material_evaluate(ts, mat, decode_incident(incEnc), ex, true); lvalue = ev.value; lcos = ev.cosOut; }
				f3 bxdfProd = make3(w, w, w) * lvalue;
				const float cosProd = 1.0f * lcos;
				if(T.density || (any_pos(bxdfProd) && cosProd > 0.0f)) {
					const f3 vGeo = kind == LV_SURFACE ? ts.geoN : (kind == LV_AREA ? normal : make3(0.0f, 0.0f, 0.0f));
					f3 so, sd;
					float stmax;
					shadow_ray(camPos, position, make3(0.0f, 0.0f, 0.0f), vGeo, dir, so, sd, stmax);
					if(!occluded_wide(S, so, sd, stmax, cnt, stack)) {
						bxdfProd = bxdfProd / distSq;
						const f3 rad = (throughput * cosProd) * bxdfProd;
						const float light = __fdiv_rn((throughput.x + throughput.y) + throughput.z, 3.0f) * cosProd;
						float dens = 0.0f;
						if(T.density) {
							dens = __fdiv_rn(w * 1.0f, distSq);
							const float gf = kind == LV_SURFACE ? dot(dir, ts.shadingN) : (kind == LV_AREA ? dot(dir, normal) : 0.0f);
							dens *= fabsf(gf);
						}
						const float4 v = make_float4(nan_to_zero(rad.x), nan_to_zero(rad.y), nan_to_zero(rad.z), nan_to_zero(light));
						const size_t pix = size_t(py) * T.width + size_t(px);
						atomicAdd(T.iter + pix, v);
						if(T.density) atomicAdd(T.iterDensity + pix, nan_to_zero(dens));
						if(T.recPixel) {
							T.recPixel[rec + pathLen] = int(pix);
							float* o = T.recValue + 5 * (rec + pathLen);
							o[0] = v.x; o[1] = v.y; o[2] = v.z; o[3] = v.w; o[4] = nan_to_zero(dens);
						}
					}
				}
			}
		}
		// walk (random_walk.hpp:38-113), Russian roulette always on
		const u64 x0 = pcg_next(rng), x1 = pcg_next(rng);
		const float ru0 = sample_uniform(uint32_t(x0)), ru1 = sample_uniform(uint32_t(x0 >> 32));
		const float rr = sample_uniform(uint32_t(pcg_next(rng)));
		f3 excident, sThroughput;
		if(kind == LV_POINT) {
			// sample_light_dir_point (light_sampling.hpp:85-89)
			excident = sample_dir_sphere_uniform(ru0, ru1);
			sThroughput = (intensity * 4.0f) * PI;
		} else if(kind == LV_AREA) {
			// sample_light_dir_area (light_sampling.hpp:197-210)
			const f3 d = sample_dir_cosine(ru0, ru1);
			const f3 tx = normalize(perpendicular(normal));
			const f3 ty = cross(normal, tx);
			excident = (d.x * tx + d.y * ty) + d.z * normal;
			sThroughput = intensity * PI;
		} else {
			const PathSample smp = material_sample(ts, mat, decode_incident(incEnc), ru0, ru1, x1, true);
			if(!smp.valid) break;
			excident = smp.excident;
			sThroughput = smp.throughput;
		}
		throughput = throughput * sThroughput;
		const float cp = fmin_(maxc(throughput) + 0.1f, 1.0f);
		if(rr >= cp) break;
		throughput = throughput / cp;
		const f3 geoN = kind == LV_SURFACE ? ts.geoN : (kind == LV_AREA ? normal : make3(0.0f, 0.0f, 0.0f));
		f3 origin = position;
		add_epsilon(origin, excident, geoN);
		const HitRec hr = closest_hit_wide(S, origin, excident, MAX_SCENE_SIZE, cnt, stack);
		if(!hr.has) break;
		const Intersection hit = hit_attributes(S, origin, excident, hr);
		position = origin + excident * hit.distance;
		ts = tangent_space(S, hit);
		mat = fetch_material(S, material_index(S, hit.inst, hit.prim), hit.uv);
		incEnc = make3(excident.x, excident.y, hit.distance * sgn(excident.z));
		kind = LV_SURFACE;
		++pathLen;
	} while(pathLen < P.maxPathLength);
}

__global__ void __launch_bounds__(128) k_lt(const DScene S, const LtParams P, const LtTargets T,
                                            unsigned int* workCounter, TraceCounters* counters) {
	LocalStack stack;
	LocalCounters cnt;
	const unsigned lane = threadIdx.x & 31u;
	const uint32_t n = T.width * T.height;
	for(;;) {
		unsigned base = 0;
		if(lane == 0) base = atomicAdd(workCounter, 32u);
		base = __shfl_sync(0xffffffffu, base, 0);
		if(base >= n) break;
		const uint32_t photon = base + lane;
		if(photon < n) {
			u64 rng = T.rngState[photon];
			lt_sample(S, P, T, photon, n, rng, cnt, stack);
			T.rngState[photon] = rng;
		}
	}
	unsigned long long rays = cnt.rays, shadow = cnt.shadow, nodes = cnt.nodes, prims = cnt.prims, inst = cnt.instances;
	unsigned errs = cnt.errors;
	for(int o = 16; o > 0; o >>= 1) {
		rays += __shfl_down_sync(0xffffffffu, rays, o);
		shadow += __shfl_down_sync(0xffffffffu, shadow, o);
		nodes += __shfl_down_sync(0xffffffffu, nodes, o);
		prims += __shfl_down_sync(0xffffffffu, prims, o);
		inst += __shfl_down_sync(0xffffffffu, inst, o);
		errs += __shfl_down_sync(0xffffffffu, errs, o);
	}
	if(lane == 0) {
		atomicAdd(&counters->rays, rays);
		atomicAdd(&counters->shadowRays, shadow);
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
