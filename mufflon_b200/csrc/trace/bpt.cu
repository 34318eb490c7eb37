// Bidirectional path tracer (the CUDA "Bidirectional Pathtracer" of the C
// API). The reference has it on the CPU only (src/core/renderer/bpt/
// cpu_bpt.cpp:170-232); this is the same estimator on the GPU traversal.
//
// Per pixel and iteration: a light subpath from a light chosen through the
// light tree (as the light tracer's photons), then a view subpath from the
// camera. Every view vertex is connected to every light vertex with a shadow
// ray, and every emitter the view subpath hits counts as well; each such
// estimate is weighted by the balance heuristic over all ways the path could
// have been built, evaluated recursively from the MIS data each vertex keeps
// (BptVertexExt, cpu_bpt.cpp:18-60 and 68-115).
//
// Two schedules with the same contributions. The default runs in stages per
// path length (k_bptw_*: the light subpaths of all pixels, then the view
// subpaths, each generation one trace launch over its queued segments and
// connections and one shade launch over the vertices they reach). The other
// ("Megakernel") is one persistent kernel whose lanes run a state machine (as
// the light tracer's): a lane takes a new pixel as soon as its own finishes,
// and every pass of the loop traces at most one ray per lane (a light-subpath
// segment, a connection's shadow ray or a view-subpath segment) in one
// traversal loop shared by the warp; a lane keeps its light subpath in its
// own slice of a scratch array (max. path length vertices) and the last two
// view vertices in local memory. Connections from the camera land in other
// pixels, so all contributions go to an iteration buffer with vector atomics.
#include "accumulate.cuh"
#include "wide_traverse.cuh"
#include "ray_queue.cuh"
#include "emit.cuh"
#include "lt_api.hpp"

#include <algorithm>

namespace mb {
namespace {

enum BKind { BV_VIRTUAL = 0, BV_CAMERA, BV_SURFACE, BV_VOID, BV_POINT, BV_AREA, BV_ENV };

// A path vertex with the reference's PathVertex<BptVertexExt> contents:
// incEnc is the encoded incident direction (surfaces: x, y of the direction
// and the distance with the sign of z; a miss: the direction; an area light:
// its normal; a point light: its intensity; the environment: the photon's
// direction).
struct BV {
	int kind;
	f3 position, incEnc, intensity;
	float projSceneArea;
	TangentSpace ts;
	Params mat;
	int inst, prim;
	f2 sp;
	float incidentPdf;  // BptVertexExt::incidentPdf
	float prevRelSum;   // BptVertexExt::prevRelativeProbabilitySum
	f3 throughput;      // BptVertexExt::throughput
};

MBD bool bv_ortho(int k) { return k == BV_VOID || k == BV_ENV; } // path_util.hpp:41-46
MBD bool bv_end(int k) { return k != BV_SURFACE; }               // path_util.hpp:33-35

// path_util.hpp:160-176
MBD float bv_geo_factor(const BV& v, f3 dir) {
	if(v.kind == BV_AREA) return dot(dir, v.incEnc);
	if(v.kind == BV_SURFACE) return dot(dir, v.ts.shadingN);
	if(v.kind == BV_ENV || v.kind == BV_VOID) return 1.0f;
	return 0.0f;
}
MBD f3 bv_geo_normal(const BV& v) {
	if(v.kind == BV_AREA) return v.incEnc;
	if(v.kind == BV_SURFACE) return v.ts.geoN;
	return make3(0.0f, 0.0f, 0.0f);
}
MBD f3 bv_incident_dir(const BV& v) { return decode_incident(v.incEnc); }
MBD float bv_incident_dist_sq(const BV& v) { return bv_end(v.kind) ? 0.0f : v.incEnc.z * v.incEnc.z; }
// path_util.hpp:130-137
MBD f3 bv_position(const BV& v, f3 ref) {
	return v.kind == BV_ENV ? ref - bv_incident_dir(v) * MAX_SCENE_SIZE : v.position;
}
// path_util.hpp:208-221: a sampling pdf converted into an area pdf at v
MBD float bv_convert_pdf(const BV& v, int source, float samplePdf, f3 dir, float distSq) {
	if(source == BV_VIRTUAL) return samplePdf;
	const float geo = bv_geo_factor(v, dir);
	if(bv_ortho(source) || bv_ortho(v.kind)) return samplePdf * fabsf(geo);
	return __fdiv_rn(samplePdf * fabsf(geo), distSq);
}

// path_util.hpp:245-293: value, cosine and pdfs of leaving v along excident;
// a camera also yields the pixel (px = -1 off the image)
MBD EvalValue bv_evaluate(const DScene& S, const BV& v, f3 excident, bool adjoint, int& px, int& py) {
	EvalValue r;
	r.value = make3(0.0f, 0.0f, 0.0f); r.cosOut = 0.0f; r.pdfF = 0.0f; r.pdfB = 0.0f;
	if(v.kind == BV_POINT) { r.value = v.incEnc; r.cosOut = 1.0f; r.pdfF = __fdiv_rn(1.0f, 4.0f * PI); }
	else if(v.kind == BV_AREA) {
		const float cosOut = dot(v.incEnc, excident);
		if(cosOut > 0.0f) { r.value = v.intensity; r.cosOut = cosOut; r.pdfF = __fdiv_rn(cosOut, PI); }
	} else if(v.kind == BV_ENV) { r.value = v.intensity; r.cosOut = 1.0f; r.pdfF = __fdiv_rn(1.0f, v.projSceneArea); }
	else if(v.kind == BV_CAMERA) {
		float w = 0.0f;
		r.cosOut = 1.0f;
		if(!pinhole_project(S.camera, excident, px, py, w)) { px = -1; py = -1; }
		else { r.value = make3(w, w, w); r.pdfF = w; }
	} else if(v.kind == BV_SURFACE) r = material_evaluate(v.ts, v.mat, bv_incident_dir(v), excident, adjoint);
	return r;
}

// cpu_bpt.cpp:68-88: the relative probabilities of the events before v
MBD float bpt_mis_part(const BV& v, const BV* prev, float vertexPdfBack, float nextPdfBack, int nextType, f3 dir,
                       float distSq) {
	float reversePdf = bv_convert_pdf(v, nextType, nextPdfBack, dir, distSq);
	const float relPdf = __fdiv_rn(reversePdf, v.incidentPdf);
	if(prev) {
		reversePdf = bv_convert_pdf(*prev, v.kind, vertexPdfBack, bv_incident_dir(v), bv_incident_dist_sq(v));
		const float prevRelPdf = __fdiv_rn(reversePdf, prev->incidentPdf);
		return relPdf + relPdf * (prevRelPdf + prevRelPdf * prev->prevRelSum);
	}
	return relPdf;
}

// random_walk.hpp:38-75 for a BPT vertex: samples v, updates its MIS data
// (cpu_bpt.cpp:49-58) and applies Russian roulette; false: cancelled.
static __device__ __noinline__ bool bpt_sample(const DScene& S, BV& v, const BV* prev, int px, int py, u64& rng,
                                               bool adjoint, f3& throughput, f3& origin, f3& excident, float& pdfF) {
	const u64 x0 = pcg_next(rng), x1 = pcg_next(rng);
	const float ru0 = sample_uniform(uint32_t(x0)), ru1 = sample_uniform(uint32_t(x0 >> 32));
	const float rr = sample_uniform(uint32_t(pcg_next(rng)));
	f3 sThroughput;
	float pdfB = 0.0f;
	origin = v.position;
	if(v.kind == BV_POINT) {
		excident = sample_dir_sphere_uniform(ru0, ru1);
		sThroughput = (v.incEnc * 4.0f) * PI;
		pdfF = __fdiv_rn(1.0f, 4.0f * PI);
	} else if(v.kind == BV_AREA) {
		const f3 d = sample_dir_cosine(ru0, ru1);
		const f3 tx = normalize(perpendicular(v.incEnc));
		const f3 ty = cross(v.incEnc, tx);
		excident = (d.x * tx + d.y * ty) + d.z * v.incEnc;
		sThroughput = v.intensity * PI;
		pdfF = __fdiv_rn(d.z, PI);
	} else if(v.kind == BV_ENV) {
		float pdf;
		origin = sample_position(S, v.incEnc, ru0, ru1, pdf);
		excident = v.incEnc;
		sThroughput = v.intensity / pdf;
		pdfF = pdf;
	} else if(v.kind == BV_CAMERA) {
		excident = pinhole_ray(S.camera, px, py, ru0, ru1, pdfF);
		sThroughput = make3(1.0f, 1.0f, 1.0f);
	} else {
		const PathSample smp = material_sample(v.ts, v.mat, bv_incident_dir(v), ru0, ru1, x1, adjoint);
		if(!smp.valid) return false;
		excident = smp.excident;
		sThroughput = smp.throughput;
		pdfF = smp.pdfF;
		pdfB = smp.pdfB;
	}
	if(prev) {
		const float prevReversePdf = bv_convert_pdf(*prev, v.kind, pdfB, bv_incident_dir(v), bv_incident_dist_sq(v));
		const float relToPrev = __fdiv_rn(prevReversePdf, prev->incidentPdf);
		v.prevRelSum = relToPrev + relToPrev * prev->prevRelSum;
	}
	throughput = throughput * sThroughput;
	const float cp = fmin_(maxc(throughput) + 0.1f, 1.0f);
	if(rr >= cp) return false;
	throughput = throughput / cp;
	add_epsilon(origin, excident, bv_geo_normal(v));
	return true;
}

// random_walk.hpp:77-113 and cpu_bpt.cpp:36-47: the vertex a segment from
// `from` ends in (a surface or a miss), with its incident pdf and throughput.
static __device__ __noinline__ void bpt_new_vertex(const DScene& S, const BV& from, f3 ro, f3 rd, const HitRec& best,
                                                   float pdfF, f3 throughput, BV& out) {
	out.inst = -1; out.prim = -1;
	out.prevRelSum = 0.0f;
	float dist = best.t;
	if(!best.has) {
		out.kind = BV_VOID;
		out.position = make3(0.0f, 0.0f, 0.0f);
		out.incEnc = rd;
	} else {
		const Intersection hit = hit_attributes(S, ro, rd, best);
		dist = hit.distance;
		out.kind = BV_SURFACE;
		out.position = ro + rd * hit.distance;
		out.incEnc = make3(rd.x, rd.y, hit.distance * sgn(rd.z));
		out.ts = tangent_space(S, hit);
		out.inst = hit.inst;
		out.prim = hit.prim;
		out.sp = hit.sp;
		out.mat = fetch_material(S, material_index(S, hit.inst, hit.prim), hit.uv);
	}
	const float inCosAbs = fabsf(bv_geo_factor(out, rd));
	const bool ortho = bv_ortho(from.kind) || bv_ortho(out.kind);
	out.incidentPdf = ortho ? pdfF * inCosAbs : __fdiv_rn(pdfF * fabsf(inCosAbs), dist * dist);
	out.throughput = throughput;
}

// The start vertex of the light subpath (path_util.hpp:568-625 create_light with
// BptVertexExt::init and mis_start_pdf, :763-771).
MBD void bpt_light_vertex(const DScene& S, const Emitter& em, BV& v) {
	v.position = em.position;
	v.throughput = make3(1.0f, 1.0f, 1.0f);
	v.prevRelSum = 0.0f;
	v.inst = -1; v.prim = -1;
	if(em.kind == LV_POINT) { v.kind = BV_POINT; v.incEnc = em.intensity; v.incidentPdf = em.pChoice; }
	else if(em.kind == LV_AREA) { v.kind = BV_AREA; v.incEnc = em.normal; v.intensity = em.intensity; v.incidentPdf = em.pdf * em.pChoice; }
	else {
		v.kind = BV_ENV; v.incEnc = em.normal; v.intensity = em.intensity; v.incidentPdf = em.pdf * em.pChoice;
		v.position = make3(0.0f, 0.0f, 0.0f);
		v.projSceneArea = projected_area(-em.normal, S.aabbMin, S.aabbMax);
	}
}

// A connection's shadow ray and what it adds.
struct BptConn {
	f3 ro, rd;
	float tmax;
	uint32_t pix;       // the pixel it adds to
	float4 add;         // radiance rgb, lightness when the shadow ray is unoccluded
	unsigned zeroSigns; // sign bits of the zeros an occluded one records (bit c: component c)
};

// cpu_bpt.cpp:120-148: the connection of view vertex v (its predecessor pv)
// with light vertex w (its predecessor pw) for view throughput thr. 1: it
// carries light if its shadow ray is unoccluded (c holds the ray, the pixel
// and both values; the balance-heuristic weight does not depend on the
// visibility, so it is taken before the ray is traced); 0: it carries
// nothing and records a zero in pixel c.pix; -1: it records nothing (a camera
// connection off the image).
MBD int bpt_connect(const DScene& S, uint32_t width, const BV& v, const BV* pv, const BV& w, const BV* pw, f3 thr, int px,
                    int py, BptConn& c) {
	int ox = px, oy = py;
	const bool possible = !((bv_ortho(v.kind) && bv_ortho(w.kind)) || (bv_ortho(v.kind) && w.kind == BV_CAMERA) ||
	                        (v.kind == BV_CAMERA && bv_ortho(w.kind)));
	if(possible) {
		f3 dir;
		float distSq;
		if(bv_ortho(w.kind)) { dir = -w.incEnc; distSq = 1.0f; }
		else {
			const f3 cv = w.position - v.position;
			distSq = lensq(cv);
			const float dist = sqrt_(distSq);
			dir = make3(sdiv(cv.x, dist), sdiv(cv.y, dist), sdiv(cv.z, dist));
		}
		const EvalValue val0 = bv_evaluate(S, v, dir, false, ox, oy);
		const EvalValue val1 = bv_evaluate(S, w, -dir, true, ox, oy);
		if(ox != -1) {
			const f3 bxdfProd = val0.value * val1.value;
			const float cosProd = val0.cosOut * val1.cosOut;
			if(any_pos(bxdfProd) && cosProd > 0.0f) {
				shadow_ray(v.position, bv_position(w, v.position), bv_geo_normal(v), bv_geo_normal(w), dir, c.ro, c.rd, c.tmax);
				c.pix = uint32_t(oy) * width + uint32_t(ox);
				const float rp0 = bpt_mis_part(v, pv, val0.pdfB, val1.pdfF, w.kind, dir, distSq);
				const float rp1 = bpt_mis_part(w, pw, val1.pdfB, val0.pdfF, v.kind, dir, distSq);
				const float mis = __fdiv_rn(1.0f, (1.0f + rp0) + rp1);
				const f3 bxdfs = bxdfProd * __fdiv_rn(mis, distSq);
				const f3 full = thr * w.throughput;
				const f3 rad = (full * cosProd) * bxdfs;
				const float light = __fdiv_rn((full.x + full.y) + full.z, 3.0f) * cosProd;
				c.add = make_float4(nan_to_zero(rad.x), nan_to_zero(rad.y), nan_to_zero(rad.z), nan_to_zero(light));
				// an occluded connection adds (throughput * 0) * 0
				const f3 zr = (full * 0.0f) * make3(0.0f, 0.0f, 0.0f);
				const float zl = __fdiv_rn((full.x + full.y) + full.z, 3.0f) * 0.0f;
				c.zeroSigns = (__float_as_uint(nan_to_zero(zr.x)) >> 31) | ((__float_as_uint(nan_to_zero(zr.y)) >> 31) << 1) |
				              ((__float_as_uint(nan_to_zero(zr.z)) >> 31) << 2) | ((__float_as_uint(nan_to_zero(zl)) >> 31) << 3);
				return 1;
			}
		}
	}
	if(ox == -1) return -1;
	c.pix = uint32_t(oy) * width + uint32_t(ox);
	return 0;
}

MBD float4 bpt_zeros(unsigned signs) {
	return make_float4(__uint_as_float((signs & 1u) << 31), __uint_as_float(((signs >> 1) & 1u) << 31),
	                   __uint_as_float(((signs >> 2) & 1u) << 31), __uint_as_float(((signs >> 3) & 1u) << 31));
}

// get_emission (path_util.hpp:410-458) and the random-hit weight
// (cpu_bpt.cpp:104-115): what view vertex h (predecessor pv, throughput thr)
// adds by reaching an emitter or leaving the scene.
MBD float4 bpt_emission(const DScene& S, const BV& h, const BV& pv, f3 thr) {
	f3 value = make3(0.0f, 0.0f, 0.0f);
	float backPdf = 0.0f, startPdf = 0.0f;
	if(h.kind == BV_VOID) {
		if(S.hasBackground) {
			value = lv(S.bgColor) * lv(S.bgScale);
			if(nonzero(value)) {
				backPdf = __fdiv_rn(1.0f, projected_area(h.incEnc, S.aabbMin, S.aabbMax));
				const float bgFlux = (S.bgFlux[0] + S.bgFlux[1]) + S.bgFlux[2];
				const float pb = __fdiv_rn(bgFlux, (S.dirFlux + S.rootFlux) + bgFlux);
				startPdf = __fdiv_rn(1.0f, 4.0f * PI) * pb;
			}
		}
	} else if(h.mat.type == MAT_EMISSIVE) {
		const float cosOut = dot(h.ts.geoN, -bv_incident_dir(h));
		if(cosOut > 0.0f) {
			value = h.mat.radiance;
			backPdf = __fdiv_rn(cosOut, PI);
			// the bidirectional weight counts the light's emission pdf (cpu_bpt.cpp:228)
			if(nonzero(value)) startPdf = light_pdfs(S, h.inst, h.prim, h.sp, pv.position).emit;
		}
	}
	if(nonzero(value)) {
		const float sum = bpt_mis_part(h, &pv, backPdf, startPdf, BV_VIRTUAL, make3(0.0f, 0.0f, 0.0f), 0.0f);
		value = value * __fdiv_rn(1.0f, 1.0f + sum);
	}
	const f3 rad = thr * value;
	const float light = __fdiv_rn((thr.x + thr.y) + thr.z, 3.0f) * __fdiv_rn((value.x + value.y) + value.z, 3.0f);
	return make_float4(nan_to_zero(rad.x), nan_to_zero(rad.y), nan_to_zero(rad.z), nan_to_zero(light));
}

enum BPhase { BP_IDLE = 0, BP_LWALK, BP_VCONNECT, BP_VWALK, BP_EXIT };

struct BptRec {
	const LtTargets& T;
	size_t base;
	MBD void put(size_t slot, uint32_t pix, float4 v) const {
		if(!T.recPixel) return;
		T.recPixel[base + slot] = int(pix);
		float* o = T.recValue + 4 * (base + slot);
		o[0] = v.x; o[1] = v.y; o[2] = v.z; o[3] = v.w;
	}
};

MBD void bpt_add(const LtTargets& T, uint32_t pix, float4 v) {
	if(v.x != 0.0f || v.y != 0.0f || v.z != 0.0f || v.w != 0.0f) atomicAdd(T.iter + pix, v);
}

// cpu_bpt.cpp:170-232 as a per-lane state machine
template < int AM >
__global__ void __launch_bounds__(128, 4) k_bpt(const DScene S, const LtParams P, const LtTargets T, BV* lightVerts,
                                                unsigned int* workCounter, TraceCounters* counters) {
	LocalStack stack;
	LocalCounters cnt;
	const unsigned lane = threadIdx.x & 31u;
	const uint32_t n = T.width * T.height;
	const int maxP = P.maxPathLength > 0 ? P.maxPathLength : 1;
	const size_t slots = size_t(maxP) * size_t(maxP) + size_t(maxP);
	BV* lp = lightVerts + (size_t(blockIdx.x) * blockDim.x + threadIdx.x) * size_t(maxP);
	BV vp[2];
	int phase = BP_IDLE;
	uint32_t pixel = 0;
	int px = 0, py = 0, lightLen = -1, viewLen = 0, cur = 0, l = 0, maxL = 0;
	u64 rng = 0;
	f3 lthr = make3(1.0f, 1.0f, 1.0f), thr = make3(1.0f, 1.0f, 1.0f);
	// a connection waiting for its shadow ray
	BptConn conn;
	conn.pix = 0; conn.add = make_float4(0.0f, 0.0f, 0.0f, 0.0f); conn.zeroSigns = 0;
	// the segment being traced
	float segPdf = 0.0f;
	auto start_view = [&]() {
		BV& c = vp[0];
		c.kind = BV_CAMERA;
		c.position = lv(S.camera.position);
		c.incEnc = make3(float(px), float(py), 0.0f);
		c.incidentPdf = 1.0f;
		c.prevRelSum = 0.0f;
		c.throughput = make3(1.0f, 1.0f, 1.0f);
		(void)pcg_next(rng); // create_camera consumes one number (unused by the pinhole camera)
		thr = make3(1.0f, 1.0f, 1.0f);
		viewLen = 0;
		cur = 0;
		l = max(0, P.minPathLength - 1);
		maxL = min(lightLen + 1, maxP);
		phase = BP_VCONNECT;
	};
	auto finish = [&]() {
		T.rngState[pixel] = rng;
		phase = BP_IDLE;
	};
	for(;;) {
		const unsigned idle = __ballot_sync(0xffffffffu, phase == BP_IDLE);
		if(idle) {
			const int leader = __ffs(idle) - 1;
			unsigned base = 0;
			if(int(lane) == leader) base = atomicAdd(workCounter, unsigned(__popc(idle)));
			base = __shfl_sync(0xffffffffu, base, leader);
			if(phase == BP_IDLE) {
				const uint32_t p = base + unsigned(__popc(idle & ((1u << lane) - 1u)));
				if(p >= n) phase = BP_EXIT;
				else {
					pixel = p;
					px = int(p % T.width);
					py = int(p / T.width);
					rng = T.rngState[p];
					const u64 r0 = pcg_next(rng);
					const float su0 = sample_uniform(uint32_t(r0)), su1 = sample_uniform(uint32_t(r0 >> 32));
					const u64 treeSeed = pcg_next(rng);
					const Emitter em = lights_emit(S, p, n, treeSeed, su0, su1);
					lightLen = -1;
					lthr = make3(1.0f, 1.0f, 1.0f);
					if(em.valid) {
						bpt_light_vertex(S, em, lp[0]);
						lightLen = 0;
					}
					if(lightLen == 0 && maxP > 1) phase = BP_LWALK;
					else start_view();
				}
			}
		}
		if(__all_sync(0xffffffffu, phase == BP_EXIT)) break;
		const BptRec rec{ T, size_t(pixel) * slots };
		bool trace = false, shadow = false;
		f3 ro = make3(0.0f, 0.0f, 0.0f), rd = make3(0.0f, 0.0f, 1.0f);
		float tmax = MAX_SCENE_SIZE;
		// The warp serves one kind of work per pass, the phase most of its
		// lanes are in: the lanes' phases run different code (light-subpath
		// sampling, connections, view-subpath sampling), and a warp running
		// all of them in one pass spent most cycles waiting for instructions
		// (185 vs 149 Mrays/s at 1080p).
		const unsigned nL = __popc(__ballot_sync(0xffffffffu, phase == BP_LWALK));
		const unsigned nC = __popc(__ballot_sync(0xffffffffu, phase == BP_VCONNECT));
		const unsigned nW = __popc(__ballot_sync(0xffffffffu, phase == BP_VWALK));
		const int pick = (nL >= nC && nL >= nW) ? BP_LWALK : (nC >= nW ? BP_VCONNECT : BP_VWALK);
		const bool mine = phase == pick;
		if(mine && phase == BP_LWALK) {
			BV& v = lp[lightLen];
			if(bpt_sample(S, v, lightLen > 0 ? &lp[lightLen - 1] : nullptr, px, py, rng, true, lthr, ro, rd, segPdf)) trace = true;
			else start_view();
		}
		if(mine && !trace && phase == BP_VCONNECT) {
			const BV& v = vp[cur];
			const BV* pv = viewLen > 0 ? &vp[1 - cur] : nullptr;
			while(l < maxL) {
				const int k = bpt_connect(S, T.width, v, pv, lp[l], l > 0 ? &lp[l - 1] : nullptr, thr, px, py, conn);
				if(k > 0) {
					ro = conn.ro; rd = conn.rd; tmax = conn.tmax;
					trace = shadow = true;
					break;
				}
				if(k == 0) rec.put(size_t(viewLen) * size_t(maxP) + size_t(l), conn.pix, make_float4(0.0f, 0.0f, 0.0f, 0.0f));
				++l;
			}
			if(!trace) phase = BP_VWALK;
		}
		if(mine && pick == BP_VWALK && !trace && phase == BP_VWALK) {
			BV& v = vp[cur];
			if(bpt_sample(S, v, viewLen > 0 ? &vp[1 - cur] : nullptr, px, py, rng, false, thr, ro, rd, segPdf)) {
				trace = true;
				tmax = MAX_SCENE_SIZE;
			} else finish();
		}
		if(!trace) continue;
		++cnt.rays;
		if(shadow) ++cnt.shadow;
		WideTracerT<AM> t;
		t.init(S, ro, rd, tmax, shadow, cnt);
		while(!t.step(S, cnt, stack)) {}
		if(shadow) {
			const float4 add = t.occluded ? bpt_zeros(conn.zeroSigns) : conn.add;
			if(!t.occluded) bpt_add(T, conn.pix, add);
			rec.put(size_t(viewLen) * size_t(maxP) + size_t(l), conn.pix, add);
			++l;
		} else if(phase == BP_LWALK) {
			if(!t.best.has) start_view();
			else {
				bpt_new_vertex(S, lp[lightLen], ro, rd, t.best, segPdf, lthr, lp[lightLen + 1]);
				++lightLen;
				if(lightLen >= maxP - 1) start_view();
			}
		} else {
			const int nxt = 1 - cur;
			bpt_new_vertex(S, vp[cur], ro, rd, t.best, segPdf, thr, vp[nxt]);
			++viewLen;
			cur = nxt;
			const BV& h = vp[cur];
			if(viewLen >= P.minPathLength) {
				const float4 add = bpt_emission(S, h, vp[1 - cur], thr);
				bpt_add(T, pixel, add);
				rec.put(size_t(maxP) * size_t(maxP) + size_t(viewLen - 1), pixel, add);
			}
			if(bv_end(h.kind) || viewLen >= maxP) finish();
			else {
				l = max(0, P.minPathLength - viewLen - 1);
				maxL = min(lightLen + 1, maxP - viewLen);
				phase = BP_VCONNECT;
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

// Staged schedule: the light subpaths of all pixels first, one trace and
// one shade launch per path length, then the view subpaths the same way, so
// the traversal runs in a kernel of its own (ray_queue.cuh) and each shade
// launch runs one vertex's code for all its lanes. A pixel draws its random
// numbers in the single kernel's order (emission, light-subpath samples, the
// camera, view-subpath samples), so every contribution and record is the
// single kernel's bit for bit; only the order of the atomic additions into
// the image differs.
//
// Generation g of the light phase traces the segments from light vertex g;
// generation maxPathLength - 1 + k of the view phase those from view vertex
// k and the connections of view vertex k. Queue state (BptwState) lives in
// one device allocation carved by bptw_carve.
enum { BPTW_EXT0 = 0, BPTW_SH0 = 2, BPTW_WORK = 4 };
constexpr int BPTW_COUNTERS = 4 + 2 * BPTW_MAX_PATH;

struct BptwState {
	BV* lv;             // light subpath vertices: vertex l of pixel p at l * n + p
	BV* vp[2];          // the view vertex with path length k of pixel p at vp[k & 1][p]
	float4* thr;        // per pixel: throughput of the subpath being walked, the pdf of its segment in w
	int* lightLen;      // per pixel: index of the light subpath's last vertex (-1: no light)
	int* qPixel[2];     // segment queues (double buffered by generation)
	float4* qOrg[2];    // origin (offset)
	float4* qDir[2];    // direction
	float4* qHit[2];    // t, instance bits, primitive bits, surface u
	float* qHitV[2];    // surface v
	float4* sOrg;       // connections: origin, length
	float4* sDir;       // direction
	float4* sAdd;       // radiance rgb, lightness if unoccluded
	uint4* sMeta;       // pixel, record slot (low, high word), sign bits of the occluded zeros
	unsigned* counters; // BPTW_COUNTERS
	uint32_t n;
};

MBD void bptw_queue_segment(const BptwState& W, int gen, uint32_t p, f3 o, f3 d, f3 thr, float pdf) {
	const int q = gen & 1;
	const unsigned i = queue_reserve(W.counters + BPTW_EXT0 + q);
	W.qPixel[q][i] = int(p);
	W.qOrg[q][i] = make_float4(o.x, o.y, o.z, 0.0f);
	W.qDir[q][i] = make_float4(d.x, d.y, d.z, 0.0f);
	W.thr[p] = make_float4(thr.x, thr.y, thr.z, pdf);
}

// The connections of view vertex v (path length viewLen, predecessor pv) with
// light vertices lo .. hi-1 of pixel p: shadow rays of generation gen, or
// the zero records of those that carry nothing.
MBD void bptw_connect(const DScene& S, const LtParams& P, const LtTargets& T, const BptwState& W, const BV& v, const BV* pv,
                      int viewLen, uint32_t p, int px, int py, f3 thr, int lo, int hi, int gen) {
	const size_t maxP = size_t(P.maxPathLength > 0 ? P.maxPathLength : 1);
	const size_t base = size_t(p) * (maxP * maxP + maxP) + size_t(viewLen) * maxP;
	for(int l = lo; l < hi; ++l) {
		BptConn c;
		const BV& w = W.lv[size_t(l) * W.n + p];
		const int k = bpt_connect(S, T.width, v, pv, w, l > 0 ? &W.lv[size_t(l - 1) * W.n + p] : nullptr, thr, px, py, c);
		const size_t slot = base + size_t(l);
		if(k > 0) {
			const unsigned i = queue_reserve(W.counters + BPTW_SH0 + (gen & 1));
			W.sOrg[i] = make_float4(c.ro.x, c.ro.y, c.ro.z, c.tmax);
			W.sDir[i] = make_float4(c.rd.x, c.rd.y, c.rd.z, 0.0f);
			W.sAdd[i] = c.add;
			W.sMeta[i] = make_uint4(c.pix, uint32_t(slot), uint32_t(slot >> 32), c.zeroSigns);
		} else if(k == 0 && T.recPixel) {
			T.recPixel[slot] = int(c.pix);
			float* o = T.recValue + 4 * slot;
			o[0] = 0.0f; o[1] = 0.0f; o[2] = 0.0f; o[3] = 0.0f;
		}
	}
}

// Every pixel: the light subpath's start vertex and first segment.
__global__ void __launch_bounds__(128) k_bptw_light_start(const DScene S, const LtParams P, const LtTargets T, BptwState W) {
	const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
	if(p >= W.n) return;
	const int maxP = P.maxPathLength > 0 ? P.maxPathLength : 1;
	u64 rng = T.rngState[p];
	const u64 r0 = pcg_next(rng);
	const float su0 = sample_uniform(uint32_t(r0)), su1 = sample_uniform(uint32_t(r0 >> 32));
	const u64 treeSeed = pcg_next(rng);
	const Emitter em = lights_emit(S, p, W.n, treeSeed, su0, su1);
	int lightLen = -1;
	if(em.valid) {
		BV v;
		bpt_light_vertex(S, em, v);
		lightLen = 0;
		if(maxP > 1) {
			f3 thr = make3(1.0f, 1.0f, 1.0f), o, d;
			float pdf;
			if(bpt_sample(S, v, nullptr, 0, 0, rng, true, thr, o, d, pdf)) bptw_queue_segment(W, 0, p, o, d, thr, pdf);
		}
		W.lv[p] = v;
	}
	W.lightLen[p] = lightLen;
	T.rngState[p] = rng;
}

// The trace stage of generation gen: segments (closest hit) and connections
// (any hit; a visible one adds its value, each one records what it added).
template < int AM >
__global__ void __launch_bounds__(128, 6) k_bptw_trace(const DScene S, const LtTargets T, BptwState W, int gen,
                                                    TraceCounters* counters) {
	const int q = gen & 1;
	if(blockIdx.x == 0 && threadIdx.x == 0) {
		W.counters[BPTW_EXT0 + (q ^ 1)] = 0u; // filled by this generation's shade
		W.counters[BPTW_SH0 + (q ^ 1)] = 0u;
	}
	RayQueue Q;
	Q.org = W.qOrg[q]; Q.dir = W.qDir[q]; Q.hit = W.qHit[q]; Q.hitV = W.qHitV[q];
	Q.sOrg = W.sOrg; Q.sDir = W.sDir;
	Q.nExt = *reinterpret_cast<volatile unsigned*>(W.counters + BPTW_EXT0 + q);
	Q.nSh = *reinterpret_cast<volatile unsigned*>(W.counters + BPTW_SH0 + q);
	Q.work = W.counters + BPTW_WORK + gen;
	trace_ray_queue<AM>(S, Q, counters, [&](unsigned s, bool occluded) {
		const uint4 meta = __ldcs(W.sMeta + s);
		float4 add;
		if(occluded) add = bpt_zeros(meta.w);
		else {
			add = __ldcs(W.sAdd + s);
			bpt_add(T, meta.x, add);
		}
		if(T.recPixel) {
			const size_t slot = size_t(meta.y) | (size_t(meta.z) << 32);
			T.recPixel[slot] = int(meta.x);
			float* o = T.recValue + 4 * slot;
			o[0] = add.x; o[1] = add.y; o[2] = add.z; o[3] = add.w;
		}
	});
}

MBD HitRec bptw_hit(const BptwState& W, int q, unsigned i) {
	const float4 hh = __ldcs(W.qHit[q] + i);
	HitRec hr;
	hr.t = hh.x;
	hr.inst = __float_as_int(hh.y);
	hr.prim = __float_as_int(hh.z);
	hr.sp = make2(hh.w, __ldcs(W.qHitV[q] + i));
	hr.has = hr.inst >= 0;
	return hr;
}

// Light phase, generation g: a segment from light vertex g that hit a surface
// becomes vertex g + 1, which takes the next segment unless it is the last
// one the path length allows.
__global__ void __launch_bounds__(128, 4) k_bptw_light_shade(const DScene S, const LtParams P, const LtTargets T, BptwState W,
                                                          int g) {
	const int q = g & 1;
	const unsigned count = *reinterpret_cast<volatile unsigned*>(W.counters + BPTW_EXT0 + q);
	const int maxP = P.maxPathLength > 0 ? P.maxPathLength : 1;
	for(unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
		const HitRec hr = bptw_hit(W, q, i);
		if(!hr.has) continue; // the light subpath ends with vertex g
		const uint32_t p = uint32_t(__ldcs(W.qPixel[q] + i));
		const f3 ro = f4to3(__ldcs(W.qOrg[q] + i)), rd = f4to3(__ldcs(W.qDir[q] + i));
		const float4 tp = W.thr[p];
		f3 thr = f4to3(tp);
		const BV* from = W.lv + size_t(g) * W.n + p;
		BV v;
		bpt_new_vertex(S, *from, ro, rd, hr, tp.w, thr, v);
		W.lightLen[p] = g + 1;
		if(g + 1 < maxP - 1) {
			u64 rng = T.rngState[p];
			f3 o, d;
			float pdf;
			if(bpt_sample(S, v, from, 0, 0, rng, true, thr, o, d, pdf)) bptw_queue_segment(W, g + 1, p, o, d, thr, pdf);
			T.rngState[p] = rng;
		}
		W.lv[size_t(g + 1) * W.n + p] = v;
	}
}

// View phase, first generation (gen): every pixel's camera vertex, its
// connections with the light subpath and its first segment.
__global__ void __launch_bounds__(128, 4) k_bptw_view_start(const DScene S, const LtParams P, const LtTargets T, BptwState W,
                                                         int gen) {
	const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
	if(p >= W.n) return;
	const int maxP = P.maxPathLength > 0 ? P.maxPathLength : 1;
	const int px = int(p % T.width), py = int(p / T.width);
	u64 rng = T.rngState[p];
	BV c;
	c.kind = BV_CAMERA;
	c.position = lv(S.camera.position);
	c.incEnc = make3(float(px), float(py), 0.0f);
	c.incidentPdf = 1.0f;
	c.prevRelSum = 0.0f;
	c.throughput = make3(1.0f, 1.0f, 1.0f);
	(void)pcg_next(rng); // create_camera consumes one number (unused by the pinhole camera)
	f3 thr = make3(1.0f, 1.0f, 1.0f);
	const int lightLen = W.lightLen[p];
	bptw_connect(S, P, T, W, c, nullptr, 0, p, px, py, thr, max(0, P.minPathLength - 1), min(lightLen + 1, maxP), gen);
	f3 o, d;
	float pdf;
	if(bpt_sample(S, c, nullptr, px, py, rng, false, thr, o, d, pdf)) {
		bptw_queue_segment(W, gen, p, o, d, thr, pdf);
		W.vp[0][p] = c;
	}
	T.rngState[p] = rng;
}

// View phase, generation gen: a segment from view vertex k (k + 1 < path
// length) becomes vertex k + 1 (a surface or a miss): what it adds by
// reaching an emitter or the background, then, unless the path ends there,
// its connections and its segment of generation gen + 1.
__global__ void __launch_bounds__(128, 4) k_bptw_view_shade(const DScene S, const LtParams P, const LtTargets T, BptwState W,
                                                         int gen, int k) {
	const int q = gen & 1;
	const unsigned count = *reinterpret_cast<volatile unsigned*>(W.counters + BPTW_EXT0 + q);
	const int maxP = P.maxPathLength > 0 ? P.maxPathLength : 1;
	const int viewLen = k + 1;
	for(unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
		const HitRec hr = bptw_hit(W, q, i);
		const uint32_t p = uint32_t(__ldcs(W.qPixel[q] + i));
		const f3 ro = f4to3(__ldcs(W.qOrg[q] + i)), rd = f4to3(__ldcs(W.qDir[q] + i));
		const float4 tp = W.thr[p];
		f3 thr = f4to3(tp);
		const BV pv = W.vp[k & 1][p];
		BV h;
		bpt_new_vertex(S, pv, ro, rd, hr, tp.w, thr, h);
		if(viewLen >= P.minPathLength) {
			const float4 add = bpt_emission(S, h, pv, thr);
			bpt_add(T, p, add);
			if(T.recPixel) {
				const size_t slot = size_t(p) * (size_t(maxP) * maxP + maxP) + size_t(maxP) * maxP + size_t(viewLen - 1);
				T.recPixel[slot] = int(p);
				float* o = T.recValue + 4 * slot;
				o[0] = add.x; o[1] = add.y; o[2] = add.z; o[3] = add.w;
			}
		}
		if(bv_end(h.kind) || viewLen >= maxP) continue;
		const int px = int(p % T.width), py = int(p / T.width);
		const int lightLen = W.lightLen[p];
		bptw_connect(S, P, T, W, h, &pv, viewLen, p, px, py, thr, max(0, P.minPathLength - viewLen - 1),
		             min(lightLen + 1, maxP - viewLen), gen + 1);
		u64 rng = T.rngState[p];
		f3 o, d;
		float pdf;
		if(bpt_sample(S, h, &pv, px, py, rng, false, thr, o, d, pdf)) {
			bptw_queue_segment(W, gen + 1, p, o, d, thr, pdf);
			W.vp[viewLen & 1][p] = h;
		}
		T.rngState[p] = rng;
	}
}

int bptw_trace_blocks() {
	static int blocks = 0;
	if(blocks == 0) {
		int dev = 0, sms = 148, a = 0, b = 0;
		cudaGetDevice(&dev);
		cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
		cudaOccupancyMaxActiveBlocksPerMultiprocessor(&a, k_bptw_trace<ALPHA_NEVER>, 128, 0);
		cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_bptw_trace<ALPHA_ALWAYS>, 128, 0);
		blocks = sms * std::max(1, std::min(a, b));
	}
	return blocks;
}

size_t bptw_size(size_t n, size_t m) {
	auto al = [](size_t b) { return (b + 255) & ~size_t(255); };
	return al(n * m * sizeof(BV)) + 2 * al(n * sizeof(BV)) + al(n * 16) + al(n * 4) +
	       2 * (al(n * 4) + 3 * al(n * 16) + al(n * 4)) + 4 * al(n * m * 16) + al(BPTW_COUNTERS * sizeof(unsigned));
}

BptwState bptw_carve(void* memory, size_t n, size_t m) {
	auto al = [](size_t b) { return (b + 255) & ~size_t(255); };
	char* mem = static_cast<char*>(memory);
	auto take = [&](size_t b) { char* r = mem; mem += al(b); return r; };
	BptwState W;
	W.n = uint32_t(n);
	W.lv = reinterpret_cast<BV*>(take(n * m * sizeof(BV)));
	W.vp[0] = reinterpret_cast<BV*>(take(n * sizeof(BV)));
	W.vp[1] = reinterpret_cast<BV*>(take(n * sizeof(BV)));
	W.thr = reinterpret_cast<float4*>(take(n * 16));
	W.lightLen = reinterpret_cast<int*>(take(n * 4));
	for(int q = 0; q < 2; ++q) {
		W.qPixel[q] = reinterpret_cast<int*>(take(n * 4));
		W.qOrg[q] = reinterpret_cast<float4*>(take(n * 16));
		W.qDir[q] = reinterpret_cast<float4*>(take(n * 16));
		W.qHit[q] = reinterpret_cast<float4*>(take(n * 16));
		W.qHitV[q] = reinterpret_cast<float*>(take(n * 4));
	}
	// a view vertex has at most max. path length connections
	W.sOrg = reinterpret_cast<float4*>(take(n * m * 16));
	W.sDir = reinterpret_cast<float4*>(take(n * m * 16));
	W.sAdd = reinterpret_cast<float4*>(take(n * m * 16));
	W.sMeta = reinterpret_cast<uint4*>(take(n * m * 16));
	W.counters = reinterpret_cast<unsigned*>(take(BPTW_COUNTERS * sizeof(unsigned)));
	return W;
}

// output_handler_variance.hpp:7-31: running means and variances
__global__ void k_bpt_finalize(LtTargets T) {
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
}

int bpt_blocks() {
	static int blocks = 0;
	if(blocks == 0) {
		int dev = 0, sms = 148, perSm = 0;
		cudaGetDevice(&dev);
		cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
		// both variants (scenes with and without alpha textures) fit as many blocks
		int perSmAlpha = 0;
		cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, k_bpt<ALPHA_NEVER>, 128, 0);
		cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSmAlpha, k_bpt<ALPHA_ALWAYS>, 128, 0);
		if(perSmAlpha > perSm) perSm = perSmAlpha;
		blocks = sms * (perSm > 0 ? perSm : 1);
	}
	return blocks;
}

} // namespace

size_t bpt_scratch_bytes(int maxPathLength) {
	return size_t(bpt_blocks()) * 128u * size_t(maxPathLength > 0 ? maxPathLength : 1) * sizeof(BV);
}

size_t bptw_bytes(size_t numPixels, int maxPathLength) {
	return bptw_size(numPixels, size_t(maxPathLength > 0 ? maxPathLength : 1));
}

cudaError_t launch_bpt(const DScene& S, const LtParams& P, const LtTargets& T, void* scratch, unsigned int* workCounter,
                       TraceCounters* counters, cudaStream_t stream, void* wavefront) {
	const uint32_t n = T.width * T.height;
	if(n == 0) return cudaSuccess;
	const int maxP = P.maxPathLength > 0 ? P.maxPathLength : 1;
	cudaError_t e;
	if((e = cudaMemsetAsync(T.iter, 0, size_t(n) * sizeof(float4), stream)) != cudaSuccess) return e;
	if(T.recPixel) {
		const size_t m = size_t(maxP);
		const size_t slots = size_t(n) * (m * m + m);
		if((e = cudaMemsetAsync(T.recPixel, 0xFF, slots * sizeof(int32_t), stream)) != cudaSuccess) return e;
		if((e = cudaMemsetAsync(T.recValue, 0, slots * 4 * sizeof(float), stream)) != cudaSuccess) return e;
	}
	if(wavefront) {
		// queue indices are 32-bit: up to max. path length connections per pixel
		if(maxP > BPTW_MAX_PATH || size_t(n) * size_t(maxP) > size_t(0xFFFFFFFFu)) return cudaErrorInvalidValue;
		const BptwState W = bptw_carve(wavefront, n, size_t(maxP));
		if((e = cudaMemsetAsync(W.counters, 0, BPTW_COUNTERS * sizeof(unsigned), stream)) != cudaSuccess) return e;
		const int tb = bptw_trace_blocks();
		int dev = 0, sms = 148;
		cudaGetDevice(&dev);
		cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
		auto trace = [&](int gen) {
			if(S.hasAlpha) k_bptw_trace<ALPHA_ALWAYS><<<tb, 128, 0, stream>>>(S, T, W, gen, counters);
			else k_bptw_trace<ALPHA_NEVER><<<tb, 128, 0, stream>>>(S, T, W, gen, counters);
		};
		k_bptw_light_start<<<(n + 127) / 128, 128, 0, stream>>>(S, P, T, W);
		const int lightGens = maxP - 1;
		for(int g = 0; g < lightGens; ++g) {
			trace(g);
			k_bptw_light_shade<<<sms * 4, 128, 0, stream>>>(S, P, T, W, g);
		}
		k_bptw_view_start<<<(n + 127) / 128, 128, 0, stream>>>(S, P, T, W, lightGens);
		for(int k = 0; k < maxP; ++k) {
			trace(lightGens + k);
			k_bptw_view_shade<<<sms * 4, 128, 0, stream>>>(S, P, T, W, lightGens + k, k);
		}
	} else {
		if((e = cudaMemsetAsync(workCounter, 0, sizeof(unsigned int), stream)) != cudaSuccess) return e;
		// the variant for the scene: alpha textures or none (no alpha code in the loop)
		if(S.hasAlpha) k_bpt<ALPHA_ALWAYS><<<bpt_blocks(), 128, 0, stream>>>(S, P, T, static_cast<BV*>(scratch), workCounter, counters);
		else k_bpt<ALPHA_NEVER><<<bpt_blocks(), 128, 0, stream>>>(S, P, T, static_cast<BV*>(scratch), workCounter, counters);
	}
	if((e = cudaGetLastError()) != cudaSuccess) return e;
	k_bpt_finalize<<<(n + 255) / 256, 256, 0, stream>>>(T);
	return cudaGetLastError();
}

} // namespace mb
