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
// Schedule: one persistent kernel whose lanes run a state machine (as the
// light tracer's): a lane takes a new pixel as soon as its own finishes, and
// every pass of the loop traces at most one ray per lane (a light-subpath
// segment, a connection's shadow ray or a view-subpath segment) in one
// traversal loop shared by the warp. A lane keeps its light subpath in its
// own slice of a scratch array (max. path length vertices) and the last two
// view vertices in local memory. Connections from the camera land in other
// pixels, so all contributions go to an iteration buffer with vector atomics.
#include "accumulate.cuh"
#include "wide_traverse.cuh"
#include "emit.cuh"
#include "lt_api.hpp"

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
	uint32_t cpix = 0;
	f3 cbxdf = make3(0.0f, 0.0f, 0.0f), cdir = make3(0.0f, 0.0f, 1.0f);
	float ccos = 0.0f, cdistSq = 1.0f, c0F = 0.0f, c0B = 0.0f, c1F = 0.0f, c1B = 0.0f;
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
			while(l < maxL) {
				const BV& w = lp[l];
				// connect (cpu_bpt.cpp:120-148)
				int ox = px, oy = py;
				bool possible = !((bv_ortho(v.kind) && bv_ortho(w.kind)) || (bv_ortho(v.kind) && w.kind == BV_CAMERA) ||
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
							shadow_ray(v.position, bv_position(w, v.position), bv_geo_normal(v), bv_geo_normal(w), dir, ro, rd, tmax);
							cpix = uint32_t(oy) * T.width + uint32_t(ox);
							cbxdf = bxdfProd; ccos = cosProd; cdir = dir; cdistSq = distSq;
							c0F = val0.pdfF; c0B = val0.pdfB; c1F = val1.pdfF; c1B = val1.pdfB;
							trace = shadow = true;
							break;
						}
					}
				}
				if(ox != -1) rec.put(size_t(viewLen) * size_t(maxP) + size_t(l), uint32_t(oy) * T.width + uint32_t(ox),
				                     make_float4(0.0f, 0.0f, 0.0f, 0.0f));
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
			float4 add = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
			const BV& v = vp[cur];
			const BV& w = lp[l];
			if(!t.occluded) {
				const float rp0 = bpt_mis_part(v, viewLen > 0 ? &vp[1 - cur] : nullptr, c0B, c1F, w.kind, cdir, cdistSq);
				const float rp1 = bpt_mis_part(w, l > 0 ? &lp[l - 1] : nullptr, c1B, c0F, v.kind, cdir, cdistSq);
				const float mis = __fdiv_rn(1.0f, (1.0f + rp0) + rp1);
				const f3 bxdfs = cbxdf * __fdiv_rn(mis, cdistSq);
				const f3 full = thr * w.throughput;
				const f3 rad = (full * ccos) * bxdfs;
				const float light = __fdiv_rn((full.x + full.y) + full.z, 3.0f) * ccos;
				add = make_float4(nan_to_zero(rad.x), nan_to_zero(rad.y), nan_to_zero(rad.z), nan_to_zero(light));
				bpt_add(T, cpix, add);
			} else {
				// an occluded connection adds (throughput * 0) * 0
				const f3 full = thr * w.throughput;
				const f3 rad = (full * 0.0f) * make3(0.0f, 0.0f, 0.0f);
				const float light = __fdiv_rn((full.x + full.y) + full.z, 3.0f) * 0.0f;
				add = make_float4(nan_to_zero(rad.x), nan_to_zero(rad.y), nan_to_zero(rad.z), nan_to_zero(light));
			}
			rec.put(size_t(viewLen) * size_t(maxP) + size_t(l), cpix, add);
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
				// get_emission (path_util.hpp:410-458) and the random-hit weight (cpu_bpt.cpp:104-115)
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
						if(nonzero(value)) startPdf = light_pdfs(S, h.inst, h.prim, h.sp, vp[1 - cur].position).emit;
					}
				}
				if(nonzero(value)) {
					const float sum = bpt_mis_part(h, &vp[1 - cur], backPdf, startPdf, BV_VIRTUAL, make3(0.0f, 0.0f, 0.0f), 0.0f);
					value = value * __fdiv_rn(1.0f, 1.0f + sum);
				}
				const f3 rad = thr * value;
				const float light = __fdiv_rn((thr.x + thr.y) + thr.z, 3.0f) * __fdiv_rn((value.x + value.y) + value.z, 3.0f);
				const float4 add = make_float4(nan_to_zero(rad.x), nan_to_zero(rad.y), nan_to_zero(rad.z), nan_to_zero(light));
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

cudaError_t launch_bpt(const DScene& S, const LtParams& P, const LtTargets& T, void* scratch,
                       unsigned int* workCounter, TraceCounters* counters, cudaStream_t stream) {
	const uint32_t n = T.width * T.height;
	if(n == 0) return cudaSuccess;
	cudaError_t e;
	if((e = cudaMemsetAsync(T.iter, 0, size_t(n) * sizeof(float4), stream)) != cudaSuccess) return e;
	if(T.recPixel) {
		const size_t m = size_t(P.maxPathLength > 0 ? P.maxPathLength : 1);
		const size_t slots = size_t(n) * (m * m + m);
		if((e = cudaMemsetAsync(T.recPixel, 0xFF, slots * sizeof(int32_t), stream)) != cudaSuccess) return e;
		if((e = cudaMemsetAsync(T.recValue, 0, slots * 4 * sizeof(float), stream)) != cudaSuccess) return e;
	}
	if((e = cudaMemsetAsync(workCounter, 0, sizeof(unsigned int), stream)) != cudaSuccess) return e;
	// the variant for the scene: alpha textures or none (no alpha code in the loop)
	if(S.hasAlpha) k_bpt<ALPHA_ALWAYS><<<bpt_blocks(), 128, 0, stream>>>(S, P, T, static_cast<BV*>(scratch), workCounter, counters);
	else k_bpt<ALPHA_NEVER><<<bpt_blocks(), 128, 0, stream>>>(S, P, T, static_cast<BV*>(scratch), workCounter, counters);
	if((e = cudaGetLastError()) != cudaSuccess) return e;
	k_bpt_finalize<<<(n + 255) / 256, 256, 0, stream>>>(T);
	return cudaGetLastError();
}

} // namespace mb
