// Path vertices and the staged schedule shared by the bidirectional path
// tracer (bpt.cu) and vertex connection and merging (vcm.cu): the vertex
// record with the reference's PathVertex contents and both renderers' MIS
// extensions, its sampling and creation, and the stage state of the staged
// schedules (every pixel's light subpath, its last two view vertices, the
// segment and connection queues) with their trace kernel.
#pragma once

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
struct alignas(16) BV {
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
	int pathLen;        // segments from the subpath's start (PathVertex::m_pathLen)
	float prevConv;     // VcmVertexExt::prevConversionFactor: |cos| / d^2 towards the previous vertex
};

// The stages keep vertices in device arrays; a vertex moves as 11 16-byte
// words (one vector load or store each) instead of 44 scalar ones.
static_assert(sizeof(BV) == 176 && sizeof(BV) % 16 == 0, "BV moves as float4 words");
MBD BV bv_load(const BV* p) {
	BV v;
	const float4* s = reinterpret_cast<const float4*>(p);
	float4* d = reinterpret_cast<float4*>(&v);
#pragma unroll
	for(int i = 0; i < int(sizeof(BV) / 16); ++i) d[i] = s[i];
	return v;
}
MBD void bv_store(BV* p, const BV& v) {
	const float4* s = reinterpret_cast<const float4*>(&v);
	float4* d = reinterpret_cast<float4*>(p);
#pragma unroll
	for(int i = 0; i < int(sizeof(BV) / 16); ++i) d[i] = s[i];
}

MBD bool bv_ortho(int k) { return k == BV_VOID || k == BV_ENV; } // path_util.hpp:41-46
MBD bool bv_end(int k) { return k != BV_SURFACE; }               // path_util.hpp:33-35
// path_util.hpp:53-58
MBD bool bv_hitable(int k) { return k == BV_SURFACE || k == BV_AREA || k == BV_ENV || k == BV_VOID; }

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

// cpu_vcm.cpp:21-32: the relative probabilities of the events before v
// (connections and merges) for the reverse sampling pdf pdfBack at v; prev is
// v's predecessor (null at a subpath's start). nPhotons and mergeArea: the
// number of light subpaths and the merge disc's area.
MBD float vcm_prev_rel_sum(const BV& v, const BV* prev, float pdfBack, float nPhotons, float mergeArea) {
	if(!prev) return 0.0f;
	const float pdfBackA = pdfBack * v.prevConv;
	const float relMerge = prev->pathLen > 0 ? (pdfBackA * nPhotons) * mergeArea : 0.0f; // no merges at start points
	const float relConn = __fdiv_rn(pdfBackA, prev->incidentPdf);
	return (relConn + relMerge) + relConn * prev->prevRelSum;
}

// random_walk.hpp:38-75: samples v, updates its MIS data (the bidirectional
// path tracer's, cpu_bpt.cpp:49-58, or with VCM those of VcmVertexExt,
// cpu_vcm.cpp:140-146) and applies Russian roulette; false: cancelled.
template < bool VCM >
static __device__ __noinline__ bool bpt_sample(const DScene& S, BV& v, const BV* prev, int px, int py, u64& rng,
                                               bool adjoint, f3& throughput, f3& origin, f3& excident, float& pdfF,
                                               float nPhotons = 0.0f, float mergeArea = 0.0f) {
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
	if(VCM) v.prevRelSum = vcm_prev_rel_sum(v, prev, pdfB, nPhotons, mergeArea);
	else if(prev) {
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
// `from` ends in (a surface or a miss), with its incident pdf and throughput;
// with VCM also the conversion factor towards `from` (cpu_vcm.cpp:117-137).
template < bool VCM >
static __device__ __noinline__ void bpt_new_vertex(const DScene& S, const BV& from, f3 ro, f3 rd, const HitRec& best,
                                                   float pdfF, f3 throughput, BV& out) {
	out.inst = -1; out.prim = -1;
	out.prevRelSum = 0.0f;
	out.prevConv = 0.0f;
	out.pathLen = from.pathLen + 1;
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
	if(VCM && bv_hitable(from.kind)) {
		const float outCosAbs = fabsf(bv_geo_factor(from, rd));
		out.prevConv = ortho ? outCosAbs : __fdiv_rn(outCosAbs, dist * dist);
	}
}

// The start vertex of the light subpath (path_util.hpp:568-625 create_light with
// BptVertexExt::init and mis_start_pdf, :763-771).
MBD void bpt_light_vertex(const DScene& S, const Emitter& em, BV& v) {
	v.position = em.position;
	v.throughput = make3(1.0f, 1.0f, 1.0f);
	v.prevRelSum = 0.0f;
	v.pathLen = 0;
	v.prevConv = 0.0f;
	v.inst = -1; v.prim = -1;
	if(em.kind == LV_POINT) { v.kind = BV_POINT; v.incEnc = em.intensity; v.incidentPdf = em.pChoice; }
	else if(em.kind == LV_AREA) { v.kind = BV_AREA; v.incEnc = em.normal; v.intensity = em.intensity; v.incidentPdf = em.pdf * em.pChoice; }
	else {
		v.kind = BV_ENV; v.incEnc = em.normal; v.intensity = em.intensity; v.incidentPdf = em.pdf * em.pChoice;
		v.position = make3(0.0f, 0.0f, 0.0f);
		v.projSceneArea = projected_area(-em.normal, S.aabbMin, S.aabbMax);
	}
}


// The camera vertex of pixel (px, py) (path_util.hpp:540-566 create_camera).
MBD void bpt_camera_vertex(const DScene& S, int px, int py, BV& c) {
	c.kind = BV_CAMERA;
	c.position = lv(S.camera.position);
	c.incEnc = make3(float(px), float(py), 0.0f);
	c.incidentPdf = 1.0f;
	c.prevRelSum = 0.0f;
	c.throughput = make3(1.0f, 1.0f, 1.0f);
	c.pathLen = 0;
	c.prevConv = 0.0f;
}

// Sign bits of the zeros a connection adds when it carries nothing (occluded,
// or no light either way): (value * 0) * 0 keeps the signs of the radiance
// factor rad and of the lightness factor light; NaN components give +0.
MBD unsigned zero_signs(f3 rad, float light) {
	const f3 zr = (rad * 0.0f) * make3(0.0f, 0.0f, 0.0f);
	const float zl = light * 0.0f;
	return (__float_as_uint(nan_to_zero(zr.x)) >> 31) | ((__float_as_uint(nan_to_zero(zr.y)) >> 31) << 1) |
	       ((__float_as_uint(nan_to_zero(zr.z)) >> 31) << 2) | ((__float_as_uint(nan_to_zero(zl)) >> 31) << 3);
}

// A connection's shadow ray and what it adds.
struct BptConn {
	f3 ro, rd;
	float tmax;
	uint32_t pix;       // the pixel it adds to
	float4 add;         // radiance rgb, lightness when the shadow ray is unoccluded
	unsigned zeroSigns; // sign bits of the zeros an occluded one records (bit c: component c)
};

MBD float4 bpt_zeros(unsigned signs) {
	return make_float4(__uint_as_float((signs & 1u) << 31), __uint_as_float(((signs >> 1) & 1u) << 31),
	                   __uint_as_float(((signs >> 2) & 1u) << 31), __uint_as_float(((signs >> 3) & 1u) << 31));
}

MBD void bpt_add(const LtTargets& T, uint32_t pix, float4 v) {
	if(v.x != 0.0f || v.y != 0.0f || v.z != 0.0f || v.w != 0.0f) atomicAdd(T.iter + pix, v);
}


enum { BPTW_EXT0 = 0, BPTW_SH0 = 2, BPTW_WORK = 4 };
// Resident blocks of 128 threads per SM that the shade-side stage kernels
// (light shade, view start, view shade) are compiled for; their grids are
// this many blocks per SM. They wait on scattered vertex loads, so occupancy
// beats registers: 8 blocks (64 registers) measured fastest, bidirectional
// path tracer 748 / 765 / 764 and VCM 468 / 479 / 490 Mrays/s at 4 / 6 / 8;
// 12 blocks (42 registers, more spills) fell back to 715 and 497.
constexpr int BPTW_SHADE_BLOCKS = 8;
// ... and the trace stage (5 and 6 measured alike; 8 was 6 % slower).
constexpr int BPTW_TRACE_BLOCKS = 6;
// Resident blocks per SM of the connection kernels (k_bptw_connect,
// k_vcmw_connect) and of VCM's merge kernel. Measured at 1080p (Mrays/s,
// connections at 8 / 6 / 4 blocks): BPT 778 / 780 / 785, VCM 569 / 569 / 571;
// the merges at 6 / 8 / 10 / 12 blocks: VCM 567 / 569 / 560 / 560.
constexpr int BPTW_CONNECT_BLOCKS = 4;
constexpr int VCM_MERGE_BLOCKS = 8;
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
	BV* hv;             // per item of a view generation's segment queue: the vertex it reached
	float4* hThr;       // its throughput, and its pixel + 1 (bits; 0: nothing more to do for it)
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

// The trace stage of generation gen: segments (closest hit) and connections
// (any hit; a visible one adds its value, each one records what it added).
template < int AM >
__global__ void __launch_bounds__(128, BPTW_TRACE_BLOCKS) k_bptw_trace(const DScene S, const LtTargets T, BptwState W, int gen,
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
// one the path length allows. VCM: with its MIS data (nPhotons light
// subpaths, merge area mergeArea).
template < bool VCM >
__global__ void __launch_bounds__(128, BPTW_SHADE_BLOCKS) k_bptw_light_shade(const DScene S, const LtParams P, const LtTargets T, BptwState W,
                                                          int g, float nPhotons = 0.0f, float mergeArea = 0.0f) {
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
		bpt_new_vertex<VCM>(S, *from, ro, rd, hr, tp.w, thr, v);
		W.lightLen[p] = g + 1;
		if(g + 1 < maxP - 1) {
			u64 rng = T.rngState[p];
			f3 o, d;
			float pdf;
			if(bpt_sample<VCM>(S, v, from, 0, 0, rng, true, thr, o, d, pdf, nPhotons, mergeArea))
				bptw_queue_segment(W, g + 1, p, o, d, thr, pdf);
			T.rngState[p] = rng;
		}
		bv_store(W.lv + size_t(g + 1) * W.n + p, v);
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
	       2 * (al(n * 4) + 3 * al(n * 16) + al(n * 4)) + 4 * al(n * m * 16) + al(n * sizeof(BV)) + al(n * 16) +
	       al(BPTW_COUNTERS * sizeof(unsigned));
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
	W.hv = reinterpret_cast<BV*>(take(n * sizeof(BV)));
	W.hThr = reinterpret_cast<float4*>(take(n * 16));
	W.counters = reinterpret_cast<unsigned*>(take(BPTW_COUNTERS * sizeof(unsigned)));
	return W;
}


} // namespace
} // namespace mb
