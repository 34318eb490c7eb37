// Vertex connection and merging (the CUDA "Vertex Connection and Merging" of
// the C API). The reference has it on the CPU only (src/core/renderer/vcm/
// cpu_vcm.cpp:148-290); this is the same estimator on the GPU traversal.
//
// Per iteration: one light subpath per pixel (the bidirectional path
// tracer's light phase with VCM's MIS data), all light vertices after the
// start stored as photons in a hash grid, then per pixel a view subpath whose
// vertices connect to every vertex of one light subpath (chosen by a hash of
// the pixel index), count the emitters they hit and merge with the photons
// within the merge radius. Connections, hits and merges share one balance
// heuristic (VcmVertexExt, cpu_vcm.cpp:17-146).
//
// Schedule: the bidirectional path tracer's stages (bidir.cuh). Light phase:
// k_vcm_seed (the light tree's shared seed from pixel 0's generator),
// k_vcmw_light_start, then per generation the shared trace kernel and
// k_bptw_light_shade<true>. Photon grid (photon_map.hpp): k_vcm_keys appends
// every light vertex after the start with the key (bucket, slot), a onesweep
// radix sort over the photons (their count read back first) orders them by
// bucket and, within a bucket, by ascending (subpath, vertex) slot,
// k_vcm_ranges finds the bucket ranges and k_vcm_gather packs each photon's
// merge data (80 B) in bucket order. View phase: k_vcmw_view_start, then per generation the trace
// kernel, k_vcmw_view_shade (the vertex reached: its emitter term and next
// segment; it hands the vertex on), k_vcmw_merge (the vertex's merges) and
// k_vcmw_connect (its connections). A bucket's photons are visited
// from the last to the first, the order of the reference's head-inserted
// lists when one thread fills them, so every contribution is the oracle's bit
// for bit.
#include "bidir.cuh"
#include "../lbvh/radix_sort.cuh"

#include <cmath>
#include <mutex>

namespace mb {
namespace {

// ---------------------------------------------------------------- photon grid
// photon_map.hpp:29-52: a cell's hash; the insert's cell is ceil(p / edge),
// a query's base cell round(p / edge) and its 8 cells base + {0, 1}^3
constexpr uint32_t VCM_MAGIC_X = 0xb286aff7u, VCM_MAGIC_Y = 0x35e4a487u, VCM_MAGIC_Z = 0x75a9c18fu;
// an integral float as an unsigned grid coordinate (two's complement wrap
// for negative cells, as the conversion does on the reference's x86 hosts)
MBD uint32_t vcm_cell_coord(float x) { return uint32_t((long long)(x)); }
MBD uint32_t vcm_cell_hash(uint32_t x, uint32_t y, uint32_t z) { return x * VCM_MAGIC_X + y * VCM_MAGIC_Y + z * VCM_MAGIC_Z; }
MBD uint32_t vcm_insert_hash(f3 p, float density) {
	return vcm_cell_hash(vcm_cell_coord(ceilf(p.x * density)), vcm_cell_coord(ceilf(p.y * density)),
	                     vcm_cell_coord(ceilf(p.z * density)));
}
MBD uint32_t vcm_query_hash(f3 p, float density) {
	return vcm_cell_hash(vcm_cell_coord(roundf(p.x * density)), vcm_cell_coord(roundf(p.y * density)),
	                     vcm_cell_coord(roundf(p.z * density)));
}
// Thomas Wang's 32-bit integer hash (cn::WangHash, cpu_vcm.cpp:224): the
// light subpath a pixel's view subpath connects to
MBD uint32_t wang_hash(uint32_t x) {
	x = (x ^ 61u) ^ (x >> 16);
	x = x * 9u;
	x = x ^ (x >> 4);
	x = x * 0x27d4eb2du;
	x = x ^ (x >> 15);
	return x;
}

// One iteration's constants (CpuVcm::iterate, cpu_vcm.cpp:148-157).
struct VcmConsts {
	float nPhotons;   // light subpaths (= pixels)
	float lightArea;  // merge area of the light walk: (pi r) r (trace_photon)
	float viewArea;   // of the view walk, the weights and the density estimate: pi (r r) (sample)
	float radiusSq;
	float density;    // 1 / cell edge (edge = 2.0001 r)
	uint32_t mapSize; // buckets
	int slotBits;     // bits of a light-vertex slot index p * M + l (the low part of a photon's sort key)
};

// The photon grid, carved after the stages' state.
struct VcmGrid {
	u64* keys;            // per photon: its bucket << slotBits | its slot p * M + l, then sorted
	int32_t* vals;        // the slot, sorted with the keys
	u64* keysAlt;         // the sort's ping-pong buffers
	int32_t* valsAlt;
	uint32_t* status;     // the sort's look-back tile status
	uint32_t* hist;       // 8 x 256 digit counts
	unsigned* tileCounter;
	unsigned* error;      // an expired bounded wait of the sort
	uint32_t* start;      // per bucket: range of sorted photons
	uint32_t* end;
	float4* photons;      // 5 per sorted photon: position, vertex index (bits); incident direction,
	                      // incident pdf; geometric normal, conversion factor; throughput, the previous
	                      // vertex's incident pdf; the previous vertex's relative-probability sum
	u64* seed;            // the light tree's seed of the iteration
	unsigned* count;      // photons of the iteration (light vertices after the start)
};

__global__ void k_vcm_seed(const LtTargets T, VcmGrid G) {
	// cpu_vcm.cpp:160: the photons' light-tree seed is pixel 0's next number
	u64 rng = T.rngState[0];
	*G.seed = pcg_next(rng);
	T.rngState[0] = rng;
}

// Every light vertex l >= 1 of pixel p's subpath (slot s = p * M + l) is a
// photon: key (bucket << slotBits) | s, value s, appended in any order. The
// key makes the sorted order the same whatever the order of the appends: by
// bucket, and within a bucket by ascending slot.
__global__ void k_vcm_keys(const BptwState W, VcmGrid G, VcmConsts C, uint32_t maxP) {
	const size_t total = size_t(W.n) * maxP;
	for(size_t s = size_t(blockIdx.x) * blockDim.x + threadIdx.x; s < total; s += size_t(gridDim.x) * blockDim.x) {
		const uint32_t p = uint32_t(s / maxP), l = uint32_t(s % maxP);
		if(l >= 1 && int(l) <= W.lightLen[p]) {
			const uint32_t b = vcm_insert_hash(W.lv[size_t(l) * W.n + p].position, C.density) % C.mapSize;
			const unsigned i = queue_reserve(G.count);
			G.keys[i] = (u64(b) << C.slotBits) | u64(s);
			G.vals[i] = int32_t(s);
		}
	}
}

__global__ void k_vcm_ranges(VcmGrid G, uint32_t total, int slotBits) {
	for(uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
		const uint32_t b = uint32_t(G.keys[i] >> slotBits);
		if(i == 0 || uint32_t(G.keys[i - 1] >> slotBits) != b) G.start[b] = i;
		if(i + 1 == total || uint32_t(G.keys[i + 1] >> slotBits) != b) G.end[b] = i + 1;
	}
}

__global__ void k_vcm_gather(const BptwState W, VcmGrid G, uint32_t total, uint32_t maxP) {
	for(uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
		const uint32_t s = uint32_t(G.vals[i]);
		const uint32_t p = s / maxP, l = s % maxP;
		const BV& w = W.lv[size_t(l) * W.n + p];
		const BV& pw = W.lv[size_t(l - 1) * W.n + p];
		const f3 inc = bv_incident_dir(w);
		float4* o = G.photons + 5 * size_t(i);
		o[0] = make_float4(w.position.x, w.position.y, w.position.z, __int_as_float(int(l)));
		o[1] = make_float4(inc.x, inc.y, inc.z, w.incidentPdf);
		o[2] = make_float4(w.ts.geoN.x, w.ts.geoN.y, w.ts.geoN.z, w.prevConv);
		o[3] = make_float4(w.throughput.x, w.throughput.y, w.throughput.z, pw.incidentPdf);
		o[4] = make_float4(pw.prevRelSum, 0.0f, 0.0f, 0.0f);
	}
}

__global__ void k_vcm_sort_status(VcmGrid G, TraceCounters* counters) {
	if(*G.error) atomicAdd(&counters->waitErrors, 1u);
}

// ---------------------------------------------------------------- weights
// cpu_vcm.cpp:50-68: a connection of view vertex v (predecessor pv) with
// light vertex w (predecessor pw)
MBD float vcm_connection_weight(const BV& v, const BV* pv, const EvalValue& vPdf, const BV& w, const BV* pw,
                                const EvalValue& lPdf, f3 dir, float distSq, float n, float area) {
	float relSumV = 1.0f + vcm_prev_rel_sum(v, pv, vPdf.pdfB, n, area);
	float relSumL = 1.0f + vcm_prev_rel_sum(w, pw, lPdf.pdfB, n, area);
	const float lightToView = bv_convert_pdf(v, w.kind, lPdf.pdfF, dir, distSq);
	relSumV = relSumV * __fdiv_rn(lightToView, v.incidentPdf);
	if(pv) relSumV = relSumV + (lightToView * n) * area;
	const float viewToLight = bv_convert_pdf(w, v.kind, vPdf.pdfF, dir, distSq);
	relSumL = relSumL * __fdiv_rn(viewToLight, w.incidentPdf);
	if(pw) relSumL = relSumL + (viewToLight * n) * area;
	return __fdiv_rn(1.0f, (1.0f + relSumV) + relSumL);
}

// cpu_vcm.cpp:71-78: an emitter or background hit at h (predecessor pv)
MBD float vcm_hit_weight(const BV& h, const BV& pv, float pdfBack, float startPdf, float n, float area) {
	float relSum = 1.0f + vcm_prev_rel_sum(h, &pv, pdfBack, n, area);
	relSum = relSum * __fdiv_rn(startPdf, h.incidentPdf);
	return __fdiv_rn(1.0f, 1.0f + relSum);
}

// ---------------------------------------------------------------- view vertex terms
// cpu_vcm.cpp:120-146 connect and :232-246: the connection of view vertex v
// with light vertex w; returns as bpt_connect (1: a shadow ray; 0: a zero
// record in c.pix; -1: nothing).
MBD int vcm_connect(const DScene& S, uint32_t width, const BV& v, const BV* pv, const BV& w, const BV* pw, f3 thr, int px,
                    int py, const VcmConsts& C, BptConn& c) {
	int ox = px, oy = py;
	const bool possible = !((bv_ortho(v.kind) && bv_ortho(w.kind)) || (bv_ortho(v.kind) && w.kind == BV_CAMERA) ||
	                        (v.kind == BV_CAMERA && bv_ortho(w.kind)));
	const f3 full = thr * w.throughput;
	const float avgThr = __fdiv_rn((thr.x + thr.y) + thr.z, 3.0f);
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
				const float mis = vcm_connection_weight(v, pv, val0, w, pw, val1, dir, distSq, C.nPhotons, C.viewArea);
				const f3 bxdfs = bxdfProd * __fdiv_rn(mis, distSq);
				const f3 rad = (full * cosProd) * bxdfs;
				const float light = avgThr * cosProd;
				c.add = make_float4(nan_to_zero(rad.x), nan_to_zero(rad.y), nan_to_zero(rad.z), nan_to_zero(light));
				c.zeroSigns = zero_signs(full, avgThr);
				return 1;
			}
		}
	}
	if(ox == -1) return -1;
	c.pix = uint32_t(oy) * width + uint32_t(ox);
	c.zeroSigns = zero_signs(full, avgThr);
	return 0;
}

// path_util.hpp:410-458 get_emission with the weight of cpu_vcm.cpp:259-268
MBD float4 vcm_emission(const DScene& S, const BV& h, const BV& pv, f3 thr, const VcmConsts& C) {
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
			if(nonzero(value)) startPdf = light_pdfs(S, h.inst, h.prim, h.sp, pv.position).emit;
		}
	}
	if(nonzero(value)) value = value * vcm_hit_weight(h, pv, backPdf, startPdf, C.nPhotons, C.viewArea);
	const f3 rad = thr * value;
	const float light = __fdiv_rn((thr.x + thr.y) + thr.z, 3.0f) * __fdiv_rn((value.x + value.y) + value.z, 3.0f);
	return make_float4(nan_to_zero(rad.x), nan_to_zero(rad.y), nan_to_zero(rad.z), nan_to_zero(light));
}

// cpu_vcm.cpp:271-288: the merges of view vertex h (predecessor pv, path
// length viewLen, throughput thr) with the photons within the radius, and
// cpu_vcm.cpp:35-47 their weights.
MBD float4 vcm_merge(const DScene& S, const LtParams& P, const VcmGrid& G, const VcmConsts& C, const BV& h, const BV& pv,
                     int viewLen, f3 thr) {
	f3 rad = make3(0.0f, 0.0f, 0.0f);
	// a photon has at least one segment, so none fits past the max. path length
	if(viewLen + 1 <= P.maxPathLength) {
		const uint32_t base = vcm_query_hash(h.position, C.density);
		const f3 inc = bv_incident_dir(h);
		for(int cell = 0; cell < 8; ++cell) {
			uint32_t hh = base;
			if(cell & 1) hh += VCM_MAGIC_X;
			if(cell & 2) hh += VCM_MAGIC_Y;
			if(cell & 4) hh += VCM_MAGIC_Z;
			const uint32_t b = hh % C.mapSize;
			const uint32_t first = __ldg(G.start + b);
			for(uint32_t k = __ldg(G.end + b); k > first;) {
				--k;
				const float4* ph = G.photons + 5 * size_t(k);
				const float4 f0 = __ldg(ph);
				const int l = __float_as_int(f0.w);
				const int pathLen = viewLen + l;
				const f3 d = make3(f0.x, f0.y, f0.z) - h.position;
				if(l > 0 && pathLen >= P.minPathLength && pathLen <= P.maxPathLength && lensq(d) < C.radiusSq) {
					const float4 f1 = __ldg(ph + 1), f2 = __ldg(ph + 2), f3v = __ldg(ph + 3), f4 = __ldg(ph + 4);
					const f3 geoN = make3(f2.x, f2.y, f2.z);
					const EvalValue bsdf = material_evaluate(h.ts, h.mat, inc, -make3(f1.x, f1.y, f1.z), false, &geoN);
					// the weight (cpu_vcm.cpp:35-47); the photon's predecessor exists (l >= 1)
					float relSumV = 1.0f + vcm_prev_rel_sum(h, &pv, bsdf.pdfB, C.nPhotons, C.viewArea);
					const float pdfBackA = bsdf.pdfF * f2.w;
					const float relMerge = l >= 2 ? (pdfBackA * C.nPhotons) * C.viewArea : 0.0f;
					const float relConn = __fdiv_rn(pdfBackA, f3v.w);
					float relSumL = 1.0f + ((relConn + relMerge) + relConn * f4.x);
					relSumV = __fdiv_rn(relSumV, (h.incidentPdf * C.nPhotons) * C.viewArea);
					relSumL = __fdiv_rn(relSumL, (f1.w * C.nPhotons) * C.viewArea);
					const float mis = __fdiv_rn(1.0f, (1.0f + relSumV) + relSumL);
					rad = rad + (bsdf.value * make3(f3v.x, f3v.y, f3v.z)) * mis;
				}
			}
		}
	}
	const float norm = C.viewArea * C.nPhotons;
	rad = make3(__fdiv_rn(rad.x, norm), __fdiv_rn(rad.y, norm), __fdiv_rn(rad.z, norm));
	const f3 out = thr * rad;
	const float light = __fdiv_rn((thr.x + thr.y) + thr.z, 3.0f) * __fdiv_rn((rad.x + rad.y) + rad.z, 3.0f);
	return make_float4(nan_to_zero(out.x), nan_to_zero(out.y), nan_to_zero(out.z), nan_to_zero(light));
}

__host__ __device__ inline size_t vcm_slots(int maxP) { return size_t(maxP) * size_t(maxP) + 2 * size_t(maxP); }

MBD void vcm_record(const LtTargets& T, size_t slot, uint32_t pix, float4 v) {
	if(!T.recPixel) return;
	T.recPixel[slot] = int(pix);
	float* o = T.recValue + 4 * slot;
	o[0] = v.x; o[1] = v.y; o[2] = v.z; o[3] = v.w;
}

// The connections of view vertex v (path length viewLen, predecessor pv) of
// pixel p with every vertex of light subpath lp whose path length fits,
// from the subpath's end (cpu_vcm.cpp:232-246): shadow rays of generation gen
// or zero records.
MBD void vcmw_connect(const DScene& S, const LtParams& P, const LtTargets& T, const BptwState& W, const VcmConsts& C,
                      const BV& v, const BV* pv, int viewLen, uint32_t p, int px, int py, f3 thr, int gen) {
	const int maxP = P.maxPathLength > 0 ? P.maxPathLength : 1;
	const uint32_t lp = wang_hash(p) % W.n;
	const size_t base = size_t(p) * vcm_slots(maxP) + size_t(viewLen) * size_t(maxP);
	for(int l = W.lightLen[lp]; l >= 0; --l) {
		const int pathLen = l + 1 + viewLen;
		if(pathLen < P.minPathLength || pathLen > P.maxPathLength) continue;
		BptConn c;
		const BV w = bv_load(W.lv + size_t(l) * W.n + lp);
		const int k = vcm_connect(S, T.width, v, pv, w, l > 0 ? &W.lv[size_t(l - 1) * W.n + lp] : nullptr, thr, px, py, C, c);
		const size_t slot = base + size_t(l);
		if(k > 0) {
			const unsigned i = queue_reserve(W.counters + BPTW_SH0 + (gen & 1));
			W.sOrg[i] = make_float4(c.ro.x, c.ro.y, c.ro.z, c.tmax);
			W.sDir[i] = make_float4(c.rd.x, c.rd.y, c.rd.z, 0.0f);
			W.sAdd[i] = c.add;
			W.sMeta[i] = make_uint4(c.pix, uint32_t(slot), uint32_t(slot >> 32), c.zeroSigns);
		} else if(k == 0) vcm_record(T, slot, c.pix, bpt_zeros(c.zeroSigns));
	}
}

// ---------------------------------------------------------------- stages
// Every pixel: its light subpath's start vertex and first segment
// (CpuVcm::trace_photon, cpu_vcm.cpp:191-218: one number for the start
// point, the iteration's shared seed for the light tree).
__global__ void __launch_bounds__(128) k_vcmw_light_start(const DScene S, const LtParams P, const LtTargets T, BptwState W,
                                                       VcmGrid G, VcmConsts C) {
	const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
	if(p >= W.n) return;
	const int maxP = P.maxPathLength > 0 ? P.maxPathLength : 1;
	u64 rng = T.rngState[p];
	const u64 r0 = pcg_next(rng);
	const Emitter em = lights_emit(S, p, W.n, *G.seed, sample_uniform(uint32_t(r0)), sample_uniform(uint32_t(r0 >> 32)));
	int lightLen = -1;
	if(em.valid) {
		BV v;
		bpt_light_vertex(S, em, v);
		lightLen = 0;
		if(maxP > 1) {
			f3 thr = make3(1.0f, 1.0f, 1.0f), o, d;
			float pdf;
			if(bpt_sample<true>(S, v, nullptr, 0, 0, rng, true, thr, o, d, pdf, C.nPhotons, C.lightArea))
				bptw_queue_segment(W, 0, p, o, d, thr, pdf);
		}
		bv_store(W.lv + p, v);
	}
	W.lightLen[p] = lightLen;
	T.rngState[p] = rng;
}

// View phase, first generation (gen): every pixel's camera vertex, its
// connections and its first segment.
__global__ void __launch_bounds__(128, BPTW_SHADE_BLOCKS) k_vcmw_view_start(const DScene S, const LtParams P, const LtTargets T, BptwState W,
                                                         VcmConsts C, int gen) {
	const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
	if(p >= W.n) return;
	const int px = int(p % T.width), py = int(p / T.width);
	u64 rng = T.rngState[p];
	BV c;
	bpt_camera_vertex(S, px, py, c);
	(void)pcg_next(rng); // create_camera consumes one number (unused by the pinhole camera)
	f3 thr = make3(1.0f, 1.0f, 1.0f);
	vcmw_connect(S, P, T, W, C, c, nullptr, 0, p, px, py, thr, gen);
	f3 o, d;
	float pdf;
	if(bpt_sample<true>(S, c, nullptr, px, py, rng, false, thr, o, d, pdf, C.nPhotons, C.viewArea)) {
		bptw_queue_segment(W, gen, p, o, d, thr, pdf);
		bv_store(W.vp[0] + p, c);
	}
	T.rngState[p] = rng;
}

// View phase, generation gen: a segment from view vertex k becomes vertex
// k + 1; its emitter term, then unless the path ends there its merges, and
// below the max. path length its connections and next segment.
__global__ void __launch_bounds__(128, BPTW_SHADE_BLOCKS) k_vcmw_view_shade(const DScene S, const LtParams P, const LtTargets T, BptwState W,
                                                         VcmGrid G, VcmConsts C, int gen, int k) {
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
		const BV pv = bv_load(W.vp[k & 1] + p);
		BV h;
		bpt_new_vertex<true>(S, pv, ro, rd, hr, tp.w, thr, h);
		const size_t base = size_t(p) * vcm_slots(maxP) + size_t(maxP) * size_t(maxP);
		if(viewLen >= P.minPathLength) {
			const float4 add = vcm_emission(S, h, pv, thr, C);
			bpt_add(T, p, add);
			vcm_record(T, base + size_t(viewLen - 1), p, add);
		}
		// the merges and connections run in k_vcmw_merge and k_vcmw_connect:
		// with them this kernel waited on instruction fetches more than on memory
		__stcs(W.hThr + i, make_float4(thr.x, thr.y, thr.z, __uint_as_float(bv_end(h.kind) ? 0u : p + 1u)));
		if(bv_end(h.kind)) continue;
		bv_store(W.hv + i, h);
		if(viewLen >= maxP) continue;
		const int px = int(p % T.width), py = int(p / T.width);
		u64 rng = T.rngState[p];
		f3 o, d;
		float pdf;
		if(bpt_sample<true>(S, h, &pv, px, py, rng, false, thr, o, d, pdf, C.nPhotons, C.viewArea)) {
			bptw_queue_segment(W, gen + 1, p, o, d, thr, pdf);
			bv_store(W.vp[viewLen & 1] + p, h);
		}
		T.rngState[p] = rng;
	}
}

// The merges of the vertices k_vcmw_view_shade reached in generation gen
// (view path length k + 1), item by item of the same queue; the predecessors
// are still in vp[k & 1].
__global__ void __launch_bounds__(128, VCM_MERGE_BLOCKS) k_vcmw_merge(const DScene S, const LtParams P, const LtTargets T, BptwState W,
                                                    VcmGrid G, VcmConsts C, int gen, int k) {
	const int q = gen & 1;
	const unsigned count = *reinterpret_cast<volatile unsigned*>(W.counters + BPTW_EXT0 + q);
	const int maxP = P.maxPathLength > 0 ? P.maxPathLength : 1;
	const int viewLen = k + 1;
	for(unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
		const float4 tm = W.hThr[i];
		const uint32_t tag = __float_as_uint(tm.w);
		if(tag == 0u) continue;
		const uint32_t p = tag - 1u;
		const BV h = bv_load(W.hv + i);
		const BV pv = bv_load(W.vp[k & 1] + p);
		const float4 merged = vcm_merge(S, P, G, C, h, pv, viewLen, f4to3(tm));
		bpt_add(T, p, merged);
		vcm_record(T, size_t(p) * vcm_slots(maxP) + size_t(maxP) * size_t(maxP) + size_t(maxP) + size_t(viewLen - 1), p, merged);
	}
}

// The connections of the same vertices with the light subpath each pixel is
// paired with; the shadow rays go to generation gen + 1.
__global__ void __launch_bounds__(128, BPTW_CONNECT_BLOCKS) k_vcmw_connect(const DScene S, const LtParams P, const LtTargets T, BptwState W,
                                                      VcmConsts C, int gen, int k) {
	const int q = gen & 1;
	const unsigned count = *reinterpret_cast<volatile unsigned*>(W.counters + BPTW_EXT0 + q);
	const int viewLen = k + 1;
	for(unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
		const float4 tm = __ldcs(W.hThr + i);
		const uint32_t tag = __float_as_uint(tm.w);
		if(tag == 0u) continue;
		const uint32_t p = tag - 1u;
		const BV h = bv_load(W.hv + i);
		const BV pv = bv_load(W.vp[k & 1] + p);
		vcmw_connect(S, P, T, W, C, h, &pv, viewLen, p, int(p % T.width), int(p / T.width), f4to3(tm), gen + 1);
	}
}

__global__ void k_vcm_finalize(LtTargets T) {
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

// ---------------------------------------------------------------- memory
size_t al256(size_t b) { return (b + 255) & ~size_t(255); }

size_t vcm_grid_size(size_t slots, uint32_t mapSize) {
	const size_t tiles = (slots + SORT_TILE - 1) / SORT_TILE;
	return 2 * al256(slots * 8) + 2 * al256(slots * 4) + al256(tiles * 256 * 4) + al256(8 * 256 * 4) + al256(8 * 4) +
	       al256(4) + 2 * al256(size_t(mapSize) * 4) + al256(slots * 80) + al256(8) + al256(4);
}

VcmGrid vcm_grid_carve(char* m, size_t slots, uint32_t mapSize) {
	auto take = [&](size_t b) { char* r = m; m += al256(b); return r; };
	const size_t tiles = (slots + SORT_TILE - 1) / SORT_TILE;
	VcmGrid G;
	G.keys = reinterpret_cast<u64*>(take(slots * 8));
	G.keysAlt = reinterpret_cast<u64*>(take(slots * 8));
	G.vals = reinterpret_cast<int32_t*>(take(slots * 4));
	G.valsAlt = reinterpret_cast<int32_t*>(take(slots * 4));
	G.status = reinterpret_cast<uint32_t*>(take(tiles * 256 * 4));
	G.hist = reinterpret_cast<uint32_t*>(take(8 * 256 * 4));
	G.tileCounter = reinterpret_cast<unsigned*>(take(8 * 4));
	G.error = reinterpret_cast<unsigned*>(take(4));
	G.start = reinterpret_cast<uint32_t*>(take(size_t(mapSize) * 4));
	G.end = reinterpret_cast<uint32_t*>(take(size_t(mapSize) * 4));
	G.photons = reinterpret_cast<float4*>(take(slots * 80));
	G.seed = reinterpret_cast<u64*>(take(8));
	G.count = reinterpret_cast<unsigned*>(take(4));
	return G;
}

// Stable sort of the grid's photon keys by their low 8 * passes bits (passes
// even, at most 8).
cudaError_t vcm_sort(const VcmGrid& G, uint32_t n, int passes, cudaStream_t stream) {
	cudaError_t e;
	// the error word is read after the sort even when there is nothing to sort
	if((e = cudaMemsetAsync(G.error, 0, sizeof(unsigned), stream)) != cudaSuccess) return e;
	if(n <= 1) return cudaSuccess;
	static std::once_flag once;
	static cudaError_t attr = cudaSuccess;
	std::call_once(once, [] { attr = cudaFuncSetAttribute(k_onesweep, cudaFuncAttributeMaxDynamicSharedMemorySize, int(SORT_SMEM)); });
	if(attr != cudaSuccess) return attr;
	const uint32_t tiles = (n + SORT_TILE - 1) / SORT_TILE;
	if((e = cudaMemsetAsync(G.hist, 0, 8 * 256 * sizeof(uint32_t), stream)) != cudaSuccess) return e;
	if((e = cudaMemsetAsync(G.tileCounter, 0, 8 * sizeof(unsigned), stream)) != cudaSuccess) return e;
	k_sort_hist<<<std::min<unsigned>((n + 255) / 256, 148u * 8u), 256, 0, stream>>>(G.keys, n, G.hist);
	k_sort_scan<<<8, 256, 0, stream>>>(G.hist);
	u64* kin = G.keys; u64* kout = G.keysAlt;
	int32_t* vin = G.vals; int32_t* vout = G.valsAlt;
	for(int pass = 0; pass < passes; ++pass) {
		if((e = cudaMemsetAsync(G.status, 0, size_t(tiles) * 256 * sizeof(uint32_t), stream)) != cudaSuccess) return e;
		k_onesweep<<<tiles, SORT_THREADS, SORT_SMEM, stream>>>(kin, vin, kout, vout, n, 8 * pass, G.hist + 256 * pass,
		                                                       G.status, G.tileCounter + pass, G.error);
		std::swap(kin, kout);
		std::swap(vin, vout);
	}
	return cudaGetLastError(); // after an even number of passes the pairs are back in keys / vals
}

} // namespace

// HashGridManager::resize (photon_map.hpp:216-229): the next prime above
// 1.15 x the capacity (pixels x max. path length) that is 3 mod 4.
uint32_t vcm_map_size(uint32_t capacity) {
	auto prime = [](uint32_t v) {
		if(v < 2) return false;
		for(uint32_t d = 2; uint64_t(d) * d <= v; ++d) if(v % d == 0) return false;
		return true;
	};
	uint32_t v = uint32_t(float(capacity) * 1.15f);
	do { ++v; while(!prime(v)) ++v; } while((v & 3u) != 3u);
	return v;
}

size_t vcm_bytes(size_t numPixels, int maxPathLength) {
	const size_t m = size_t(maxPathLength > 0 ? maxPathLength : 1);
	const size_t slots = numPixels * m;
	return al256(bptw_size(numPixels, m)) + vcm_grid_size(slots, vcm_map_size(uint32_t(slots)));
}

cudaError_t launch_vcm(const DScene& S, const LtParams& P, const VcmSettings& V, const LtTargets& T, TraceCounters* counters,
                       cudaStream_t stream, void* memory) {
	const uint32_t n = T.width * T.height;
	if(n == 0) return cudaSuccess;
	const int maxP = P.maxPathLength > 0 ? P.maxPathLength : 1;
	// queue and photon indices are 32-bit: max. path length slots per pixel
	if(maxP > BPTW_MAX_PATH || size_t(n) * size_t(maxP) >= size_t(0xFFFFFFFFu)) return cudaErrorInvalidValue;
	const uint32_t slots = n * uint32_t(maxP);
	// the bucket count of the last size this thread launched (the prime search is cheap but not free)
	thread_local uint32_t cachedSlots = 0, cachedMap = 0;
	if(cachedSlots != slots) { cachedMap = vcm_map_size(slots); cachedSlots = slots; }
	// CpuVcm::iterate (cpu_vcm.cpp:148-157) and the areas of trace_photon / sample
	const float dx = S.aabbMax[0] - S.aabbMin[0], dy = S.aabbMax[1] - S.aabbMin[1], dz = S.aabbMax[2] - S.aabbMin[2];
	const float diag = std::sqrt((dx * dx + dy * dy) + dz * dz);
	float radius = V.mergeRadius * diag;
	if(V.progressive) radius *= std::pow(float(T.iteration + 1), -1.0f / 6.0f);
	VcmConsts C;
	C.nPhotons = float(n);
	C.lightArea = PI * radius * radius;
	C.radiusSq = radius * radius;
	C.viewArea = PI * C.radiusSq;
	C.density = 1.0f / (radius * 2.0001f);
	C.mapSize = cachedMap;
	auto bits = [](uint64_t v) { int b = 0; while(v) { ++b; v >>= 1; } return b; };
	C.slotBits = bits(uint64_t(slots) - 1);
	// key bits: bucket and slot, sorted 8 per pass in an even number of passes
	const int keyBits = bits(uint64_t(C.mapSize) - 1) + C.slotBits;
	if(keyBits > 64) return cudaErrorInvalidValue;
	const int passes = std::max(2, ((keyBits + 15) / 16) * 2);

	cudaError_t e;
	if((e = cudaMemsetAsync(T.iter, 0, size_t(n) * sizeof(float4), stream)) != cudaSuccess) return e;
	if(T.recPixel) {
		const size_t rs = size_t(n) * vcm_slots(maxP);
		if((e = cudaMemsetAsync(T.recPixel, 0xFF, rs * sizeof(int32_t), stream)) != cudaSuccess) return e;
		if((e = cudaMemsetAsync(T.recValue, 0, rs * 4 * sizeof(float), stream)) != cudaSuccess) return e;
	}
	char* mem = static_cast<char*>(memory);
	const BptwState W = bptw_carve(mem, n, size_t(maxP));
	const VcmGrid G = vcm_grid_carve(mem + al256(bptw_size(n, size_t(maxP))), slots, C.mapSize);
	if((e = cudaMemsetAsync(W.counters, 0, BPTW_COUNTERS * sizeof(unsigned), stream)) != cudaSuccess) return e;
	const int tb = bptw_trace_blocks();
	int dev = 0, sms = 148;
	cudaGetDevice(&dev);
	cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
	auto trace = [&](int gen) {
		if(S.hasAlpha) k_bptw_trace<ALPHA_ALWAYS><<<tb, 128, 0, stream>>>(S, T, W, gen, counters);
		else k_bptw_trace<ALPHA_NEVER><<<tb, 128, 0, stream>>>(S, T, W, gen, counters);
	};
	// light phase
	k_vcm_seed<<<1, 1, 0, stream>>>(T, G);
	k_vcmw_light_start<<<(n + 127) / 128, 128, 0, stream>>>(S, P, T, W, G, C);
	const int lightGens = maxP - 1;
	for(int g = 0; g < lightGens; ++g) {
		trace(g);
		k_bptw_light_shade<true><<<sms * BPTW_SHADE_BLOCKS, 128, 0, stream>>>(S, P, T, W, g, C.nPhotons, C.lightArea);
	}
	// photon grid: the photons' keys, their count (read back to size the
	// sort), the sort, the bucket ranges and the packed merge data
	const unsigned gb = std::min<unsigned>((slots + 255) / 256, unsigned(sms) * 16u);
	if((e = cudaMemsetAsync(G.count, 0, sizeof(unsigned), stream)) != cudaSuccess) return e;
	k_vcm_keys<<<gb, 256, 0, stream>>>(W, G, C, uint32_t(maxP));
	unsigned photons = 0;
	if((e = cudaMemcpyAsync(&photons, G.count, sizeof(unsigned), cudaMemcpyDeviceToHost, stream)) != cudaSuccess) return e;
	if((e = cudaStreamSynchronize(stream)) != cudaSuccess) return e;
	if((e = vcm_sort(G, photons, passes, stream)) != cudaSuccess) return e;
	k_vcm_sort_status<<<1, 1, 0, stream>>>(G, counters);
	if((e = cudaMemsetAsync(G.start, 0, size_t(C.mapSize) * 4, stream)) != cudaSuccess) return e;
	if((e = cudaMemsetAsync(G.end, 0, size_t(C.mapSize) * 4, stream)) != cudaSuccess) return e;
	if(photons > 0) {
		const unsigned pb = std::min<unsigned>((photons + 255) / 256, unsigned(sms) * 16u);
		k_vcm_ranges<<<pb, 256, 0, stream>>>(G, photons, C.slotBits);
		k_vcm_gather<<<pb, 256, 0, stream>>>(W, G, photons, uint32_t(maxP));
	}
	// view phase
	k_vcmw_view_start<<<(n + 127) / 128, 128, 0, stream>>>(S, P, T, W, C, lightGens);
	for(int k = 0; k < maxP; ++k) {
		trace(lightGens + k);
		k_vcmw_view_shade<<<sms * BPTW_SHADE_BLOCKS, 128, 0, stream>>>(S, P, T, W, G, C, lightGens + k, k);
		k_vcmw_merge<<<sms * VCM_MERGE_BLOCKS, 128, 0, stream>>>(S, P, T, W, G, C, lightGens + k, k);
		if(k + 1 < maxP) k_vcmw_connect<<<sms * BPTW_CONNECT_BLOCKS, 128, 0, stream>>>(S, P, T, W, C, lightGens + k, k);
	}
	if((e = cudaGetLastError()) != cudaSuccess) return e;
	k_vcm_finalize<<<(n + 255) / 256, 256, 0, stream>>>(T);
	return cudaGetLastError();
}

} // namespace mb
