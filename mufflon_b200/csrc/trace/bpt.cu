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
#include "bidir.cuh"

namespace mb {
namespace {

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
				c.zeroSigns = zero_signs(full, __fdiv_rn((full.x + full.y) + full.z, 3.0f));
				return 1;
			}
		}
	}
	if(ox == -1) return -1;
	c.pix = uint32_t(oy) * width + uint32_t(ox);
	const f3 full = thr * w.throughput;
	c.zeroSigns = zero_signs(full, __fdiv_rn((full.x + full.y) + full.z, 3.0f));
	return 0;
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
		bpt_camera_vertex(S, px, py, vp[0]);
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
			if(bpt_sample<false>(S, v, lightLen > 0 ? &lp[lightLen - 1] : nullptr, px, py, rng, true, lthr, ro, rd, segPdf)) trace = true;
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
				if(k == 0) rec.put(size_t(viewLen) * size_t(maxP) + size_t(l), conn.pix, bpt_zeros(conn.zeroSigns));
				++l;
			}
			if(!trace) phase = BP_VWALK;
		}
		if(mine && pick == BP_VWALK && !trace && phase == BP_VWALK) {
			BV& v = vp[cur];
			if(bpt_sample<false>(S, v, viewLen > 0 ? &vp[1 - cur] : nullptr, px, py, rng, false, thr, ro, rd, segPdf)) {
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
				bpt_new_vertex<false>(S, lp[lightLen], ro, rd, t.best, segPdf, lthr, lp[lightLen + 1]);
				++lightLen;
				if(lightLen >= maxP - 1) start_view();
			}
		} else {
			const int nxt = 1 - cur;
			bpt_new_vertex<false>(S, vp[cur], ro, rd, t.best, segPdf, thr, vp[nxt]);
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
// The connections of view vertex v (path length viewLen, predecessor pv) with
// light vertices lo .. hi-1 of pixel p: shadow rays of generation gen, or
// the zero records of those that carry nothing.
MBD void bptw_connect(const DScene& S, const LtParams& P, const LtTargets& T, const BptwState& W, const BV& v, const BV* pv,
                      int viewLen, uint32_t p, int px, int py, f3 thr, int lo, int hi, int gen) {
	const size_t maxP = size_t(P.maxPathLength > 0 ? P.maxPathLength : 1);
	const size_t base = size_t(p) * (maxP * maxP + maxP) + size_t(viewLen) * maxP;
	for(int l = lo; l < hi; ++l) {
		BptConn c;
		const BV w = bv_load(W.lv + size_t(l) * W.n + p);
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
			const float4 z = bpt_zeros(c.zeroSigns);
			float* o = T.recValue + 4 * slot;
			o[0] = z.x; o[1] = z.y; o[2] = z.z; o[3] = z.w;
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
			if(bpt_sample<false>(S, v, nullptr, 0, 0, rng, true, thr, o, d, pdf)) bptw_queue_segment(W, 0, p, o, d, thr, pdf);
		}
		bv_store(W.lv + p, v);
	}
	W.lightLen[p] = lightLen;
	T.rngState[p] = rng;
}

// View phase, first generation (gen): every pixel's camera vertex, its
// connections with the light subpath and its first segment.
__global__ void __launch_bounds__(128, BPTW_SHADE_BLOCKS) k_bptw_view_start(const DScene S, const LtParams P, const LtTargets T, BptwState W,
                                                         int gen) {
	const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
	if(p >= W.n) return;
	const int maxP = P.maxPathLength > 0 ? P.maxPathLength : 1;
	const int px = int(p % T.width), py = int(p / T.width);
	u64 rng = T.rngState[p];
	BV c;
	bpt_camera_vertex(S, px, py, c);
	(void)pcg_next(rng); // create_camera consumes one number (unused by the pinhole camera)
	f3 thr = make3(1.0f, 1.0f, 1.0f);
	const int lightLen = W.lightLen[p];
	bptw_connect(S, P, T, W, c, nullptr, 0, p, px, py, thr, max(0, P.minPathLength - 1), min(lightLen + 1, maxP), gen);
	f3 o, d;
	float pdf;
	if(bpt_sample<false>(S, c, nullptr, px, py, rng, false, thr, o, d, pdf)) {
		bptw_queue_segment(W, gen, p, o, d, thr, pdf);
		bv_store(W.vp[0] + p, c);
	}
	T.rngState[p] = rng;
}

// View phase, generation gen: a segment from view vertex k (k + 1 < path
// length) becomes vertex k + 1 (a surface or a miss): what it adds by
// reaching an emitter or the background, then, unless the path ends there,
// its connections and its segment of generation gen + 1.
__global__ void __launch_bounds__(128, BPTW_SHADE_BLOCKS) k_bptw_view_shade(const DScene S, const LtParams P, const LtTargets T, BptwState W,
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
		const BV pv = bv_load(W.vp[k & 1] + p);
		BV h;
		bpt_new_vertex<false>(S, pv, ro, rd, hr, tp.w, thr, h);
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
		// the connections run in k_bptw_connect: with them this kernel waited
		// on instruction fetches more than on memory
		const bool more = !bv_end(h.kind) && viewLen < maxP;
		__stcs(W.hThr + i, make_float4(thr.x, thr.y, thr.z, __uint_as_float(more ? p + 1u : 0u)));
		if(!more) continue;
		bv_store(W.hv + i, h);
		const int px = int(p % T.width), py = int(p / T.width);
		u64 rng = T.rngState[p];
		f3 o, d;
		float pdf;
		if(bpt_sample<false>(S, h, &pv, px, py, rng, false, thr, o, d, pdf)) {
			bptw_queue_segment(W, gen + 1, p, o, d, thr, pdf);
			bv_store(W.vp[viewLen & 1] + p, h);
		}
		T.rngState[p] = rng;
	}
}

// The connections of the vertices k_bptw_view_shade reached in generation gen
// (view path length k + 1) with their pixels' light subpaths, item by item of
// the same queue; the predecessors are still in vp[k & 1]. The shadow rays go
// to generation gen + 1.
__global__ void __launch_bounds__(128, BPTW_CONNECT_BLOCKS) k_bptw_connect(const DScene S, const LtParams P, const LtTargets T, BptwState W,
                                                      int gen, int k) {
	const int q = gen & 1;
	const unsigned count = *reinterpret_cast<volatile unsigned*>(W.counters + BPTW_EXT0 + q);
	const int maxP = P.maxPathLength > 0 ? P.maxPathLength : 1;
	const int viewLen = k + 1;
	for(unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
		const float4 tm = __ldcs(W.hThr + i);
		const uint32_t tag = __float_as_uint(tm.w);
		if(tag == 0u) continue;
		const uint32_t p = tag - 1u;
		const BV h = bv_load(W.hv + i);
		const BV pv = bv_load(W.vp[k & 1] + p);
		const int lightLen = W.lightLen[p];
		bptw_connect(S, P, T, W, h, &pv, viewLen, p, int(p % T.width), int(p / T.width), f4to3(tm),
		             max(0, P.minPathLength - viewLen - 1), min(lightLen + 1, maxP - viewLen), gen + 1);
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
			k_bptw_light_shade<false><<<sms * BPTW_SHADE_BLOCKS, 128, 0, stream>>>(S, P, T, W, g);
		}
		k_bptw_view_start<<<(n + 127) / 128, 128, 0, stream>>>(S, P, T, W, lightGens);
		for(int k = 0; k < maxP; ++k) {
			trace(lightGens + k);
			k_bptw_view_shade<<<sms * BPTW_SHADE_BLOCKS, 128, 0, stream>>>(S, P, T, W, lightGens + k, k);
			if(k + 1 < maxP) k_bptw_connect<<<sms * BPTW_CONNECT_BLOCKS, 128, 0, stream>>>(S, P, T, W, lightGens + k, k);
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
