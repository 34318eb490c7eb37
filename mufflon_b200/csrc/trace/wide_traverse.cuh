// Traversal of the compressed 8-wide hierarchies (lbvh/wide.hpp) for closest
// hits and shadow rays; the counterpart of intersection.cu:319-492 and
// 624-753 of the reference, over a different hierarchy with the same result.
//
// One loop runs both levels. The state of a ray is
//   * a node group: the child base of the last visited node, its internal-slot
//     mask and the still unvisited hit internal children as bits in
//     traversal order (bit k = slot k ^ flip, flip chosen from the ray's
//     direction octant so that bit order is roughly near to far),
//   * a primitive group: the last visited node's primitive base and one bit
//     per primitive of its hit leaves,
//   * a stack of node groups (and, at the instance level, primitive groups of
//     instances not yet entered).
// Entering an instance transforms the ray into object space and remembers the
// stack depth; when the object level's groups are exhausted at that depth the
// world ray is restored. Every step visits one node (eight box tests that do
// the same arithmetic in every lane) and then that node's hit primitives.
//
// The box test cannot cull a box that contains a hit point (wide.hpp), so the
// closest hit is the minimum of (world t, instance, primitive) over all
// primitive hits, exactly as with the binary hierarchy.
#pragma once

#include "intersect.cuh"
#include "../lbvh/wide.hpp"

namespace mb {

constexpr int WIDE_STACK = 64;

// The traversal stack of one ray. The node group being visited lives in
// registers (WideTracer::ngBase/ngImask/ngHits, pgBase/pgHits); pushed groups
// go to this per-thread array in local memory, which the L1 cache serves.
// (Keeping the first 4, 8 or 16 entries in shared memory instead, thread-
// interleaved, measured 5-7 % slower in the trace kernel on the B200.)
struct LocalStack {
	uint2 e[WIDE_STACK];
	MBD void put(int i, uint2 v) { e[i] = v; }
	MBD uint2 get(int i) const { return e[i]; }
};
constexpr uint32_t PRIM_GROUP = 0x80000000u;
// Primitive masks use bits 0..8*leafMax-1; bit 31 tags primitive groups.
static_assert(8 * WIDE_LEAF_MAX <= 31 && 8 * WIDE_TLAS_LEAF_MAX <= 31, "primitive mask width");

MBD uint32_t octant_flip(f3 d) {
	return 7u ^ ((d.x < 0.0f ? 4u : 0u) | (d.y < 0.0f ? 2u : 0u) | (d.z < 0.0f ? 1u : 0u));
}

// Byte b (0..3) of w as an exact float: 0x4B0000bb is the float 2^23 + bb.
MBD float qbyte(uint32_t w, int b) {
	return __fsub_rn(__int_as_float(int(__byte_perm(w, 0x4B000000u, 0x7440u | uint32_t(b)))), 8388608.0f);
}

// Out-of-line pieces of the traversal loop that run at most a few times per
// ray (instance transitions) or rarely (non-triangle primitives); keeping them
// out of the loop body keeps the loop in the instruction cache.
static __device__ __noinline__ FastRay make_ray_ool(f3 o, f3 d) { return make_ray(o, d); }
static __device__ __noinline__ InstRay instance_ray_ool(const DScene& S, uint32_t i, f3 o, f3 d) {
	return instance_ray(load_w2i(S, i), o, d);
}
struct PrimHit { float t; f2 uv; bool hit; };
static __device__ __noinline__ PrimHit other_prim_test(const DLod* l, FastRay r, int p) {
	PrimHit h;
	h.hit = prim_test(*l, r, 0, p, h.t, h.uv);
	return h;
}
static __device__ __noinline__ PrimHit other_prim_test_alpha(const DLod* l, FastRay r, int p, AlphaCtx alpha) {
	PrimHit h;
	h.hit = prim_test(*l, r, 0, p, h.t, h.uv, alpha);
	return h;
}

// Three-operand minimum and maximum of sm_100 (one instruction each; a NaN
// operand is dropped like fminf/fmaxf drop it).
MBD float min3_(float a, float b, float c) {
	float d;
	asm("min.f32 %0, %1, %2, %3;" : "=f"(d) : "f"(a), "f"(b), "f"(c));
	return d;
}
MBD float max3_(float a, float b, float c) {
	float d;
	asm("max.f32 %0, %1, %2, %3;" : "=f"(d) : "f"(a), "f"(b), "f"(c));
	return d;
}

// Tests the eight child boxes of node `idx`; returns the child's node group
// and primitive group. A child is hit when
//   max(near planes, 0) <= min(far planes * (1 + 2^-20), tmaxBox).
// The far-plane tolerance is applied to the per-node scale and offset, not per
// child; that moves a far plane by a few ulp of its t, far less than the grid
// step of margin every quantised box carries, so the test stays conservative.
MBD void wide_node_test(const WideNode* nodes, uint32_t idx, const FastRay& r, uint32_t flip, float tmaxBox,
                        uint32_t& ngBase, uint32_t& ngImask, uint32_t& ngHits, uint32_t& pgBase, uint32_t& pgHits) {
	const float4* q = reinterpret_cast<const float4*>(nodes + idx);
	const float4 n0 = __ldg(q), n1 = __ldg(q + 1), n2 = __ldg(q + 2), n3 = __ldg(q + 3), n4 = __ldg(q + 4);
	const uint32_t eim = __float_as_uint(n0.w);
	const float sx = __fmul_rn(__uint_as_float((eim & 0xFFu) << 23), r.inv.x);
	const float sy = __fmul_rn(__uint_as_float(((eim >> 8) & 0xFFu) << 23), r.inv.y);
	const float sz = __fmul_rn(__uint_as_float(((eim >> 16) & 0xFFu) << 23), r.inv.z);
	const float ox = __fmul_rn(__fsub_rn(n0.x, r.o.x), r.inv.x);
	const float oy = __fmul_rn(__fsub_rn(n0.y, r.o.y), r.inv.y);
	const float oz = __fmul_rn(__fsub_rn(n0.z, r.o.z), r.inv.z);
	const float fsx = __fmul_rn(sx, BOX_FAR_SLACK), fsy = __fmul_rn(sy, BOX_FAR_SLACK), fsz = __fmul_rn(sz, BOX_FAR_SLACK);
	const float fox = __fmul_rn(ox, BOX_FAR_SLACK), foy = __fmul_rn(oy, BOX_FAR_SLACK), foz = __fmul_rn(oz, BOX_FAR_SLACK);
	const uint32_t imask = eim >> 24;
	const bool fx = r.inv.x < 0.0f, fy = r.inv.y < 0.0f, fz = r.inv.z < 0.0f;
	const uint32_t lx0 = __float_as_uint(n2.x), lx1 = __float_as_uint(n2.y);
	const uint32_t ly0 = __float_as_uint(n2.z), ly1 = __float_as_uint(n2.w);
	const uint32_t lz0 = __float_as_uint(n3.x), lz1 = __float_as_uint(n3.y);
	const uint32_t hx0 = __float_as_uint(n3.z), hx1 = __float_as_uint(n3.w);
	const uint32_t hy0 = __float_as_uint(n4.x), hy1 = __float_as_uint(n4.y);
	const uint32_t hz0 = __float_as_uint(n4.z), hz1 = __float_as_uint(n4.w);
	const uint32_t nx[2] = { fx ? hx0 : lx0, fx ? hx1 : lx1 }, fxw[2] = { fx ? lx0 : hx0, fx ? lx1 : hx1 };
	const uint32_t ny[2] = { fy ? hy0 : ly0, fy ? hy1 : ly1 }, fyw[2] = { fy ? ly0 : hy0, fy ? ly1 : hy1 };
	const uint32_t nz[2] = { fz ? hz0 : lz0, fz ? hz1 : lz1 }, fzw[2] = { fz ? lz0 : hz0, fz ? lz1 : hz1 };
	const uint32_t meta[2] = { __float_as_uint(n1.z), __float_as_uint(n1.w) };
	uint32_t nh = 0, ph = 0;
#pragma unroll
	for(int i = 0; i < 8; ++i) {
		const int w = i >> 2, b = i & 3;
		const float tnx = __fmaf_rn(qbyte(nx[w], b), sx, ox);
		const float tny = __fmaf_rn(qbyte(ny[w], b), sy, oy);
		const float tnz = __fmaf_rn(qbyte(nz[w], b), sz, oz);
		const float tfx = __fmaf_rn(qbyte(fxw[w], b), fsx, fox);
		const float tfy = __fmaf_rn(qbyte(fyw[w], b), fsy, foy);
		const float tfz = __fmaf_rn(qbyte(fzw[w], b), fsz, foz);
		const float tnear = max3_(tnx, tny, fmax_(tnz, 0.0f));
		const float tfar = min3_(tfx, tfy, fmin_(tfz, tmaxBox));
		if(tnear <= tfar) {
			if(imask & (1u << i)) {
				nh |= 1u << (uint32_t(i) ^ flip);
			} else {
				const uint32_t m = (meta[w] >> (8 * b)) & 0xFFu;
				ph |= ((1u << (m >> 5)) - 1u) << (m & 31u);
			}
		}
	}
	ngBase = __float_as_uint(n1.x);
	ngImask = imask;
	ngHits = nh;
	pgBase = __float_as_uint(n1.y);
	pgHits = ph;
}

// Resumable traversal of one ray: init() sets it up, every step() visits at
// most one node and that node's hit primitives (or enters / leaves an
// instance), and returns true once the ray is finished. Kernels that refill
// lanes as soon as their ray finishes call step() from one loop shared by the
// whole warp. Alpha mode AM: ALPHA_NEVER, every surface is opaque (scenes
// without alpha textures, and the wireframe renderer's
// first_intersection<CURRENT_DEV, false>, wireframe_common.hpp:108);
// ALPHA_ALWAYS, the materials' alpha textures apply (kernels launched for
// scenes with alpha textures); ALPHA_SCENE, decided per step by the scene.
enum AlphaMode { ALPHA_NEVER = 0, ALPHA_ALWAYS = 1, ALPHA_SCENE = 2 };
template < int AM >
struct WideTracerT {
	FastRay wr;           // world ray, prepared (wr.o, wr.d: the ray as given)
	FastRay r;            // ray of the current level
	float scale;          // object-space length of a world-space unit
	float tmaxW;          // shadow rays: world-space segment length
	HitRec best;          // closest hit so far (best.t holds the incoming tmax)
	const DLod* lod;
	const WideNode* nodes;
	uint32_t flip, ngBase, ngImask, ngHits, pgBase, pgHits;
	int inst, sp, instSp, steps; // steps: what is left of the scene's step limit
	bool any, single, occluded, done;

	template < class C >
	MBD void init(const DScene& S, f3 o, f3 d, float tmax, bool anyHit, C& cnt) {
		tmaxW = tmax;
		any = anyHit;
		occluded = false;
		best.t = tmax; best.inst = -1; best.prim = -1; best.sp = make2(0.0f, 0.0f); best.has = false;
		sp = 0; instSp = -1; steps = S.maxSteps; inst = -1; lod = nullptr;
		scale = 1.0f;
		ngBase = 0; ngImask = 1; ngHits = 0; pgBase = 0; pgHits = 0;
		single = S.activeInstances == 1;
		done = S.activeInstances <= 0;
		if(done) return;
		wr = make_ray_ool(o, d);
		r = wr;
		flip = octant_flip(d);
		nodes = S.tlasWide;
		if(single) enter(S, uint32_t(S.validInstance), cnt);
		else ngHits = S.tlasNumWide > 0 ? (1u << flip) : 0u;
	}

	template < class C >
	MBD void enter(const DScene& S, uint32_t i, C& cnt) {
		++cnt.instances;
		inst = int(i);
		lod = S.lods + __ldg(S.instanceLod + i);
		const InstRay ir = instance_ray_ool(S, i, wr.o, wr.d);
		r = ir.ray;
		scale = ir.scale;
		flip = octant_flip(r.d);
		nodes = lod->wnodes;
		const int np = lod->numPrims;
		ngBase = 0; ngImask = 1; ngHits = 0; pgBase = 0; pgHits = 0;
		if(np >= 2) ngHits = 1u << flip; // the root, slot 0 of a virtual parent
		else if(np == 1) pgHits = 1u;
		instSp = sp;
	}

	// One step. The hot kernels are compiled once per alpha mode and launched
	// with ALPHA_NEVER for scenes without alpha textures, so their step carries
	// no alpha code (any alpha check in a step shared by both kinds of scenes
	// made the trace stage 5-7 % slower: more registers spilled).
	template < class Stack, class C >
	MBD bool step(const DScene& S, C& cnt, Stack& stack) {
		if constexpr(AM == ALPHA_SCENE) {
			if(S.hasAlpha) return step_impl<true>(S, cnt, stack);
			return step_impl<false>(S, cnt, stack);
		} else {
			return step_impl<AM == ALPHA_ALWAYS>(S, cnt, stack);
		}
	}

	template < bool ALPHA, class Stack, class C >
	MBD bool step_impl(const DScene& S, C& cnt, Stack& stack) {
		if(done) return true;
		if(--steps < 0) { ++cnt.errors; done = true; return true; }
		if(ngHits) {
			const uint32_t k = uint32_t(__ffs(int(ngHits)) - 1);
			ngHits &= ngHits - 1u;
			const uint32_t s = k ^ flip;
			const uint32_t child = ngBase + uint32_t(__popc(ngImask & ((1u << s) - 1u)));
			if(ngHits) {
				if(sp >= WIDE_STACK) { ++cnt.errors; done = true; return true; }
				stack.put(sp++, make_uint2(ngBase, ngImask | (ngHits << 8)));
			}
			++cnt.nodes;
			const float tmaxBox = (any ? tmaxW : best.t) * scale * BOX_SLACK;
			wide_node_test(nodes, child, r, flip, tmaxBox, ngBase, ngImask, ngHits, pgBase, pgHits);
		}
		if(pgHits) {
			if(instSp >= 0) {
				const float4* soup = lod->wsoup;
				const uint32_t ntri = lod->numTriangles;
				do {
					const uint32_t j = uint32_t(__ffs(int(pgHits)) - 1);
					pgHits &= pgHits - 1u;
					// all three rows at once (every primitive has them), so a
					// triangle costs one round trip to memory, not two
					const float4* s4 = soup + 3 * size_t(pgBase + j);
					const float4 a = __ldg(s4), b = __ldg(s4 + 1), c = __ldg(s4 + 2);
					const int p = __float_as_int(a.w);
					++cnt.prims;
					float t;
					f2 uv;
					bool hit;
					if(uint32_t(p) < ntri) {
						hit = tri_test(r, f4to3(a), f4to3(b), f4to3(c), t, uv) && t > 0.0f;
						if(ALPHA && hit) hit = !alpha_cuts_triangle(alpha_ctx(S), *lod, p, uv);
					} else {
						const PrimHit ph = ALPHA ? other_prim_test_alpha(lod, r, p, alpha_ctx(S)) : other_prim_test(lod, r, p);
						hit = ph.hit; t = ph.t; uv = ph.uv;
					}
					if(hit) {
						if(any) {
							if(t < tmaxW * scale) { occluded = true; done = true; return true; }
						} else {
							const float tw = __fdiv_rn(t, scale);
							if(better(tw, inst, p, best)) { best.t = tw; best.inst = inst; best.prim = p; best.sp = uv; best.has = true; }
						}
					}
				} while(pgHits);
			} else {
				// instance leaves of the top level: enter one, keep the rest
				const uint32_t j = uint32_t(__ffs(int(pgHits)) - 1);
				pgHits &= pgHits - 1u;
				const uint32_t id = uint32_t(__ldg(S.tlasWidePrims + pgBase + j));
				if(sp + 2 > WIDE_STACK) { ++cnt.errors; done = true; return true; }
				if(ngHits) stack.put(sp++, make_uint2(ngBase, ngImask | (ngHits << 8)));
				if(pgHits) stack.put(sp++, make_uint2(pgBase, pgHits | PRIM_GROUP));
				enter(S, id, cnt);
				return false;
			}
		}
		if(!ngHits) {
			if(instSp >= 0 && sp == instSp) {
				if(single) { done = true; return true; }
				r = wr;
				flip = octant_flip(wr.d);
				scale = 1.0f;
				nodes = S.tlasWide;
				instSp = -1;
			}
			if(sp == 0) { done = true; return true; }
			const uint2 e = stack.get(--sp);
			if(e.y & PRIM_GROUP) { pgBase = e.x; pgHits = e.y & ~PRIM_GROUP; }
			else { ngBase = e.x; ngImask = e.y & 0xFFu; ngHits = e.y >> 8; }
		}
		return false;
	}

};

using WideTracer = WideTracerT<ALPHA_SCENE>;

// Closest hit of a world-space ray whose origin is already offset.
template < int AM = ALPHA_SCENE, class Stack, class C >
MBD HitRec closest_hit_wide(const DScene& S, f3 o, f3 dir, float tmax, C& cnt, Stack& stack) {
	++cnt.rays;
	WideTracerT<AM> t;
	t.init(S, o, dir, tmax, false, cnt);
	while(!t.step(S, cnt, stack)) {}
	return t.best;
}

// Occlusion of a prepared shadow ray (origin offset, unit direction, length tmax).
template < class Stack, class C >
MBD bool occluded_wide(const DScene& S, f3 a, f3 dir, float tmax, C& cnt, Stack& stack) {
	++cnt.rays; ++cnt.shadow;
	WideTracerT<ALPHA_SCENE> t;
	t.init(S, a, dir, tmax, true, cnt);
	while(!t.step(S, cnt, stack)) {}
	return t.occluded;
}

} // namespace mb
