// Two-level BVH traversal and primitive tests on the device.
//
// Behaviour follows src/core/scene/accel_structs/intersection.cu:16-753:
//   * add_epsilon origin offset (intersection.cu:16-24),
//   * two-level traversal with an object-space transition per instance
//     (intersection.cu:319-361), single-primitive LoDs without a BVH,
//   * triangle, bilinear quad (Ramsey 2004) and sphere tests,
//   * hit attribute synthesis (intersection.cu:511-620) and
//     tangent_space_geom_to_shader (tangent_space.hpp:10-66).
// Closest hits are ordered by (world t, instance, primitive), which makes the
// result independent of the traversal order, and boxes are culled against
// tmax * (1 + 2^-16). The CPU oracle uses the same rules, so both report the
// same hit for every ray.
#pragma once

#include "dmath.cuh"
#include "scene_types.hpp"

namespace mb {

constexpr int BLAS_STACK = 100;
constexpr int TLAS_STACK = 64;

struct FastRay {
	f3 o, d, inv;
	int kx, ky, kz;
	float Sx, Sy, Sz;
};

// Reciprocal of a direction component for the slab tests, clamped to
// +-2^64. With an infinite reciprocal (a zero component), an offset of 0 in a
// slab test gives 0 * inf = NaN, which the min/max chains drop; in the 8-wide
// test every child plane on the node's origin has offset 0, so that axis
// stops culling and a ray along a coordinate axis visits every box (one such
// photon ray took a second). The finite value keeps the culling: a box whose
// slab holds the ray's constant coordinate spans t = -2^64 * d .. +2^64 * d
// and is kept, one whose slab does not starts beyond any ray length. Hits
// depend on the choice only for a ray lying exactly in a box's face plane.
MBD float slab_rcp(float x) {
	return fminf(fmaxf(__fdiv_rn(1.0f, x), -18446744073709551616.0f), 18446744073709551616.0f);
}

MBD FastRay make_ray(f3 o, f3 d) {
	FastRay r;
	r.o = o;
	r.d = d;
	r.inv = make3(slab_rcp(d.x), slab_rcp(d.y), slab_rcp(d.z));
	const float ax = fabsf(d.x), ay = fabsf(d.y), az = fabsf(d.z);
	int kz = (ax >= ay && ax >= az) ? 0 : (ay >= az ? 1 : 2);
	int kx = kz + 1 == 3 ? 0 : kz + 1;
	int ky = kx + 1 == 3 ? 0 : kx + 1;
	if(d[kz] < 0.0f) { const int t = kx; kx = ky; ky = t; }
	r.kx = kx; r.ky = ky; r.kz = kz;
	r.Sx = __fdiv_rn(d[kx], d[kz]);
	r.Sy = __fdiv_rn(d[ky], d[kz]);
	r.Sz = __fdiv_rn(1.0f, d[kz]);
	return r;
}

// Slab test of intersection.cu:47-55 in a robust form: per axis
// t = (bound - origin) * invDir, which has a relative error of a few ulp and
// the exact sign (the reference's fma(bound, invDir, -origin * invDir) errs
// relative to the origin's magnitude); the entry is clamped at 0 and the
// interval is accepted up to far * (1 + 2^-20). A box that contains a
// primitive's hit point is therefore never culled, and every hierarchy over
// the same primitives yields the same closest hit.
MBD bool box_test(float mnx, float mny, float mnz, float mxx, float mxy, float mxz,
                  const FastRay& r, float tmax, float& cmin) {
	const float lox = __fmul_rn(__fsub_rn(mnx, r.o.x), r.inv.x);
	const float loy = __fmul_rn(__fsub_rn(mny, r.o.y), r.inv.y);
	const float loz = __fmul_rn(__fsub_rn(mnz, r.o.z), r.inv.z);
	const float hix = __fmul_rn(__fsub_rn(mxx, r.o.x), r.inv.x);
	const float hiy = __fmul_rn(__fsub_rn(mxy, r.o.y), r.inv.y);
	const float hiz = __fmul_rn(__fsub_rn(mxz, r.o.z), r.inv.z);
	cmin = fmax_(fmax_(fmin_(lox, hix), fmin_(loy, hiy)), fmax_(fmin_(loz, hiz), 0.0f));
	const float cfar = fmin_(fmin_(fmax_(lox, hix), fmax_(loy, hiy)), fmax_(loz, hiz));
	return cmin <= tmax && cmin <= cfar * BOX_FAR_SLACK;
}

// Edge functions in double precision, the watertight test's fallback when a
// single-precision edge function is exactly zero (kept out of line: rare).
static __device__ __noinline__ float3 edge_functions_double(float Ax, float Ay, float Bx, float By, float Cx, float Cy) {
	return make_float3(float(__dsub_rn(__dmul_rn(double(Cx), double(By)), __dmul_rn(double(Cy), double(Bx)))),
	                   float(__dsub_rn(__dmul_rn(double(Ax), double(Cy)), __dmul_rn(double(Ay), double(Cx)))),
	                   float(__dsub_rn(__dmul_rn(double(Bx), double(Ay)), __dmul_rn(double(By), double(Ax)))));
}

// Watertight ray/triangle test (Woop, Benthin, Wald, JCGT 2013).
MBD bool tri_test(const FastRay& r, f3 v0, f3 v1, f3 v2, float& t, f2& bary) {
	const f3 A = v0 - r.o, B = v1 - r.o, C = v2 - r.o;
	const float Ax = A[r.kx] - r.Sx * A[r.kz];
	const float Ay = A[r.ky] - r.Sy * A[r.kz];
	const float Bx = B[r.kx] - r.Sx * B[r.kz];
	const float By = B[r.ky] - r.Sy * B[r.kz];
	const float Cx = C[r.kx] - r.Sx * C[r.kz];
	const float Cy = C[r.ky] - r.Sy * C[r.kz];
	float U = Cx * By - Cy * Bx;
	float V = Ax * Cy - Ay * Cx;
	float W = Bx * Ay - By * Ax;
	if(U == 0.0f || V == 0.0f || W == 0.0f) {
		const float3 uvw = edge_functions_double(Ax, Ay, Bx, By, Cx, Cy);
		U = uvw.x; V = uvw.y; W = uvw.z;
	}
	if((U < 0.0f || V < 0.0f || W < 0.0f) && (U > 0.0f || V > 0.0f || W > 0.0f)) return false;
	const float det = U + V + W;
	if(det == 0.0f) return false;
	const float Az = r.Sz * A[r.kz];
	const float Bz = r.Sz * B[r.kz];
	const float Cz = r.Sz * C[r.kz];
	const float T = U * Az + V * Bz + W * Cz;
	t = __fdiv_rn(T, det);
	bary = make2(__fdiv_rn(U, det), __fdiv_rn(V, det));
	return true;
}

MBD bool solve_square(float a, float b, float c, float& x0, float& x1) {
	if(a == 0.0f) {
		if(b == 0.0f) return false;
		x0 = x1 = __fdiv_rn(-c, b);
		return true;
	}
	const float disc = b * b - 4.0f * a * c;
	if(disc < 0.0f) return false;
	const float q = -0.5f * (b + sgn(b) * sqrt_(disc));
	if(q == 0.0f) { x0 = x1 = 0.0f; return true; }
	float r0 = __fdiv_rn(q, a), r1 = __fdiv_rn(c, q);
	if(r0 > r1) { const float t = r0; r0 = r1; r1 = t; }
	x0 = r0; x1 = r1;
	return true;
}

MBD float pabs(float x) { return x < 0.0f ? -x : x; }

MBD float computeU(float v, float A1, float A2, float B1, float B2, float C1, float C2, float D1, float D2) {
	const float a = v * A2 + B2;
	const float b = v * (A2 - A1) + B2 - B1;
	if(fabsf(b) >= fabsf(a)) return __fdiv_rn(v * (C1 - C2) + D1 - D2, b);
	return __fdiv_rn(-v * C2 - D2, a);
}

// intersection.cu:99-179
// Both roots: (resT1, uv1) is the nearer positive one, (resT2, uv2) the other
// (t <= 0: none), which the alpha test falls back to.
MBD bool quad_test(f3 p00, f3 p10, f3 p11, f3 p01, const FastRay& ray, float& resT1, f2& uv1, float& resT2, f2& uv2) {
	int d0 = 0, d1 = 1, d2 = 2;
	if(pabs(ray.d.x) < pabs(ray.d.y) || pabs(ray.d.x) < pabs(ray.d.z)) {
		if(pabs(ray.d.y) >= pabs(ray.d.z)) { d0 = 1; d1 = 0; d2 = 2; }
		else { d0 = 2; d1 = 1; d2 = 0; }
	}
	const f3 a = ((p11 - p10) - p01) + p00;
	const f3 b = p10 - p00;
	const f3 c = p01 - p00;
	const f3 d = p00 - ray.o;
	const float A1 = a[d1] * ray.d[d0] - a[d0] * ray.d[d1];
	const float A2 = a[d2] * ray.d[d0] - a[d0] * ray.d[d2];
	const float B1 = b[d1] * ray.d[d0] - b[d0] * ray.d[d1];
	const float B2 = b[d2] * ray.d[d0] - b[d0] * ray.d[d2];
	const float C1 = c[d1] * ray.d[d0] - c[d0] * ray.d[d1];
	const float C2 = c[d2] * ray.d[d0] - c[d0] * ray.d[d2];
	const float D1 = d[d1] * ray.d[d0] - d[d0] * ray.d[d1];
	const float D2 = d[d2] * ray.d[d0] - d[d0] * ray.d[d2];
	float v0 = 0.0f, v1 = 0.0f;
	if(solve_square(A2 * C1 - A1 * C2, ((A2 * D1 - A1 * D2) + B2 * C1) - B1 * C2, B2 * D1 - B1 * D2, v0, v1)) {
		float u0 = 0.0f, u1 = 0.0f;
		float t0 = -1.0f, t1 = -1.0f;
		if(v0 >= 0.0f && v0 <= 1.0f) {
			u0 = computeU(v0, A1, A2, B1, B2, C1, C2, D1, D2);
			if(u0 >= 0.0f && u0 <= 1.0f)
				t0 = ((((u0 * v0) * a[d0] + u0 * b[d0]) + v0 * c[d0]) + d[d0]) * ray.inv[d0];
		}
		if(v1 == v0) {
			uv1 = make2(u0, v0);
			resT1 = t0;
			resT2 = -1.0f;
		} else {
			if(v1 >= 0.0f && v1 <= 1.0f) {
				u1 = computeU(v1, A1, A2, B1, B2, C1, C2, D1, D2);
				if(u1 >= 0.0f && u1 <= 1.0f)
					t1 = ((((u1 * v1) * a[d0] + u1 * b[d0]) + v1 * c[d0]) + d[d0]) * ray.inv[d0];
			}
			if(t0 > 0.0f) {
				if(t1 > 0.0f && t1 < t0) { uv1 = make2(u1, v1); uv2 = make2(u0, v0); resT1 = t1; resT2 = t0; }
				else { uv1 = make2(u0, v0); uv2 = make2(u1, v1); resT1 = t0; resT2 = t1; }
			} else {
				uv1 = make2(u1, v1); uv2 = make2(u0, v0); resT1 = t1; resT2 = t0;
			}
		}
		return resT1 > 0.0f;
	}
	return false;
}

// Nearest positive root t; t2 is the far root when t is the near one (the
// alpha test's fallback), else -1.
MBD bool sphere_test(const FastRay& r, f3 c, float rad, float& t, float& t2) {
	const f3 oc = r.o - c;
	const float b = dot(oc, r.d);
	const float cc = dot(oc, oc) - rad * rad;
	// The discriminant from the ray's closest approach to the centre (Haines,
	// Guenther and Akenine-Moeller, Ray Tracing Gems ch. 7): b * b - cc cancels
	// for a small sphere far from the origin, and its error then exceeds the
	// shadow rays' 1e-4 origin offset (light paths to a sphere light 15 units
	// away were occluded by the light itself).
	const f3 perp = oc - r.d * b;
	const float disc = rad * rad - dot(perp, perp);
	if(disc < 0.0f) return false;
	const float q = -(b + sgn(b) * sqrt_(disc));
	float x0, x1;
	if(q == 0.0f) { x0 = x1 = 0.0f; }
	else { x0 = q; x1 = __fdiv_rn(cc, q); if(x0 > x1) { const float tt = x0; x0 = x1; x1 = tt; } }
	if(x0 > 0.0f) { t = x0; t2 = x1; return true; }
	if(x1 > 0.0f) { t = x1; t2 = -1.0f; return true; }
	return false;
}
MBD bool sphere_test(const FastRay& r, f3 c, float rad, float& t) {
	float t2;
	return sphere_test(r, c, rad, t, t2);
}

MBD f3 vert(const DLod& l, uint32_t i) { return ldg3(l.vertices + 3 * size_t(i)); }

// Nearest-texel lookup with wrap-around (the CPU textures' nearest sampling).
MBD f3 sample_texture(const DTexture& t, f2 uv) {
	const float fx = uv.x - floorf(uv.x), fy = uv.y - floorf(uv.y);
	int x = int(fx * float(t.width)), y = int(fy * float(t.height));
	if(x >= int(t.width)) x = int(t.width) - 1;
	if(y >= int(t.height)) y = int(t.height) - 1;
	const float4 v = __ldg(t.texels + size_t(y) * t.width + x);
	return make3(v.x, v.y, v.z);
}

MBD f2 uvat(const DLod& l, uint32_t i) { return ldg2(l.uvs + 2 * size_t(i)); }
MBD f2 bilerp2(f2 x00, f2 x10, f2 x01, f2 x11, float s, float t) {
	const f2 a = (1.0f - s) * x00 + s * x10;
	const f2 b = (1.0f - s) * x01 + s * x11;
	return (1.0f - t) * a + t * b;
}

// Alpha test of intersection.cu:205-216, 235-262 and 276-302: the alpha
// texture of primitive p's material, if it has one, cuts the surface where
// its first channel is below 0.5. `sp` is the hit's barycentric (triangles)
// or bilinear (quads) parametrisation; spheres take the object-space hit
// point (o + t d) instead.
// The scene's materials and textures when the alpha test applies, else
// materials == nullptr. (Passed instead of the scene itself: taking the
// address of a kernel-parameter scene would copy it to local memory.)
struct AlphaCtx {
	const DMaterial* materials;
	const DTexture* textures;
	MBD bool on() const { return materials != nullptr; }
};
MBD AlphaCtx alpha_ctx(const DScene& S, bool enable = true) {
	AlphaCtx a;
	a.materials = enable && S.hasAlpha ? S.materials : nullptr;
	a.textures = S.textures;
	return a;
}
MBD int alpha_texture(const AlphaCtx& A, const DLod& l, int p) {
	const uint32_t faces = l.numTriangles + l.numQuads;
	const uint16_t m = uint32_t(p) < faces ? __ldg(l.faceMaterials + p) : __ldg(l.sphereMaterials + (uint32_t(p) - faces));
	return A.materials[m].alphaTex;
}
MBD bool alpha_cut_at(const AlphaCtx& A, int tex, f2 uv) { return sample_texture(A.textures[tex], uv).x < 0.5f; }
MBD f2 tri_uv(const DLod& l, int p, f2 b) {
	const uint32_t o3 = uint32_t(p) * 3;
	const f2 t0 = uvat(l, __ldg(l.indices + o3)), t1 = uvat(l, __ldg(l.indices + o3 + 1)), t2 = uvat(l, __ldg(l.indices + o3 + 2));
	return (t0 * b.x + t1 * b.y) + t2 * ((1.0f - b.x) - b.y);
}
MBD f2 quad_uv(const DLod& l, int p, f2 b) {
	const uint32_t o4 = uint32_t(p - int(l.numTriangles)) * 4 + l.numTriangles * 3;
	const f2 t0 = uvat(l, __ldg(l.indices + o4)), t1 = uvat(l, __ldg(l.indices + o4 + 1));
	const f2 t2 = uvat(l, __ldg(l.indices + o4 + 2)), t3 = uvat(l, __ldg(l.indices + o4 + 3));
	return bilerp2(t0, t1, t3, t2, b.x, b.y);
}
MBD f2 sphere_uv(f3 center, const FastRay& r, float t) {
	const f3 n = normalize((r.o + t * r.d) - center);
	return make2(__fdiv_rn(mbmath::atan2(n.z, n.x), 2.0f * PI) + 0.5f, __fdiv_rn(mbmath::acos(-n.y), PI));
}
// Triangle hits: true when the alpha texture cuts the hit (kept out of line;
// only scenes with alpha textures call it).
static __device__ __noinline__ bool alpha_cuts_triangle(AlphaCtx A, const DLod& l, int p, f2 bary) {
	const int tex = alpha_texture(A, l, p);
	return tex >= 0 && alpha_cut_at(A, tex, tri_uv(l, p, bary));
}

// Primitive test for leaf slot `slot` holding primitive `p` (object space).
// With alpha.on(), the alpha textures of its materials apply.
MBD bool prim_test(const DLod& l, const FastRay& r, int slot, int p, float& t, f2& sp, AlphaCtx alpha = AlphaCtx{ nullptr, nullptr }) {
	if(p < int(l.numTriangles)) {
		const float4* s = l.triSoup + 3 * size_t(slot);
		const float4 a = __ldg(s), b = __ldg(s + 1), c = __ldg(s + 2);
		if(!(tri_test(r, f4to3(a), f4to3(b), f4to3(c), t, sp) && t > 0.0f)) return false;
		return !(alpha.on() && alpha_cuts_triangle(alpha, l, p, sp));
	}
	const int tex = alpha.on() ? alpha_texture(alpha, l, p) : -1;
	if(p < int(l.numTriangles + l.numQuads)) {
		const uint32_t o = uint32_t(p - int(l.numTriangles)) * 4 + l.numTriangles * 3;
		const uint32_t i0 = __ldg(l.indices + o), i1 = __ldg(l.indices + o + 1), i2 = __ldg(l.indices + o + 2), i3 = __ldg(l.indices + o + 3);
		float t1, t2;
		f2 uv, uv2 = make2(0.0f, 0.0f);
		if(!quad_test(vert(l, i0), vert(l, i1), vert(l, i2), vert(l, i3), r, t1, uv, t2, uv2)) return false;
		if(tex >= 0 && alpha_cut_at(alpha, tex, quad_uv(l, p, uv))) {
			// a cut-out first root: the other part of a non-planar quad
			if(!(t2 > 0.0f) || alpha_cut_at(alpha, tex, quad_uv(l, p, uv2))) return false;
			t1 = t2; uv = uv2;
		}
		t = t1; sp = uv;
		return true;
	}
	const float4 s = __ldg(l.spheres + (p - int(l.numTriangles + l.numQuads)));
	float t2;
	if(!sphere_test(r, f4to3(s), s.w, t, t2)) return false;
	if(tex >= 0 && alpha_cut_at(alpha, tex, sphere_uv(f4to3(s), r, t))) {
		// a cut-out near side: the far side seen through it
		if(!(t2 > 0.0f) || alpha_cut_at(alpha, tex, sphere_uv(f4to3(s), r, t2))) return false;
		t = t2;
	}
	sp = make2(0.0f, 0.0f);
	return true;
}

MBD void add_epsilon(f3& o, f3 dir, f3 n) {
	const f3 off = n * SCENE_SCALE_EPS;
	if(dot(n, dir) >= 0.0f) o = o + off; else o = o - off;
}

struct Mat34 { float4 r0, r1, r2; };
MBD Mat34 load_w2i(const DScene& S, uint32_t inst) {
	const float4* p = S.worldToInstance + 3 * size_t(inst);
	Mat34 m; m.r0 = __ldg(p); m.r1 = __ldg(p + 1); m.r2 = __ldg(p + 2);
	return m;
}
MBD f3 xform_point(const Mat34& M, f3 p) {
	return make3(M.r0.x * p.x + M.r0.y * p.y + M.r0.z * p.z + M.r0.w,
	             M.r1.x * p.x + M.r1.y * p.y + M.r1.z * p.z + M.r1.w,
	             M.r2.x * p.x + M.r2.y * p.y + M.r2.z * p.z + M.r2.w);
}
MBD f3 xform_dir(const Mat34& M, f3 d) {
	return make3(M.r0.x * d.x + M.r0.y * d.y + M.r0.z * d.z,
	             M.r1.x * d.x + M.r1.y * d.y + M.r1.z * d.z,
	             M.r2.x * d.x + M.r2.y * d.y + M.r2.z * d.z);
}
MBD f3 xform_transposed(const Mat34& M, f3 n) {
	return make3(M.r0.x * n.x + M.r1.x * n.y + M.r2.x * n.z,
	             M.r0.y * n.x + M.r1.y * n.y + M.r2.y * n.z,
	             M.r0.z * n.x + M.r1.z * n.y + M.r2.z * n.z);
}

struct HitRec {
	float t;
	int inst, prim;
	f2 sp;
	bool has;
};

MBD bool better(float tw, int inst, int prim, const HitRec& h) {
	if(tw < h.t) return true;
	if(h.has && tw == h.t) return inst < h.inst || (inst == h.inst && prim < h.prim);
	return false;
}

struct LocalCounters {
	unsigned int nodes = 0, prims = 0, instances = 0, rays = 0, shadow = 0, errors = 0;
};
// Counters of a traversal that keeps no statistics: the increments of node
// visits, primitive tests, instance entries and rays compile to nothing (and
// take no registers); abandoned rays are still counted.
struct NullCount {
	MBD NullCount& operator++() { return *this; }
	MBD operator unsigned() const { return 0u; }
};
struct NoCounters {
	NullCount nodes, prims, instances, rays, shadow;
	unsigned int errors = 0;
};

// Reads the child pair of internal node `node` as four 128-bit loads.
struct NodePair { float4 a, b, c, d; };
MBD NodePair load_pair(const BvhNode* nodes, int node) {
	const float4* p = reinterpret_cast<const float4*>(nodes + 2 * size_t(node));
	NodePair n; n.a = __ldg(p); n.b = __ldg(p + 1); n.c = __ldg(p + 2); n.d = __ldg(p + 3);
	return n;
}

// Visits the binary BVH; calls leaf(first, count) for every reached leaf.
// `tmaxFn()` returns the current culling distance. Returns false if the
// stack overflowed.
template < class TmaxFn, class LeafFn >
MBD bool traverse(const BvhNode* nodes, int nInt, const FastRay& ray, TmaxFn&& tmaxFn, LeafFn&& leaf,
                  int2* stack, int capacity, int maxSteps, LocalCounters& cnt) {
	int sp = 0;
	int node = 0;
	// A well-formed BVH visits each node at most once; the cap only guards
	// against a corrupted hierarchy (it records an error instead of spinning).
	for(int guard = 0;; ++guard) {
		if(guard >= maxSteps) { ++cnt.errors; return false; }
		++cnt.nodes;
		const NodePair np = load_pair(nodes, node);
		const float tmaxBox = tmaxFn();
		float c0, c1;
		const bool h0 = box_test(np.a.x, np.a.y, np.a.z, np.a.w, np.b.x, np.b.y, ray, tmaxBox, c0);
		const bool h1 = box_test(np.c.x, np.c.y, np.c.z, np.c.w, np.d.x, np.d.y, ray, tmaxBox, c1);
		const int li = __float_as_int(np.b.z), lc = __float_as_int(np.b.w);
		const int ri = __float_as_int(np.d.z), rc = __float_as_int(np.d.w);
		if(!h0) c0 = 1e38f;
		if(!h1) c1 = 1e38f;
		bool descended = false;
		if(h0 || h1) {
			const bool leftNear = c0 <= c1;
			if(h0 && h1) {
				if(sp >= capacity) { ++cnt.errors; return false; }
				stack[sp++] = leftNear ? make_int2(ri, rc) : make_int2(li, lc);
			}
			const int ni = leftNear ? li : ri;
			const int nc = leftNear ? lc : rc;
			if(ni < nInt) { node = ni; descended = true; }
			else if(!leaf(ni - nInt, nc)) return true;
		}
		if(descended) continue;
		bool found = false;
		while(sp > 0) {
			const int2 e = stack[--sp];
			if(e.x < nInt) { node = e.x; found = true; break; }
			if(!leaf(e.x - nInt, e.y)) return true;
		}
		if(!found) return true;
	}
}

struct InstRay { FastRay ray; float scale; };

MBD InstRay instance_ray(const Mat34& W, f3 o, f3 d) {
	const f3 dirO = xform_dir(W, d);
	const float scale = len(dirO);
	InstRay ir;
	ir.ray = make_ray(xform_point(W, o), dirO / scale);
	ir.scale = scale;
	return ir;
}

// Closest hit inside one instance.
MBD void blas_closest(const DScene& S, uint32_t inst, f3 o, f3 d, HitRec& best, LocalCounters& cnt, int2* stack) {
	++cnt.instances;
	const DLod& l = S.lods[__ldg(S.instanceLod + inst)];
	if(l.numPrims <= 0) return;
	const Mat34 W = load_w2i(S, inst);
	const InstRay ir = instance_ray(W, o, d);
	float cm;
	if(!box_test(l.aabbMin[0], l.aabbMin[1], l.aabbMin[2], l.aabbMax[0], l.aabbMax[1], l.aabbMax[2], ir.ray,
	             best.t * ir.scale * BOX_SLACK, cm))
		return;
	auto consider = [&](int slot) {
		const int p = __ldg(l.primIds + slot);
		float t; f2 sp;
		++cnt.prims;
		if(prim_test(l, ir.ray, slot, p, t, sp, alpha_ctx(S))) {
			const float tw = __fdiv_rn(t, ir.scale);
			if(better(tw, int(inst), p, best)) { best.t = tw; best.inst = int(inst); best.prim = p; best.sp = sp; best.has = true; }
		}
	};
	if(l.numPrims == 1) { consider(0); return; }
	traverse(l.nodes, l.numInternal, ir.ray,
		[&]() { return best.t * ir.scale * BOX_SLACK; },
		[&](int first, int count) { for(int k = 0; k < count; ++k) consider(first + k); return true; },
		stack, BLAS_STACK, S.maxSteps, cnt);
}

MBD bool blas_any(const DScene& S, uint32_t inst, f3 o, f3 d, float tmaxWorld, LocalCounters& cnt, int2* stack) {
	++cnt.instances;
	const DLod& l = S.lods[__ldg(S.instanceLod + inst)];
	if(l.numPrims <= 0) return false;
	const Mat34 W = load_w2i(S, inst);
	const InstRay ir = instance_ray(W, o, d);
	const float tmaxObj = tmaxWorld * ir.scale;
	const float tmaxBox = tmaxObj * BOX_SLACK;
	float cm;
	if(!box_test(l.aabbMin[0], l.aabbMin[1], l.aabbMin[2], l.aabbMax[0], l.aabbMax[1], l.aabbMax[2], ir.ray,
	             tmaxWorld * ir.scale * BOX_SLACK, cm))
		return false;
	bool hit = false;
	auto test = [&](int slot) {
		const int p = __ldg(l.primIds + slot);
		float t; f2 sp;
		++cnt.prims;
		return prim_test(l, ir.ray, slot, p, t, sp, alpha_ctx(S)) && t < tmaxObj;
	};
	if(l.numPrims == 1) return test(0);
	traverse(l.nodes, l.numInternal, ir.ray,
		[&]() { return tmaxBox; },
		[&](int first, int count) {
			for(int k = 0; k < count; ++k) if(test(first + k)) { hit = true; return false; }
			return true;
		},
		stack, BLAS_STACK, S.maxSteps, cnt);
	return hit;
}

struct Intersection {
	float distance;
	int inst, prim;
	f3 normal, tangentX;
	f2 uv;
	f2 sp;
};

MBD f3 bilerp3(f3 x00, f3 x10, f3 x01, f3 x11, float s, float t) {
	const f3 a = (1.0f - s) * x00 + s * x10;
	const f3 b = (1.0f - s) * x01 + s * x11;
	return (1.0f - t) * a + t * b;
}

MBD f3 nrmat(const DLod& l, uint32_t i) { return ldg3(l.normals + 3 * size_t(i)); }

// Closest hit of a world-space ray whose origin is already offset
// (intersection.cu:366-492): returns (t, instance, primitive, surface params).
MBD HitRec closest_hit(const DScene& S, f3 o, f3 dir, float tmax, LocalCounters& cnt, int2* bstack, int2* tstack) {
	++cnt.rays;
	HitRec best;
	best.t = tmax; best.inst = -1; best.prim = -1; best.sp = make2(0.0f, 0.0f); best.has = false;
	if(S.activeInstances == 1) {
		blas_closest(S, S.validInstance, o, dir, best, cnt, bstack);
	} else if(S.activeInstances > 1) {
		const FastRay wr = make_ray(o, dir);
		traverse(S.tlasNodes, S.tlasNumInternal, wr,
			[&]() { return best.t * BOX_SLACK; },
			[&](int first, int count) {
				for(int k = 0; k < count; ++k) blas_closest(S, uint32_t(__ldg(S.tlasPrimIds + first + k)), o, dir, best, cnt, bstack);
				return true;
			},
			tstack, TLAS_STACK, S.maxSteps, cnt);
	}
	return best;
}

// Hit attribute synthesis for a closest hit (intersection.cu:511-620).
MBD Intersection hit_attributes(const DScene& S, f3 origin, f3 dir, const HitRec& best) {
	Intersection res;
	res.distance = best.t;
	res.inst = best.has ? best.inst : -1;
	res.prim = best.has ? best.prim : -1;
	res.sp = best.sp;
	res.uv = make2(0.0f, 0.0f);
	res.normal = make3(0.0f, 0.0f, 0.0f);
	res.tangentX = make3(0.0f, 0.0f, 0.0f);
	if(!best.has) return res;
	const DLod& l = S.lods[__ldg(S.instanceLod + best.inst)];
	const Mat34 W = load_w2i(S, uint32_t(best.inst));
	f3 geoNormal, tangentX;
	f2 uv;
	const int p = best.prim;
	const int sphOff = int(l.numTriangles + l.numQuads);
	if(p >= sphOff) {
		const float4 s = __ldg(l.spheres + (p - sphOff));
		const f3 hitPoint = origin + best.t * dir;
		const f3 local = xform_point(W, hitPoint);
		geoNormal = normalize(local - f4to3(s));
		if(geoNormal.x == 0.0f && geoNormal.y == 0.0f) tangentX = make3(1.0f, 0.0f, 0.0f);
		else {
			const float ll = sqrt_(geoNormal.y * geoNormal.y + (-geoNormal.x) * (-geoNormal.x));
			tangentX = make3(__fdiv_rn(geoNormal.y, ll), __fdiv_rn(-geoNormal.x, ll), 0.0f);
		}
		uv.x = __fdiv_rn(mbmath::atan2(geoNormal.z, geoNormal.x), 2.0f * PI) + 0.5f;
		uv.y = __fdiv_rn(mbmath::acos(-geoNormal.y), PI);
		res.sp = uv;
	} else if(p < int(l.numTriangles)) {
		const uint32_t o3 = uint32_t(p) * 3;
		const uint32_t i0 = __ldg(l.indices + o3), i1 = __ldg(l.indices + o3 + 1), i2 = __ldg(l.indices + o3 + 2);
		const f3 v0 = vert(l, i0);
		const f3 dx0 = vert(l, i1) - v0;
		const f3 dx1 = vert(l, i2) - v0;
		const f2 t0 = uvat(l, i0), t1 = uvat(l, i1), t2 = uvat(l, i2);
		const f2 du0 = t1 - t0;
		const f2 du1 = t2 - t0;
		const float det = du0.x * du1.y - du0.y * du1.x;
		if(det >= 1e-5f || det <= -1e5f) tangentX = (dx0 * du1.y - dx1 * du0.y) / det;
		else tangentX = dx0;
		geoNormal = cross(dx0, dx1);
		uv = (t0 * best.sp.x + t1 * best.sp.y) + t2 * ((1.0f - best.sp.x) - best.sp.y);
	} else {
		const uint32_t o4 = uint32_t(p - int(l.numTriangles)) * 4 + l.numTriangles * 3;
		const uint32_t i0 = __ldg(l.indices + o4), i1 = __ldg(l.indices + o4 + 1), i2 = __ldg(l.indices + o4 + 2), i3 = __ldg(l.indices + o4 + 3);
		const f3 v0 = vert(l, i0), v1 = vert(l, i1), v2 = vert(l, i2), v3 = vert(l, i3);
		const f2 t0 = uvat(l, i0), t1 = uvat(l, i1), t2 = uvat(l, i2), t3 = uvat(l, i3);
		const float bu = best.sp.x, bv = best.sp.y;
		const f3 dxds = (1.0f - bu) * (v3 - v0) + bu * (v2 - v1);
		const f3 dxdt = (1.0f - bv) * (v1 - v0) + bv * (v2 - v3);
		const f2 duds = (1.0f - bu) * (t3 - t0) + bu * (t2 - t1);
		const f2 dudt = (1.0f - bv) * (t1 - t0) + bv * (t2 - t3);
		const float detD = duds.x * dudt.y - dudt.x * duds.y;
		if(detD >= 1e-9f || detD <= -1e-9f) {
			const float a = __fdiv_rn(dudt.y, detD), b = __fdiv_rn(-duds.y, detD);
			tangentX = make3(dxds.x * a + dxdt.x * b, dxds.y * a + dxdt.y * b, dxds.z * a + dxdt.z * b);
		} else tangentX = dxds;
		geoNormal = cross(dxdt, dxds);
		uv = bilerp2(t0, t1, t3, t2, bu, bv);
	}
	res.normal = normalize(xform_transposed(W, geoNormal));
	res.tangentX = normalize(xform_transposed(W, tangentX));
	res.uv = (p < sphOff) ? uv : res.sp;
	return res;
}

// Closest hit for a world-space ray (intersection.cu:366-621). `origin` is
// offset by add_epsilon in place, as the reference's ray is.
MBD Intersection first_intersection(const DScene& S, f3& origin, f3 dir, f3 geoN, float tmax,
                                    LocalCounters& cnt, int2* bstack, int2* tstack) {
	add_epsilon(origin, dir, geoN);
	const HitRec best = closest_hit(S, origin, dir, tmax, cnt, bstack, tstack);
	return hit_attributes(S, origin, dir, best);
}

// Occlusion test of a prepared shadow ray (origin already offset, unit
// direction, world-space length tmax).
MBD bool occluded(const DScene& S, f3 a, f3 dir, float tmax, LocalCounters& cnt, int2* bstack, int2* tstack) {
	++cnt.rays; ++cnt.shadow;
	if(S.activeInstances == 1) return blas_any(S, S.validInstance, a, dir, tmax, cnt, bstack);
	if(S.activeInstances <= 0) return false;
	const FastRay wr = make_ray(a, dir);
	bool occ = false;
	const float tmaxBox = tmax * BOX_SLACK;
	traverse(S.tlasNodes, S.tlasNumInternal, wr,
		[&]() { return tmaxBox; },
		[&](int first, int count) {
			for(int k = 0; k < count; ++k)
				if(blas_any(S, uint32_t(__ldg(S.tlasPrimIds + first + k)), a, dir, tmax, cnt, bstack)) { occ = true; return false; }
			return true;
		},
		tstack, TLAS_STACK, S.maxSteps, cnt);
	return occ;
}

// Shadow-ray set-up of intersection.cu:624-637: both end points are offset
// along their geometric normals; returns the origin, direction and length.
MBD void shadow_ray(f3 a, f3 b, f3 geoA, f3 geoB, f3 dirAB, f3& o, f3& dir, float& tmax) {
	add_epsilon(a, dirAB, geoA);
	add_epsilon(b, -dirAB, geoB);
	const f3 corrected = b - a;
	tmax = len(corrected);
	dir = corrected / tmax;
	o = a;
}

// Shadow ray between two surface points (intersection.cu:624-753).
MBD bool any_intersection(const DScene& S, f3 a, f3 b, f3 geoA, f3 geoB, f3 dirAB,
                          LocalCounters& cnt, int2* bstack, int2* tstack) {
	f3 o, dir; float tmax;
	shadow_ray(a, b, geoA, geoB, dirAB, o, dir, tmax);
	return occluded(S, o, dir, tmax, cnt, bstack, tstack);
}

struct TangentSpace { f3 shadingN, geoN, shadingTX, shadingTY; };

MBD TangentSpace tangent_space(const DScene& S, const Intersection& h) {
	const DLod& l = S.lods[__ldg(S.instanceLod + h.inst)];
	TangentSpace ts;
	if(uint32_t(h.prim) >= l.numTriangles + l.numQuads) {
		ts.shadingN = h.normal; ts.geoN = h.normal; ts.shadingTX = h.tangentX; ts.shadingTY = cross(h.normal, h.tangentX);
		return ts;
	}
	const Mat34 W = load_w2i(S, uint32_t(h.inst));
	f3 sn;
	if(uint32_t(h.prim) < l.numTriangles) {
		const uint32_t o = 3u * uint32_t(h.prim);
		sn = (h.sp.x * nrmat(l, __ldg(l.indices + o)) + h.sp.y * nrmat(l, __ldg(l.indices + o + 1)))
			+ (1.0f - (h.sp.x + h.sp.y)) * nrmat(l, __ldg(l.indices + o + 2));
	} else {
		const uint32_t o = 4u * uint32_t(h.prim - int(l.numTriangles)) + 3u * l.numTriangles;
		sn = bilerp3(nrmat(l, __ldg(l.indices + o)), nrmat(l, __ldg(l.indices + o + 1)),
		             nrmat(l, __ldg(l.indices + o + 3)), nrmat(l, __ldg(l.indices + o + 2)), h.sp.x, h.sp.y);
	}
	sn = normalize(xform_transposed(W, sn));
	const f3 tx = normalize(h.tangentX - sn * dot(h.tangentX, sn));
	ts.shadingN = sn; ts.geoN = h.normal; ts.shadingTX = tx; ts.shadingTY = cross(sn, tx);
	return ts;
}

} // namespace mb
