// CPU oracle for the Mufflon path-tracer hot path: TEST INFRASTRUCTURE ONLY.
//
// A single-translation-unit restatement of the reference renderer's CPU path:
//   LBVH build ........ src/core/scene/accel_structs/build_lbvh.cu:59-780,
//                       src/core/math/sfcurves.hpp:26-46,
//                       src/core/scene/accel_structs/accel_structs_commons.hpp:56-109
//   traversal ......... src/core/scene/accel_structs/intersection.cu:16-753,
//                       src/core/scene/accel_structs/tangent_space.hpp:10-66
//   path tracer ....... src/core/renderer/pt/pt_common.hpp:75-156,
//                       src/core/renderer/random_walk.hpp:38-113,
//                       src/core/renderer/path_util.hpp:130-665
//   camera ............ src/core/cameras/pinhole.hpp:53-81, camera.hpp:81-96
//   materials ......... src/core/scene/materials/{material_sampling,lambert,
//                       microfacet_base,microfacet_specular,emissive}.hpp
//   lights ............ src/core/scene/lights/{light_tree_sampling,light_sampling,
//                       lights}.hpp, light_tree.cpp:120-330, lights.cpp:10-91,
//                       background.cpp:125-135
//   rng / sampling .... src/core/math/rng.hpp:126-207, sampling.hpp:23-199
//   pixel loop ........ src/core/renderer/pt/cpu_pt.cpp:18-45
//   accumulation ...... src/core/renderer/targets/output_handler_variance.hpp:7-31
//   light tracer ...... src/core/renderer/lt/lt_common.hpp:19-77, cpu_lt.cpp:18-39,
//                       src/core/scene/lights/light_tree_sampling.hpp:81-188,
//                       light_sampling.hpp:80-306, src/core/cameras/pinhole.hpp:86-116
//   bidirectional PT .. src/core/renderer/bpt/cpu_bpt.cpp:18-247,
//                       src/core/renderer/path_util.hpp:41-794
//
// Pinned deviations from the reference (each needed because the reference is
// either order-dependent or relies on the missing "epsilon" library):
//   1. exact count-leading-zeros (the Linux host path uses log2f);
//   2. stable (key, index) sort of Morton codes;
//   3. SAH merge order fixed to "right child is the arriving thread", which is
//      what a sequential run of the reference CPU loop produces;
//   4. first hits are ordered by (world t, instance, primitive), so the result
//      does not depend on traversal order; box culling uses tmax * (1 + 2^-12)
//      so that it stays conservative;
//   5. robust slab test: t = (bound - origin) * invDir per axis (relative
//      error of a few ulp and the exact sign, where the reference's
//      fma(bound, invDir, -origin * invDir) has an error relative to the
//      origin's magnitude), entry clamped at 0, interval accepted up to
//      far * (1 + 2^-20). A box that contains a primitive's hit point is
//      never culled, so every bounding hierarchy over the same primitives
//      yields the same closest hit;
//   6. watertight triangle test (Woop, Benthin, Wald, JCGT 2013);
//   7. sphere test from the quadratic with a stable root, solveSquarePoly and
//      the vector helpers (surface, bilerp, sgn, box transform) written from
//      their mathematical definitions;
//   8. sin/cos/atan2/acos from mufflon_b200/csrc/common/fmath.hpp, the only
//      file shared with the product, so that host and device round alike;
//   9. no FP contraction (-ffp-contract=off), explicit fmaf where the GPU
//      uses an FMA;
//  10. sphere primitives are indexed from the sphere offset (the reference's
//      intersection.cu:270 and descriptors.hpp:198 index the sphere arrays
//      with the global primitive id, which only works for sphere-only LoDs);
//  11. the frame of an area light's emission lobe uses n x (the axis of n's
//      smallest component) for epsilon's `perpendicular`.
#include "oracle.h"
#include "../mufflon_b200/csrc/common/fmath.hpp"

#include <algorithm>
#include <array>
#include <chrono>
#include <atomic>
#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <map>
#include <memory>
#include <utility>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

using u16 = uint16_t;
using u32 = uint32_t;
using u64 = uint64_t;
using i32 = int32_t;

constexpr float PI = 3.14159265358979f;
constexpr float MAX_SCENE_SIZE = 1048576.0f;
constexpr float SCENE_SCALE_EPS = 1e-4f;
constexpr float INF_PDF = 4294967296.0f;
constexpr float BOX_SLACK = 1.0f + 1.0f / 4096.0f;
constexpr float BOX_FAR_SLACK = 1.0f + 1.0f / 1048576.0f;
constexpr float DISTANCESQ_EPSILON = 1e-10f;
constexpr float SHADING_NORMAL_EPS = 1e-3f;
constexpr i32 TREE_HEAD = 0x10000000;

// ---------------------------------------------------------------- vectors
struct V2 { float x, y; };
struct V3 {
	float x, y, z;
	float operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
};
inline V3 operator+(V3 a, V3 b) { return { a.x + b.x, a.y + b.y, a.z + b.z }; }
inline V3 operator-(V3 a, V3 b) { return { a.x - b.x, a.y - b.y, a.z - b.z }; }
inline V3 operator-(V3 a) { return { -a.x, -a.y, -a.z }; }
inline V3 operator*(V3 a, V3 b) { return { a.x * b.x, a.y * b.y, a.z * b.z }; }
inline V3 operator*(V3 a, float s) { return { a.x * s, a.y * s, a.z * s }; }
inline V3 operator*(float s, V3 a) { return { s * a.x, s * a.y, s * a.z }; }
inline V3 operator/(V3 a, float s) { return { a.x / s, a.y / s, a.z / s }; }
inline V3 operator/(V3 a, V3 b) { return { a.x / b.x, a.y / b.y, a.z / b.z }; }
inline V2 operator+(V2 a, V2 b) { return { a.x + b.x, a.y + b.y }; }
inline V2 operator-(V2 a, V2 b) { return { a.x - b.x, a.y - b.y }; }
inline V2 operator*(V2 a, float s) { return { a.x * s, a.y * s }; }
inline V2 operator*(float s, V2 a) { return { s * a.x, s * a.y }; }
inline float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline V3 cross(V3 a, V3 b) {
	return { a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x };
}
inline float lensq(V3 a) { return dot(a, a); }
inline float len(V3 a) { return mbmath::sqrt(lensq(a)); }
inline V3 normalize(V3 a) { return a / len(a); }
inline float fmin_(float a, float b) { return std::fmin(a, b); }
inline float fmax_(float a, float b) { return std::fmax(a, b); }
// Box merges use an explicit select so that signed zeros resolve the same
// way on host and device: min(a, b) = b < a ? b : a.
inline float bmin(float a, float b) { return b < a ? b : a; }
inline float bmax(float a, float b) { return a < b ? b : a; }
inline V3 vmin(V3 a, V3 b) { return { bmin(a.x, b.x), bmin(a.y, b.y), bmin(a.z, b.z) }; }
inline V3 vmax(V3 a, V3 b) { return { bmax(a.x, b.x), bmax(a.y, b.y), bmax(a.z, b.z) }; }
inline float maxc(V3 a) { return fmax_(fmax_(a.x, a.y), a.z); }
inline float sgn(float x) { return x < 0.0f ? -1.0f : 1.0f; }
inline float sdiv(float x, float d) { return x / (d + 1e-20f * sgn(d)); }
inline V3 sdiv(V3 x, V3 d) { return { sdiv(x.x, d.x), sdiv(x.y, d.y), sdiv(x.z, d.z) }; }
inline bool any_pos(V3 a) { return a.x > 0.0f || a.y > 0.0f || a.z > 0.0f; }
inline bool nonzero(V3 a) { return a.x != 0.0f || a.y != 0.0f || a.z != 0.0f; }

struct Box { V3 mn, mx; };
inline Box empty_box() { return { { FLT_MAX, FLT_MAX, FLT_MAX }, { -FLT_MAX, -FLT_MAX, -FLT_MAX } }; }
inline Box merge(Box a, Box b) { return { vmin(a.mn, b.mn), vmax(a.mx, b.mx) }; }
inline float surface(Box b) {
	V3 d = b.mx - b.mn;
	return 2.0f * (d.x * d.y + d.x * d.z + d.y * d.z);
}
inline V3 center(Box b) { return (b.mn + b.mx) * 0.5f; }

struct Mat34 { float m[12]; };
inline V3 xform_point(const Mat34& M, V3 p) {
	const float* m = M.m;
	return { m[0] * p.x + m[1] * p.y + m[2] * p.z + m[3],
	         m[4] * p.x + m[5] * p.y + m[6] * p.z + m[7],
	         m[8] * p.x + m[9] * p.y + m[10] * p.z + m[11] };
}
inline V3 xform_dir(const Mat34& M, V3 d) {
	const float* m = M.m;
	return { m[0] * d.x + m[1] * d.y + m[2] * d.z,
	         m[4] * d.x + m[5] * d.y + m[6] * d.z,
	         m[8] * d.x + m[9] * d.y + m[10] * d.z };
}
// transpose(Mat3x3(M)) * n
inline V3 xform_transposed(const Mat34& M, V3 n) {
	const float* m = M.m;
	return { m[0] * n.x + m[4] * n.y + m[8] * n.z,
	         m[1] * n.x + m[5] * n.y + m[9] * n.z,
	         m[2] * n.x + m[6] * n.y + m[10] * n.z };
}
// descriptors.hpp:108-129
Mat34 instance_to_world(const Mat34& W) {
	const float* r = W.m;
	const float r00 = r[0], r01 = r[1], r02 = r[2], r10 = r[4], r11 = r[5], r12 = r[6],
	            r20 = r[8], r21 = r[9], r22 = r[10];
	const float m00 = r11 * r22 - r21 * r12;
	const float m01 = r21 * r02 - r01 * r22;
	const float m02 = r01 * r12 - r11 * r02;
	const float m10 = r20 * r12 - r10 * r22;
	const float m11 = r00 * r22 - r20 * r02;
	const float m12 = r10 * r02 - r00 * r12;
	const float m20 = r10 * r21 - r20 * r11;
	const float m21 = r20 * r01 - r00 * r21;
	const float m22 = r00 * r11 - r10 * r01;
	const float det = r00 * m00 + r01 * m10 + r02 * m20;
	const float id = 1.0f / det;
	const float i00 = id * m00, i01 = id * m01, i02 = id * m02, i10 = id * m10, i11 = id * m11,
	            i12 = id * m12, i20 = id * m20, i21 = id * m21, i22 = id * m22;
	const float tx = r[3], ty = r[7], tz = r[11];
	Mat34 o;
	o.m[0] = i00; o.m[1] = i01; o.m[2] = i02; o.m[3] = -(i00 * tx + i01 * ty + i02 * tz);
	o.m[4] = i10; o.m[5] = i11; o.m[6] = i12; o.m[7] = -(i10 * tx + i11 * ty + i12 * tz);
	o.m[8] = i20; o.m[9] = i21; o.m[10] = i22; o.m[11] = -(i20 * tx + i21 * ty + i22 * tz);
	return o;
}
Box xform_box(const Mat34& M, Box b) {
	Box o = empty_box();
	for(int c = 0; c < 8; ++c) {
		V3 p = { (c & 1) ? b.mx.x : b.mn.x, (c & 2) ? b.mx.y : b.mn.y, (c & 4) ? b.mx.z : b.mn.z };
		V3 q = xform_point(M, p);
		o.mn = vmin(o.mn, q);
		o.mx = vmax(o.mx, q);
	}
	return o;
}

// ---------------------------------------------------------------- rng
// rng.hpp:126-131
inline u64 scramble_seed(u32 x) {
	u64 z = u64(x) + 0x9e3779b97f4a7c15ull;
	z = (z ^ (z >> 30u)) * 0xbf58476d1ce4e5b9ull;
	z = (z ^ (z >> 27u)) * 0x94d049bb133111ebull;
	return z ^ (z >> 31u);
}
// rng.hpp:184-207
struct Pcg64 {
	u64 state;
	u64 next() {
		u64 x = state;
		const u64 count = state >> 59ull;
		state = state * 6364136223846793005ull + 1442695040888963407ull;
		x ^= x >> (5 + count);
		x *= 12605985483714917081ull;
		return x ^ (x >> 43);
	}
	static Pcg64 seeded(u32 seed) {
		Pcg64 r;
		r.state = scramble_seed(seed);
		r.next();
		r.state += seed;
		r.next();
		return r;
	}
};
// sampling.hpp:23-29
inline float sample_uniform(u32 u) { return float(u) / 4294967810.0f; }
// sampling.hpp:39-46
inline u64 percentage_of(u64 num, float p) {
	u64 pfix = u64(p * 2147483648.0f);
	return ((pfix * (num & 0x7fffffff)) >> 31) + (pfix * (num >> 31));
}

// rng.hpp:119-140: GoldenRatio2D::next, the state advanced by the golden
// ratio in 64-bit fixed point and turned from a Hilbert index into two 32-bit
// coordinates (gray code, then the Morton bits separated)
inline u64 golden_ratio2d_next(u64& state) {
	u64 s = state;
	state += 11400714819323198485ull;
	s = s ^ (s >> 1);
	s = ((s >> 1) & 0x2222222222222222ull) | ((s << 1) & 0x4444444444444444ull) | (s & 0x9999999999999999ull);
	s = ((s >> 2) & 0x0c0c0c0c0c0c0c0cull) | ((s << 2) & 0x3030303030303030ull) | (s & 0xc3c3c3c3c3c3c3c3ull);
	s = ((s >> 4) & 0x00f000f000f000f0ull) | ((s << 4) & 0x0f000f000f000f00ull) | (s & 0xf00ff00ff00ff00full);
	s = ((s >> 8) & 0x0000ff000000ff00ull) | ((s << 8) & 0x00ff000000ff0000ull) | (s & 0xff0000ffff0000ffull);
	s = ((s >> 16) & 0x00000000ffff0000ull) | ((s << 16) & 0x0000ffff00000000ull) | (s & 0xffff00000000ffffull);
	return s;
}

// ---------------------------------------------------------------- morton
// sfcurves.hpp:12-19: 16 bits spread 3 ways
inline u64 part_by_two16(u32 x) {
	u64 r = x & 0xFFFF;
	r = (r | (r << 16)) & 0x0000ff0000ffull;
	r = (r | (r << 8)) & 0x00f00f00f00full;
	r = (r | (r << 4)) & 0x0c30c30c30c3ull;
	r = (r | (r << 2)) & 0x249249249249ull;
	return r;
}
// sfcurves.hpp:58-77: Morton code of three 16-bit values, and its Hilbert
// index (the gray-code inverse of the Morton code)
inline u64 morton_code16(u32 a, u32 b, u32 c) { return part_by_two16(a) | (part_by_two16(b) << 1u) | (part_by_two16(c) << 2u); }
inline u64 hilbert_code16(u32 a, u32 b, u32 c) {
	u64 num = morton_code16(a, b, c);
	num = num ^ (num >> 32); num = num ^ (num >> 16); num = num ^ (num >> 8);
	num = num ^ (num >> 4); num = num ^ (num >> 2); num = num ^ (num >> 1);
	return num;
}
// sfcurves.hpp:35-44
inline u64 part_by_two21(u32 x) {
	u64 r = x;
	r = (r | (r << 32)) & 0x001f00000000ffffull;
	r = (r | (r << 16)) & 0x001f0000ff0000ffull;
	r = (r | (r << 8)) & 0x100f00f00f00f00full;
	r = (r | (r << 4)) & 0x10c30c30c30c30c3ull;
	r = (r | (r << 2)) & 0x1249249249249249ull;
	return r;
}
inline int clz64(u64 v) { return v == 0 ? 64 : __builtin_clzll(v); }
inline int clz32(u32 v) { return v == 0 ? 32 : __builtin_clz(v); }

// build_lbvh.cu:71-85
inline u64 morton63(V3 p, Box bb) {
	V3 span = bb.mx - bb.mn;
	V3 n = sdiv(p - bb.mn, span);
	auto disc = [](float v) {
		float x = v * 2097152.0f;
		x = std::fmin(std::fmax(x, 0.0f), 2097151.0f);
		return u32(x);
	};
	return part_by_two21(disc(n.x)) * 4 + part_by_two21(disc(n.y)) * 2 + part_by_two21(disc(n.z));
}

// sfcurves.hpp:37-46: spreads 10 bits to every third bit (multiply-and-mask form)
inline u32 part_by_two10(u32 x) {
	u32 r = x;
	r = (r * 0x00010001u) & 0xFF0000FFu;
	r = (r * 0x00000101u) & 0x0F00F00Fu;
	r = (r * 0x00000011u) & 0xC30C30C3u;
	r = (r * 0x00000005u) & 0x49249249u;
	return r;
}
// build_lbvh.cu:59-69, 81-86: the 30-bit code of a point (the reference builds
// every hierarchy with the 63-bit code; this one is kept as its alternative)
inline u32 morton30(V3 p, Box bb) {
	V3 span = bb.mx - bb.mn;
	V3 n = sdiv(p - bb.mn, span);
	auto disc = [](float v) {
		float x = v * 1024.0f;
		x = std::fmin(std::fmax(x, 0.0f), 1023.0f);
		return u32(x);
	};
	return part_by_two10(disc(n.x)) * 4u + part_by_two10(disc(n.y)) * 2u + part_by_two10(disc(n.z));
}

// ---------------------------------------------------------------- scene
struct Lod {
	u32 nV = 0, nT = 0, nQ = 0, nS = 0;
	std::vector<V3> verts, normals;
	std::vector<V2> uvs;
	std::vector<u32> idx;
	std::vector<u16> faceMat;
	std::vector<float> spheres; // 4 per sphere
	std::vector<u16> sphereMat;
	i32 numPrims = 0;
	Box aabb = empty_box();
};

struct BvhNode { V3 mn, mx; i32 index, primCount; };

struct Bvh {
	i32 numPrims = 0;
	i32 numInternal = 0; // after collapse
	std::vector<u64> mortonSorted;
	std::vector<i32> parents;
	std::vector<BvhNode> nodes; // 2 per internal node
	std::vector<i32> primIds;
};

struct Material {
	i32 type;
	V3 albedo;
	V2 roughness;
	i32 shadowing, ndf;
	V3 radiance, scale;
	i32 albedoTex;
	i32 alphaTex = -1; // cut-out texture (intersection.cu:205-216), -1: opaque
};

struct Texture { u32 w, h; std::vector<float> texels; };

enum LightType : u16 { LT_POINT = 0, LT_SPOT = 1, LT_TRI = 2, LT_QUAD = 3, LT_SPHERE = 4, LT_DIR = 5, LT_ENV = 6 };
constexpr u16 INTERNAL_NODE = 0xFFFF;

struct PosLight {
	u16 type;
	// point
	V3 position, intensity;
	// area quad (light.hpp:107-124 precomputed vectors)
	V3 posV[4];
	V2 uvV[4];
	u16 material;
	i32 primInst = -1, primId = -1;
	float radius = 0.0f; // sphere (centre in position)
};

struct LightNodeRef { float flux; i32 index; u16 type; }; // index: light index or node index
struct LightNode { LightNodeRef left, right; V3 center; };

struct LightTree {
	std::vector<PosLight> lights;
	std::vector<LightNode> nodes;
	float rootFlux = 0.0f;
	u16 rootType = INTERNAL_NODE;
	i32 rootIndex = 0;
	V3 bgFlux = { 0, 0, 0 };
	bool hasBackground = false;
	V3 bgColor = { 0, 0, 0 }, bgScale = { 0, 0, 0 };
	std::map<std::pair<i32, i32>, u32> primToNodePath;
	float dirFlux = 0.0f;
};

struct Camera {
	V3 position, viewDir, up;
	float tanVFov, nearP, farP;
	u16 resX, resY;
};

struct Counters {
	u64 rays = 0, shadowRays = 0, nodeVisits = 0, instanceVisits = 0, tri = 0, quad = 0, sphere = 0;
	void add(const Counters& o) {
		rays += o.rays; shadowRays += o.shadowRays; nodeVisits += o.nodeVisits;
		instanceVisits += o.instanceVisits; tri += o.tri; quad += o.quad; sphere += o.sphere;
	}
};

struct Scene {
	bool hasAlpha = false; // some material has an alpha texture
	std::vector<Lod> lods;
	std::vector<Bvh> lodBvh;
	std::vector<Mat34> w2i;
	std::vector<u32> instLod;
	i32 activeInstances = 0;
	u32 validInstance = 0;
	Bvh tlas;
	std::vector<Material> materials;
	std::vector<Texture> textures;
	LightTree lightTree;
	double lightBuildMs = 0.0;   // host time of the light list and tree build
	Camera cam;
	Box aabb = empty_box();
	u32 width = 0, height = 0;
};

// -------------------------------------------------------- primitive access
inline V3 sphere_center(const Lod& l, i32 s) { return { l.spheres[4 * s], l.spheres[4 * s + 1], l.spheres[4 * s + 2] }; }
inline float sphere_radius(const Lod& l, i32 s) { return l.spheres[4 * s + 3]; }

// accel_structs_commons.hpp:56-80
V3 lod_centroid(const Lod& l, i32 p) {
	const i32 sphOff = i32(l.nT + l.nQ);
	if(p >= sphOff) return sphere_center(l, p - sphOff);
	if(p >= i32(l.nT)) {
		const u32 q = u32(p - i32(l.nT)) * 4 + l.nT * 3;
		return (((l.verts[l.idx[q]] + l.verts[l.idx[q + 1]]) + l.verts[l.idx[q + 2]]) + l.verts[l.idx[q + 3]]) / 4.0f;
	}
	const u32 t = u32(p) * 3;
	return ((l.verts[l.idx[t]] + l.verts[l.idx[t + 1]]) + l.verts[l.idx[t + 2]]) / 3.0f;
}
// accel_structs_commons.hpp:85-103
Box lod_box(const Lod& l, i32 p) {
	const i32 sphOff = i32(l.nT + l.nQ);
	if(p >= sphOff) {
		V3 c = sphere_center(l, p - sphOff);
		float r = sphere_radius(l, p - sphOff);
		return { c - V3{ r, r, r }, c + V3{ r, r, r } };
	}
	Box b = empty_box();
	if(p >= i32(l.nT)) {
		const u32 q = u32(p - i32(l.nT)) * 4 + l.nT * 3;
		for(int k = 0; k < 4; ++k) { b.mn = vmin(b.mn, l.verts[l.idx[q + k]]); b.mx = vmax(b.mx, l.verts[l.idx[q + k]]); }
		return b;
	}
	const u32 t = u32(p) * 3;
	for(int k = 0; k < 3; ++k) { b.mn = vmin(b.mn, l.verts[l.idx[t + k]]); b.mx = vmax(b.mx, l.verts[l.idx[t + k]]); }
	return b;
}

// ---------------------------------------------------------------- LBVH
// Build-time descriptor abstraction over LoDs (3 primitive types, clamped
// 10-bit counts) and scenes (instances).
struct BuildDesc {
	bool isScene;
	const Scene* scene;
	const Lod* lod;
	i32 numPrims;
	Box bb;
	i32 mortonBits = 63;        // 63 (u64 keys, the reference's choice) or 30 (u32 keys)
	std::vector<Box> instBoxes; // scene only
	std::vector<V3> instCentroids;
};

struct Counts { i32 c[3]; };
inline Counts prim_count(const BuildDesc& d, i32 p) {
	if(d.isScene) return { { 1, 0, 0 } };
	const Lod& l = *d.lod;
	if(p >= i32(l.nT + l.nQ)) return { { 0, 0, 1 } };
	if(p >= i32(l.nT)) return { { 0, 1, 0 } };
	return { { 1, 0, 0 } };
}
inline Counts add(Counts a, Counts b) { return { { a.c[0] + b.c[0], a.c[1] + b.c[1], a.c[2] + b.c[2] } }; }
inline Counts clamp_counts(const BuildDesc& d, Counts a) {
	if(d.isScene) return a;
	return { { std::min(a.c[0], 0x3FF), std::min(a.c[1], 0x3FF), std::min(a.c[2], 0x3FF) } };
}
// build_lbvh.cu:319-324 with the constants of build_lbvh.cu:35-48
inline float get_cost(const BuildDesc& d, Counts c) {
	if(d.isScene) return 1.0f + float(c.c[0]) * 8.5f;
	return 2.0f + ((float(c.c[0]) * 1.2f + float(c.c[1]) * 4.0f) + float(c.c[2]) * 1.0f);
}
inline bool count_limit(const BuildDesc& d, Counts c) {
	if(d.isScene) return c.c[0] >= 1023;
	return c.c[0] >= 1023 || c.c[1] >= 1023 || c.c[2] >= 1023;
}

// build_lbvh.cu:164-178, for u64 and u32 keys (sizeof(Key) * 8 + clz of the
// index difference for equal keys)
inline int clz_key(u64 v) { return clz64(v); }
inline int clz_key(u32 v) { return clz32(v); }
template < class Key >
inline i32 lcp(const std::vector<Key>& k, i32 n, i32 i1, i32 i2, Key key1) {
	if(i2 < 0 || i2 >= n) return -1;
	const Key key2 = k[i2];
	if(key1 == key2) return i32(sizeof(Key) * 8) + clz32(u32(i1 ^ i2));
	return clz_key(Key(key1 ^ key2));
}

// build_lbvh.cu:180-245
template < class Key >
void karras_node(const std::vector<Key>& keys, i32 n, std::vector<i32>& parents, i32 idx) {
	const Key key1 = keys[idx];
	const i32 lcp1 = lcp(keys, n, idx, idx + 1, key1);
	const i32 lcp2 = lcp(keys, n, idx, idx - 1, key1);
	const i32 direction = (lcp1 - lcp2) < 0 ? -1 : 1;
	const i32 minLcp = lcp(keys, n, idx, idx - direction, key1);
	i32 lMax = 2;
	while(lcp(keys, n, idx, idx + lMax * direction, key1) > minLcp) lMax *= 2;
	i32 l = 0;
	for(i32 t = lMax; t > 1;) {
		t = t / 2;
		if(lcp(keys, n, idx, idx + (l + t) * direction, key1) > minLcp) l += t;
	}
	const i32 j = idx + l * direction;
	const i32 nodeLcp = lcp(keys, n, idx, j, key1);
	i32 s = 0;
	const i32 maxDivisor = 1 << (32 - clz32(u32(l)));
	for(i32 divisor = 2; divisor <= maxDivisor; divisor *= 2) {
		const i32 t = (l + divisor - 1) / divisor;
		if(lcp(keys, n, idx, idx + (s + t) * direction, key1) > nodeLcp) s += t;
	}
	const i32 split = idx + s * direction + std::min(direction, 0);
	const i32 leftIndex = (std::min(idx, j) == split) ? split + n - 1 : split;
	const i32 rightIndex = (std::max(idx, j) == split + 1) ? split + n : split + 1;
	parents[leftIndex] = ~idx;
	parents[rightIndex] = idx;
	if(idx == 0) parents[0] = TREE_HEAD;
}

void build_lbvh(const BuildDesc& d, i32 numPrimitives, i32 actualPrimCount, Bvh& out) {
	out = Bvh{};
	out.numPrims = numPrimitives;
	if(numPrimitives <= 0) return;
	// build_lbvh.cu:595-602: a single primitive needs no hierarchy
	if(actualPrimCount == 1) {
		out.primIds = { 0 };
		out.numInternal = 0;
		// The mask (if any) still determines which instance is the valid one;
		// the traversal goes through the single-instance shortcut instead.
		return;
	}
	const i32 used = actualPrimCount != 0 ? actualPrimCount : numPrimitives;
	const i32 numInternal = used - 1;
	const i32 numNodes = numInternal + used;

	// Morton codes (build_lbvh.cu:96-108)
	out.mortonSorted.resize(numPrimitives);
	out.primIds.resize(numPrimitives);
	out.parents.assign(numNodes, 0);
	if(d.mortonBits == 30) {
		// 30-bit codes in u32 keys: sorted, then the Karras hierarchy on u32 keys
		std::vector<std::pair<u32, i32>> kv(numPrimitives);
		for(i32 i = 0; i < numPrimitives; ++i) {
			u32 code;
			if(d.isScene) code = d.scene->instLod[i] == 0xFFFFFFFFu ? ~0u : morton30(d.instCentroids[i], d.bb);
			else code = morton30(lod_centroid(*d.lod, i), d.bb);
			kv[i] = { code, i };
		}
		std::stable_sort(kv.begin(), kv.end(), [](const auto& a, const auto& b) { return a.first < b.first; });
		std::vector<u32> keys(numPrimitives);
		for(i32 i = 0; i < numPrimitives; ++i) { keys[i] = kv[i].first; out.mortonSorted[i] = kv[i].first; out.primIds[i] = kv[i].second; }
		for(i32 i = 0; i < numInternal; ++i) karras_node(keys, used, out.parents, i);
	} else {
		std::vector<std::pair<u64, i32>> kv(numPrimitives);
		for(i32 i = 0; i < numPrimitives; ++i) {
			u64 code;
			if(d.isScene) {
				if(d.scene->instLod[i] == 0xFFFFFFFFu) code = ~0ull;
				else code = morton63(d.instCentroids[i], d.bb);
			} else {
				code = morton63(lod_centroid(*d.lod, i), d.bb);
			}
			kv[i] = { code, i };
		}
		std::stable_sort(kv.begin(), kv.end(), [](const auto& a, const auto& b) { return a.first < b.first; });
		for(i32 i = 0; i < numPrimitives; ++i) { out.mortonSorted[i] = kv[i].first; out.primIds[i] = kv[i].second; }
		// Karras hierarchy
		for(i32 i = 0; i < numInternal; ++i) karras_node(out.mortonSorted, used, out.parents, i);
	}

	// Children from the parent links (root: node 0)
	std::vector<i32> leftChild(numInternal, -1), rightChild(numInternal, -1);
	for(i32 nd = 1; nd < numNodes; ++nd) {
		i32 p = out.parents[nd];
		if(p < 0) leftChild[~p] = nd; else rightChild[p] = nd;
	}

	// Bottom-up boxes, SAH cost and counts (build_lbvh.cu:326-411), sequential
	// order: the right child's thread is the arriving one.
	std::vector<Box> box(numNodes);
	std::vector<Counts> cnt(numNodes);
	std::vector<float> cost(numNodes);
	for(i32 i = 0; i < used; ++i) {
		const i32 prim = out.primIds[i];
		const i32 leaf = numInternal + i;
		box[leaf] = d.isScene ? d.instBoxes[prim] : lod_box(*d.lod, prim);
		cnt[leaf] = prim_count(d, prim);
		cost[leaf] = get_cost(d, cnt[leaf]);
	}
	// post-order over internal nodes
	{
		std::vector<std::pair<i32, bool>> st;
		st.push_back({ 0, false });
		while(!st.empty()) {
			auto [nd, expanded] = st.back();
			st.pop_back();
			if(nd >= numInternal) continue;
			if(!expanded) {
				st.push_back({ nd, true });
				st.push_back({ rightChild[nd], false });
				st.push_back({ leftChild[nd], false });
				continue;
			}
			const i32 L = leftChild[nd], R = rightChild[nd];
			const float currentSA = surface(box[R]);
			Box b = { vmin(box[R].mn, box[L].mn), vmax(box[R].mx, box[L].mx) };
			const float newSA = surface(b);
			const float otherSA = surface(box[L]);
			const float nodeCost = d.isScene ? 1.0f : 2.0f;
			cost[nd] = (nodeCost + (currentSA / newSA) * get_cost(d, clamp_counts(d, cnt[R])))
				+ (otherSA / newSA) * get_cost(d, clamp_counts(d, cnt[L]));
			cnt[nd] = add(cnt[R], cnt[L]);
			box[nd] = b;
		}
	}
	// Marks (build_lbvh.cu:417-463)
	std::vector<i32> marks(numInternal, 1);
	for(i32 i = 0; i < used; ++i) {
		const i32 leaf = numInternal + i;
		i32 collapseNode = -1;
		i32 cur = out.parents[leaf];
		if(cur < 0) cur = ~cur;
		while(cur != 0) {
			const Counts c = clamp_counts(d, cnt[cur]);
			if(count_limit(d, c)) break;
			if(get_cost(d, c) < cost[cur]) collapseNode = cur;
			cur = out.parents[cur];
			if(cur < 0) cur = ~cur;
		}
		if(collapseNode != -1) {
			cur = out.parents[leaf];
			if(cur < 0) cur = ~cur;
			while(cur != collapseNode) {
				marks[cur] = 0;
				cur = out.parents[cur];
				if(cur < 0) cur = ~cur;
			}
			marks[cur] = 0;
		}
	}
	// Inclusive scan
	std::vector<i32> offsets(numInternal);
	i32 acc = 0;
	for(i32 i = 0; i < numInternal; ++i) { acc += marks[i]; offsets[i] = acc; }
	const i32 after = offsets[numInternal - 1];
	out.numInternal = after;
	out.nodes.assign(size_t(after) * 2, BvhNode{ { 0, 0, 0 }, { 0, 0, 0 }, 0, 0 });
	auto is_collapsed = [&](i32 nd) {
		if(nd > 0 && nd < numInternal) return (offsets[nd] - offsets[nd - 1]) == 0;
		return false;
	};
	// build_lbvh.cu:511-566
	for(i32 nd = 1; nd < numNodes; ++nd) {
		if(is_collapsed(nd)) continue;
		i32 parent = out.parents[nd];
		i32 offset;
		if(parent < 0) { offset = 0; parent = ~parent; } else offset = 1;
		i32 finalNode = nd;
		bool skip = false;
		if(finalNode >= numInternal) {
			while(is_collapsed(parent)) {
				if(offset == 1) { skip = true; break; }
				finalNode = parent;
				parent = out.parents[parent];
				if(parent < 0) { offset = 0; parent = ~parent; } else offset = 1;
			}
		}
		if(skip) continue;
		const Counts c = clamp_counts(d, cnt[finalNode]);
		const i32 primCount = d.isScene ? c.c[0] : (c.c[0] + c.c[1] + c.c[2]);
		const i32 outIdx = (offsets[parent] - 1) * 2;
		const i32 outNode = (nd >= numInternal) ? nd - numInternal + after : offsets[nd] - 1;
		const Box b = box[finalNode];
		const V3 ctr = (b.mn + b.mx) * 0.5f;
		BvhNode node;
		node.mn = (b.mn - ctr) * 1.0001f + ctr;
		node.mx = (b.mx - ctr) * 1.0001f + ctr;
		node.index = outNode;
		node.primCount = primCount;
		out.nodes[outIdx + offset] = node;
	}
}

// ---------------------------------------------------------------- rays
struct FastRay {
	V3 o, d, inv;
	// watertight test precomputation
	int kx, ky, kz;
	float Sx, Sy, Sz;
};
FastRay make_ray(V3 o, V3 d) {
	FastRay r;
	r.o = o; r.d = d;
	r.inv = { 1.0f / d.x, 1.0f / d.y, 1.0f / d.z };
	const float ax = std::fabs(d.x), ay = std::fabs(d.y), az = std::fabs(d.z);
	int kz = (ax >= ay && ax >= az) ? 0 : (ay >= az ? 1 : 2);
	int kx = kz + 1 == 3 ? 0 : kz + 1;
	int ky = kx + 1 == 3 ? 0 : kx + 1;
	if(d[kz] < 0.0f) std::swap(kx, ky);
	r.kx = kx; r.ky = ky; r.kz = kz;
	r.Sx = d[kx] / d[kz];
	r.Sy = d[ky] / d[kz];
	r.Sz = 1.0f / d[kz];
	return r;
}

// Slab test of intersection.cu:47-77 in its robust form (deviation 5).
inline bool box_test(const V3& mn, const V3& mx, const FastRay& r, float tmax, float& cmin) {
	const float lox = (mn.x - r.o.x) * r.inv.x;
	const float loy = (mn.y - r.o.y) * r.inv.y;
	const float loz = (mn.z - r.o.z) * r.inv.z;
	const float hix = (mx.x - r.o.x) * r.inv.x;
	const float hiy = (mx.y - r.o.y) * r.inv.y;
	const float hiz = (mx.z - r.o.z) * r.inv.z;
	cmin = fmax_(fmax_(fmin_(lox, hix), fmin_(loy, hiy)), fmax_(fmin_(loz, hiz), 0.0f));
	const float cfar = fmin_(fmin_(fmax_(lox, hix), fmax_(loy, hiy)), fmax_(loz, hiz));
	return cmin <= tmax && cmin <= cfar * BOX_FAR_SLACK;
}

// Watertight ray/triangle test; returns t and the barycentric weights of v0, v1.
inline bool tri_test(const FastRay& r, V3 v0, V3 v1, V3 v2, float& t, V2& bary) {
	const V3 A = v0 - r.o, B = v1 - r.o, C = v2 - r.o;
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
		U = float(double(Cx) * double(By) - double(Cy) * double(Bx));
		V = float(double(Ax) * double(Cy) - double(Ay) * double(Cx));
		W = float(double(Bx) * double(Ay) - double(By) * double(Ax));
	}
	if((U < 0.0f || V < 0.0f || W < 0.0f) && (U > 0.0f || V > 0.0f || W > 0.0f)) return false;
	const float det = U + V + W;
	if(det == 0.0f) return false;
	const float Az = r.Sz * A[r.kz];
	const float Bz = r.Sz * B[r.kz];
	const float Cz = r.Sz * C[r.kz];
	const float T = U * Az + V * Bz + W * Cz;
	t = T / det;
	bary = { U / det, V / det };
	return true;
}

// a x^2 + b x + c = 0 (real roots, x0 <= x1)
inline bool solve_square(float a, float b, float c, float& x0, float& x1) {
	if(a == 0.0f) {
		if(b == 0.0f) return false;
		x0 = x1 = -c / b;
		return true;
	}
	const float disc = b * b - 4.0f * a * c;
	if(disc < 0.0f) return false;
	const float q = -0.5f * (b + sgn(b) * mbmath::sqrt(disc));
	if(q == 0.0f) { x0 = x1 = 0.0f; return true; }
	float r0 = q / a, r1 = c / q;
	if(r0 > r1) std::swap(r0, r1);
	x0 = r0; x1 = r1;
	return true;
}

inline float pabs(float x) { return x < 0.0f ? -x : x; }

// intersection.cu:85-94
inline float computeU(float v, float A1, float A2, float B1, float B2, float C1, float C2, float D1, float D2) {
	const float a = v * A2 + B2;
	const float b = v * (A2 - A1) + B2 - B1;
	if(std::fabs(b) >= std::fabs(a)) return (v * (C1 - C2) + D1 - D2) / b;
	return (-v * C2 - D2) / a;
}

// intersection.cu:99-179 (Ramsey et al. 2004 bilinear patch)
bool quad_test(V3 p00, V3 p10, V3 p11, V3 p01, const FastRay& ray, float& resT1, float& resT2, V2& uv1, V2& uv2) {
	int d0 = 0, d1 = 1, d2 = 2;
	if(pabs(ray.d.x) < pabs(ray.d.y) || pabs(ray.d.x) < pabs(ray.d.z)) {
		if(pabs(ray.d.y) >= pabs(ray.d.z)) { d0 = 1; d1 = 0; d2 = 2; }
		else { d0 = 2; d1 = 1; d2 = 0; }
	}
	const V3 a = ((p11 - p10) - p01) + p00;
	const V3 b = p10 - p00;
	const V3 c = p01 - p00;
	const V3 d = p00 - ray.o;
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
			uv1 = { u0, v0 };
			resT1 = t0;
			resT2 = -1.0f;
		} else {
			if(v1 >= 0.0f && v1 <= 1.0f) {
				u1 = computeU(v1, A1, A2, B1, B2, C1, C2, D1, D2);
				if(u1 >= 0.0f && u1 <= 1.0f)
					t1 = ((((u1 * v1) * a[d0] + u1 * b[d0]) + v1 * c[d0]) + d[d0]) * ray.inv[d0];
			}
			if(t0 > 0.0f) {
				if(t1 > 0.0f && t1 < t0) { uv1 = { u1, v1 }; uv2 = { u0, v0 }; resT1 = t1; resT2 = t0; }
				else { uv2 = { u1, v1 }; uv1 = { u0, v0 }; resT2 = t1; resT1 = t0; }
			} else {
				uv1 = { u1, v1 }; uv2 = { u0, v0 }; resT1 = t1; resT2 = t0;
			}
		}
		return resT1 > 0.0f;
	}
	return false;
}

// Ray/sphere: nearest root with t > 0; t2 is the far root when t is the near
// one (the alpha test's fallback), else -1.
inline bool sphere_test(const FastRay& r, V3 c, float rad, float& t, float& t2) {
	const V3 oc = r.o - c;
	const float b = dot(oc, r.d);
	const float cc = dot(oc, oc) - rad * rad;
	// The discriminant from the ray's closest approach to the centre (Haines,
	// Guenther and Akenine-Moeller, Ray Tracing Gems ch. 7): b * b - cc cancels
	// for a small sphere far from the origin, and its error then exceeds the
	// shadow rays' 1e-4 origin offset (light paths to a sphere light 15 units
	// away were occluded by the light itself).
	const V3 perp = oc - r.d * b;
	const float disc = rad * rad - dot(perp, perp);
	if(disc < 0.0f) return false;
	const float q = -(b + sgn(b) * mbmath::sqrt(disc));
	float x0, x1;
	if(q == 0.0f) { x0 = x1 = 0.0f; }
	else { x0 = q; x1 = cc / q; if(x0 > x1) std::swap(x0, x1); }
	if(x0 > 0.0f) { t = x0; t2 = x1; return true; }
	if(x1 > 0.0f) { t = x1; t2 = -1.0f; return true; }
	return false;
}
inline bool sphere_test(const FastRay& r, V3 c, float rad, float& t) {
	float t2;
	return sphere_test(r, c, rad, t, t2);
}

inline V3 sample_texture(const Texture& t, V2 uv) {
	// nearest sampling with wrap-around
	float fx = uv.x - std::floor(uv.x), fy = uv.y - std::floor(uv.y);
	i32 x = i32(fx * float(t.w)), y = i32(fy * float(t.h));
	if(x >= i32(t.w)) x = i32(t.w) - 1;
	if(y >= i32(t.h)) y = i32(t.h) - 1;
	const float* p = &t.texels[(size_t(y) * t.w + x) * 4];
	return { p[0], p[1], p[2] };
}

inline V2 bilerp2(V2 x00, V2 x10, V2 x01, V2 x11, float s, float t) {
	const V2 a = (1.0f - s) * x00 + s * x10;
	const V2 b = (1.0f - s) * x01 + s * x11;
	return (1.0f - t) * a + t * b;
}

// Alpha test (intersection.cu:205-216, 235-262, 276-302): the alpha texture of
// primitive p's material, if any, cuts the surface where its first channel is
// below 0.5; uv from the hit's barycentric / bilinear parametrisation, for
// spheres from the object-space hit point.
inline i32 alpha_texture(const Scene& S, const Lod& l, i32 p) {
	const u32 faces = l.nT + l.nQ;
	const u16 m = u32(p) < faces ? l.faceMat[size_t(p)] : l.sphereMat[size_t(u32(p) - faces)];
	return S.materials[m].alphaTex;
}
inline bool alpha_cut_at(const Scene& S, i32 tex, V2 uv) { return sample_texture(S.textures[size_t(tex)], uv).x < 0.5f; }
inline V2 quad_uv(const Lod& l, i32 p, V2 b) {
	const u32 o = u32(p - i32(l.nT)) * 4 + l.nT * 3;
	return bilerp2(l.uvs[l.idx[o]], l.uvs[l.idx[o + 1]], l.uvs[l.idx[o + 3]], l.uvs[l.idx[o + 2]], b.x, b.y);
}
inline V2 sphere_uv(V3 center, const FastRay& r, float t) {
	const V3 n = normalize((r.o + t * r.d) - center);
	return { mbmath::atan2(n.z, n.x) / (2.0f * PI) + 0.5f, mbmath::acos(-n.y) / PI };
}

// Primitive test in object space: returns the object-space t (> 0) and the
// surface parametrisation (intersection.cu:181-316); with `alphaS`, the alpha
// textures of its materials apply, falling back to the second root of a quad
// or sphere whose first root is cut out.
inline bool prim_test(const Lod& l, const FastRay& r, i32 p, float& t, V2& sp, Counters& cnt, const Scene* alphaS = nullptr) {
	if(p < i32(l.nT)) {
		++cnt.tri;
		const u32 o = u32(p) * 3;
		if(!(tri_test(r, l.verts[l.idx[o]], l.verts[l.idx[o + 1]], l.verts[l.idx[o + 2]], t, sp) && t > 0.0f)) return false;
		if(alphaS) {
			const i32 tex = alpha_texture(*alphaS, l, p);
			if(tex >= 0) {
				const V2 uv = (l.uvs[l.idx[o]] * sp.x + l.uvs[l.idx[o + 1]] * sp.y) + l.uvs[l.idx[o + 2]] * ((1.0f - sp.x) - sp.y);
				if(alpha_cut_at(*alphaS, tex, uv)) return false;
			}
		}
		return true;
	}
	const i32 tex = alphaS ? alpha_texture(*alphaS, l, p) : -1;
	if(p < i32(l.nT + l.nQ)) {
		++cnt.quad;
		const u32 o = u32(p - i32(l.nT)) * 4 + l.nT * 3;
		float t1, t2; V2 b1, b2 = { 0, 0 };
		if(!quad_test(l.verts[l.idx[o]], l.verts[l.idx[o + 1]], l.verts[l.idx[o + 2]], l.verts[l.idx[o + 3]], r, t1, t2, b1, b2))
			return false;
		if(tex >= 0 && alpha_cut_at(*alphaS, tex, quad_uv(l, p, b1))) {
			if(!(t2 > 0.0f) || alpha_cut_at(*alphaS, tex, quad_uv(l, p, b2))) return false;
			t1 = t2; b1 = b2;
		}
		t = t1; sp = b1;
		return true;
	}
	++cnt.sphere;
	const i32 s = p - i32(l.nT + l.nQ);
	float t2;
	if(!sphere_test(r, sphere_center(l, s), sphere_radius(l, s), t, t2)) return false;
	if(tex >= 0 && alpha_cut_at(*alphaS, tex, sphere_uv(sphere_center(l, s), r, t))) {
		if(!(t2 > 0.0f) || alpha_cut_at(*alphaS, tex, sphere_uv(sphere_center(l, s), r, t2))) return false;
		t = t2;
	}
	sp = { 0, 0 };
	return true;
}

inline void add_epsilon(V3& o, V3 dir, V3 n) {
	const V3 off = n * SCENE_SCALE_EPS;
	if(dot(n, dir) >= 0.0f) o = o + off; else o = o - off;
}

struct InstRay { FastRay ray; float scale; };
// intersection.cu:322-348
inline InstRay instance_ray(const Scene& S, u32 inst, V3 o, V3 d) {
	const Mat34& W = S.w2i[inst];
	const V3 dirO = xform_dir(W, d);
	const float scale = len(dirO);
	InstRay ir;
	ir.ray = make_ray(xform_point(W, o), dirO / scale);
	ir.scale = scale;
	return ir;
}

struct HitRec {
	float t;
	i32 inst, prim;
	V2 sp;
	bool has;
};

inline bool better(float tw, i32 inst, i32 prim, const HitRec& h) {
	if(tw < h.t) return true;
	if(h.has && tw == h.t) return inst < h.inst || (inst == h.inst && prim < h.prim);
	return false;
}

// BVH traversal inside one instance (closest hit). The stack discipline is
// the reference's (near child first, far child pushed); the result is order
// independent because of the (t, inst, prim) ordering.
void blas_closest(const Scene& S, u32 inst, const InstRay& ir, HitRec& best, Counters& cnt, bool alphaTest = true) {
	const Lod& l = S.lods[S.instLod[inst]];
	const Bvh& bvh = S.lodBvh[S.instLod[inst]];
	const Scene* alphaS = alphaTest && S.hasAlpha ? &S : nullptr;
	auto consider = [&](i32 p) {
		float t; V2 sp;
		if(prim_test(l, ir.ray, p, t, sp, cnt, alphaS)) {
			const float tw = t / ir.scale;
			if(better(tw, i32(inst), p, best)) best = { tw, i32(inst), p, sp, true };
		}
	};
	if(l.numPrims <= 0) return;
	if(l.numPrims == 1) { consider(0); return; }
	const i32 nInt = bvh.numInternal;
	i32 stack[192];
	i32 sp = 0;
	i32 node = 0;
	for(;;) {
		// node < nInt: internal
		if(node < nInt) {
			++cnt.nodeVisits;
			const BvhNode& L = bvh.nodes[2 * node];
			const BvhNode& R = bvh.nodes[2 * node + 1];
			const float tmaxBox = best.t * ir.scale * BOX_SLACK;
			float c0, c1;
			const bool h0 = box_test(L.mn, L.mx, ir.ray, tmaxBox, c0);
			const bool h1 = box_test(R.mn, R.mx, ir.ray, tmaxBox, c1);
			if(!h0) c0 = 1e38f;
			if(!h1) c1 = 1e38f;
			if(h0 && h1) {
				const BvhNode& far = (c1 < c0) ? L : R;
				stack[sp++] = far.index;
				stack[sp++] = far.primCount;
			}
			if(h0 || h1) {
				const BvhNode& nearN = (c0 <= c1) ? L : R;
				if(nearN.index < nInt) { node = nearN.index; continue; }
				const i32 first = nearN.index - nInt;
				for(i32 k = 0; k < nearN.primCount; ++k) consider(bvh.primIds[first + k]);
			}
		} else {
			// unreachable: leaves are handled at their parent
		}
		// pop
		bool found = false;
		while(sp > 0) {
			const i32 pc = stack[--sp];
			const i32 idx = stack[--sp];
			if(idx < nInt) { node = idx; found = true; break; }
			const i32 first = idx - nInt;
			for(i32 k = 0; k < pc; ++k) consider(bvh.primIds[first + k]);
		}
		if(!found) break;
	}
}

bool blas_any(const Scene& S, u32 inst, const InstRay& ir, float tmaxObj, Counters& cnt) {
	const Lod& l = S.lods[S.instLod[inst]];
	const Bvh& bvh = S.lodBvh[S.instLod[inst]];
	auto hits = [&](i32 p) {
		float t; V2 sp;
		return prim_test(l, ir.ray, p, t, sp, cnt, S.hasAlpha ? &S : nullptr) && t < tmaxObj;
	};
	if(l.numPrims <= 0) return false;
	if(l.numPrims == 1) return hits(0);
	const i32 nInt = bvh.numInternal;
	const float tmaxBox = tmaxObj * BOX_SLACK;
	i32 stack[192];
	i32 sp = 0;
	i32 node = 0;
	for(;;) {
		++cnt.nodeVisits;
		const BvhNode& L = bvh.nodes[2 * node];
		const BvhNode& R = bvh.nodes[2 * node + 1];
		float c0, c1;
		const bool h0 = box_test(L.mn, L.mx, ir.ray, tmaxBox, c0);
		const bool h1 = box_test(R.mn, R.mx, ir.ray, tmaxBox, c1);
		if(!h0) c0 = 1e38f;
		if(!h1) c1 = 1e38f;
		if(h0 && h1) {
			const BvhNode& far = (c1 < c0) ? L : R;
			stack[sp++] = far.index;
			stack[sp++] = far.primCount;
		}
		if(h0 || h1) {
			const BvhNode& nearN = (c0 <= c1) ? L : R;
			if(nearN.index < nInt) { node = nearN.index; continue; }
			const i32 first = nearN.index - nInt;
			for(i32 k = 0; k < nearN.primCount; ++k) if(hits(bvh.primIds[first + k])) return true;
		}
		bool found = false;
		while(sp > 0) {
			const i32 pc = stack[--sp];
			const i32 idx = stack[--sp];
			if(idx < nInt) { node = idx; found = true; break; }
			const i32 first = idx - nInt;
			for(i32 k = 0; k < pc; ++k) if(hits(bvh.primIds[first + k])) return true;
		}
		if(!found) return false;
	}
}

// Instance entry: object AABB test (intersection.cu:335-346)
inline bool enter_instance(const Scene& S, u32 inst, V3 o, V3 d, float tmaxWorld, InstRay& ir, Counters& cnt) {
	++cnt.instanceVisits;
	ir = instance_ray(S, inst, o, d);
	const Box& ob = S.lods[S.instLod[inst]].aabb;
	float c;
	return box_test(ob.mn, ob.mx, ir.ray, tmaxWorld * ir.scale * BOX_SLACK, c);
}

template < class F >
void tlas_visit(const Scene& S, const FastRay& wr, const float* tmaxWorld, F&& onInstance, Counters& cnt, bool& stop) {
	stop = false;
	if(S.activeInstances <= 0) return;
	if(S.activeInstances == 1) { onInstance(S.validInstance); return; }
	const Bvh& bvh = S.tlas;
	const i32 nInt = bvh.numInternal;
	i32 stack[192];
	i32 sp = 0;
	i32 node = 0;
	for(;;) {
		++cnt.nodeVisits;
		const BvhNode& L = bvh.nodes[2 * node];
		const BvhNode& R = bvh.nodes[2 * node + 1];
		const float tmaxBox = *tmaxWorld * BOX_SLACK;
		float c0, c1;
		const bool h0 = box_test(L.mn, L.mx, wr, tmaxBox, c0);
		const bool h1 = box_test(R.mn, R.mx, wr, tmaxBox, c1);
		if(!h0) c0 = 1e38f;
		if(!h1) c1 = 1e38f;
		if(h0 && h1) {
			const BvhNode& far = (c1 < c0) ? L : R;
			stack[sp++] = far.index;
			stack[sp++] = far.primCount;
		}
		if(h0 || h1) {
			const BvhNode& nearN = (c0 <= c1) ? L : R;
			if(nearN.index < nInt) { node = nearN.index; continue; }
			const i32 first = nearN.index - nInt;
			for(i32 k = 0; k < nearN.primCount && !stop; ++k) onInstance(u32(bvh.primIds[first + k]));
			if(stop) return;
		}
		bool found = false;
		while(sp > 0) {
			const i32 pc = stack[--sp];
			const i32 idx = stack[--sp];
			if(idx < nInt) { node = idx; found = true; break; }
			const i32 first = idx - nInt;
			for(i32 k = 0; k < pc && !stop; ++k) onInstance(u32(bvh.primIds[first + k]));
			if(stop) return;
		}
		if(!found) return;
	}
}

struct Intersection {
	float distance;
	i32 inst, prim;
	V3 normal, tangentX;
	V2 uv;
	V2 sp;
};

inline V3 bilerp3(V3 x00, V3 x10, V3 x01, V3 x11, float s, float t) {
	const V3 a = (1.0f - s) * x00 + s * x10;
	const V3 b = (1.0f - s) * x01 + s * x11;
	return (1.0f - t) * a + t * b;
}

// intersection.cu:366-621; alphaTest false: every surface opaque
// (first_intersection<dev, false> of wireframe_common.hpp:108)
Intersection first_intersection(const Scene& S, V3& origin, V3 dir, V3 geoN, float tmax, Counters& cnt, bool alphaTest = true) {
	add_epsilon(origin, dir, geoN);
	++cnt.rays;
	const FastRay wr = make_ray(origin, dir);
	HitRec best = { tmax, -1, -1, { 0, 0 }, false };
	bool stop;
	tlas_visit(S, wr, &best.t, [&](u32 inst) {
		InstRay ir;
		if(enter_instance(S, inst, origin, dir, best.t, ir, cnt)) blas_closest(S, inst, ir, best, cnt, alphaTest);
	}, cnt, stop);
	Intersection res;
	res.distance = best.t;
	res.inst = best.has ? best.inst : -1;
	res.prim = best.has ? best.prim : -1;
	res.sp = best.sp;
	res.uv = { 0, 0 };
	res.normal = { 0, 0, 0 };
	res.tangentX = { 0, 0, 0 };
	if(!best.has) return res;
	const Lod& l = S.lods[S.instLod[best.inst]];
	const Mat34& W = S.w2i[best.inst];
	V3 geoNormal, tangentX;
	V2 uv;
	const i32 p = best.prim;
	const i32 sphOff = i32(l.nT + l.nQ);
	if(p >= sphOff) {
		const i32 s = p - sphOff;
		const V3 hitPoint = origin + best.t * dir;
		const V3 local = xform_point(W, hitPoint);
		geoNormal = normalize(local - sphere_center(l, s));
		if(geoNormal.x == 0.0f && geoNormal.y == 0.0f) tangentX = { 1, 0, 0 };
		else {
			const float ll = mbmath::sqrt(geoNormal.y * geoNormal.y + (-geoNormal.x) * (-geoNormal.x));
			tangentX = { geoNormal.y / ll, -geoNormal.x / ll, 0.0f };
		}
		uv.x = mbmath::atan2(geoNormal.z, geoNormal.x) / (2.0f * PI) + 0.5f;
		uv.y = mbmath::acos(-geoNormal.y) / PI;
		res.sp = uv;
	} else if(p < i32(l.nT)) {
		const u32 o = u32(p) * 3;
		const u32 i0 = l.idx[o], i1 = l.idx[o + 1], i2 = l.idx[o + 2];
		const V3 dx0 = l.verts[i1] - l.verts[i0];
		const V3 dx1 = l.verts[i2] - l.verts[i0];
		const V2 du0 = l.uvs[i1] - l.uvs[i0];
		const V2 du1 = l.uvs[i2] - l.uvs[i0];
		const float det = du0.x * du1.y - du0.y * du1.x;
		if(det >= 1e-5f || det <= -1e5f) tangentX = (dx0 * du1.y - dx1 * du0.y) / det;
		else tangentX = dx0;
		geoNormal = cross(dx0, dx1);
		uv = (l.uvs[i0] * best.sp.x + l.uvs[i1] * best.sp.y) + l.uvs[i2] * ((1.0f - best.sp.x) - best.sp.y);
	} else {
		const u32 o = u32(p - i32(l.nT)) * 4 + l.nT * 3;
		const V3 v0 = l.verts[l.idx[o]], v1 = l.verts[l.idx[o + 1]], v2 = l.verts[l.idx[o + 2]], v3 = l.verts[l.idx[o + 3]];
		const V2 t0 = l.uvs[l.idx[o]], t1 = l.uvs[l.idx[o + 1]], t2 = l.uvs[l.idx[o + 2]], t3 = l.uvs[l.idx[o + 3]];
		const float bu = best.sp.x, bv = best.sp.y;
		const V3 dxds = (1.0f - bu) * (v3 - v0) + bu * (v2 - v1);
		const V3 dxdt = (1.0f - bv) * (v1 - v0) + bv * (v2 - v3);
		const V2 duds = (1.0f - bu) * (t3 - t0) + bu * (t2 - t1);
		const V2 dudt = (1.0f - bv) * (t1 - t0) + bv * (t2 - t3);
		const float detD = duds.x * dudt.y - dudt.x * duds.y;
		if(detD >= 1e-9f || detD <= -1e-9f) {
			const float a = dudt.y / detD, b = -duds.y / detD;
			tangentX = { dxds.x * a + dxdt.x * b, dxds.y * a + dxdt.y * b, dxds.z * a + dxdt.z * b };
		} else tangentX = dxds;
		geoNormal = cross(dxdt, dxds);
		uv = bilerp2(t0, t1, t3, t2, bu, bv);
	}
	res.normal = normalize(xform_transposed(W, geoNormal));
	res.tangentX = normalize(xform_transposed(W, tangentX));
	if(p < sphOff) res.uv = uv; else res.uv = res.sp;
	return res;
}

// intersection.cu:624-753
bool any_intersection(const Scene& S, V3 a, V3 b, V3 geoA, V3 geoB, V3 dirAB, Counters& cnt) {
	add_epsilon(a, dirAB, geoA);
	add_epsilon(b, -dirAB, geoB);
	++cnt.rays; ++cnt.shadowRays;
	const V3 corrected = b - a;
	const float tmax = len(corrected);
	const V3 dir = corrected / tmax;
	const FastRay wr = make_ray(a, dir);
	bool occluded = false;
	bool stop = false;
	float tm = tmax;
	tlas_visit(S, wr, &tm, [&](u32 inst) {
		InstRay ir;
		if(enter_instance(S, inst, a, dir, tmax, ir, cnt) && blas_any(S, inst, ir, tmax * ir.scale, cnt)) {
			occluded = true;
			stop = true;
		}
	}, cnt, stop);
	return occluded;
}

struct TangentSpace { V3 shadingN, geoN, shadingTX, shadingTY; };

// tangent_space.hpp:10-66
TangentSpace tangent_space(const Scene& S, const Intersection& h) {
	const Lod& l = S.lods[S.instLod[h.inst]];
	const Mat34& W = S.w2i[h.inst];
	if(u32(h.prim) >= l.nT + l.nQ) return { h.normal, h.normal, h.tangentX, cross(h.normal, h.tangentX) };
	V3 sn;
	if(u32(h.prim) < l.nT) {
		const u32 o = 3u * u32(h.prim);
		sn = (h.sp.x * l.normals[l.idx[o]] + h.sp.y * l.normals[l.idx[o + 1]])
			+ (1.0f - (h.sp.x + h.sp.y)) * l.normals[l.idx[o + 2]];
	} else {
		const u32 o = 4u * u32(h.prim - i32(l.nT)) + 3u * l.nT;
		sn = bilerp3(l.normals[l.idx[o]], l.normals[l.idx[o + 1]], l.normals[l.idx[o + 3]], l.normals[l.idx[o + 2]], h.sp.x, h.sp.y);
	}
	sn = normalize(xform_transposed(W, sn));
	const V3 tx = normalize(h.tangentX - sn * dot(h.tangentX, sn));
	const V3 ty = cross(sn, tx);
	return { sn, h.normal, tx, ty };
}

// ---------------------------------------------------------------- materials
struct Params { i32 type; V3 albedo; V2 roughness; V3 radiance; i32 shadowing; };


inline Params fetch_material(const Scene& S, u16 matIdx, V2 uv) {
	const Material& m = S.materials[matIdx];
	Params p;
	p.type = m.type;
	p.albedo = (m.albedoTex >= 0) ? sample_texture(S.textures[m.albedoTex], uv) : m.albedo;
	p.roughness = m.roughness;
	p.radiance = m.radiance * m.scale;
	p.shadowing = m.shadowing;
	return p;
}

inline u16 material_index(const Scene& S, i32 inst, i32 prim) {
	const Lod& l = S.lods[S.instLod[inst]];
	const u32 faces = l.nT + l.nQ;
	if(u32(prim) < faces) return l.faceMat[prim];
	return l.sphereMat[u32(prim) - faces];
}

struct PathSample { V3 throughput; bool valid; V3 excident; float pdfF, pdfB; };
struct EvalValue { V3 value; float cosOut; float pdfF, pdfB; };

// sampling.hpp:175-181
inline V3 sample_dir_cosine(float u0, float u1, float& cosTheta) {
	cosTheta = mbmath::sqrt(u0);
	const float sinTheta = mbmath::sqrt(1.0f - u0);
	const float phi = u1 * 2.0f * PI;
	float s, c;
	mbmath::sincos(phi, s, c);
	return { sinTheta * s, sinTheta * c, cosTheta };
}
// sampling.hpp:184-192
inline V3 sample_dir_sphere_uniform(float u0, float u1) {
	const float cosTheta = u0 * 2.0f - 1.0f;
	const float sinTheta = mbmath::sqrt((1.0f - cosTheta) * (1.0f + cosTheta));
	const float phi = u1 * 2.0f * PI;
	float s, c;
	mbmath::sincos(phi, s, c);
	return { sinTheta * s, sinTheta * c, cosTheta };
}
inline float projected_area(V3 dir, Box b) {
	const V3 sides = b.mx - b.mn;
	const float ax = sides.y * sides.z * std::fabs(dir.x);
	const float ay = sides.x * sides.z * std::fabs(dir.y);
	const float az = sides.x * sides.y * std::fabs(dir.z);
	return ax + ay + az;
}

// microfacet_base.hpp:85-112 (GGX branch)
inline float geo_smith(float wDotH, V3 w, V2 r) {
	if(wDotH * w.z <= 0.0f) return 0.0f;
	const float a = w.x * r.x, b = w.y * r.y;
	const float oneOverASq = sdiv(a * a + b * b, w.z * w.z);
	return 2.0f / (1.0f + mbmath::sqrt(1.0f + oneOverASq));
}
// microfacet_base.hpp:296-308
inline float eval_ggx(V2 r, V3 h) {
	const float norm = fmax_(PI * r.x * r.y, 1e-30f);
	const float cosThetaSq = h.z * h.z;
	const float rx = sdiv(h.x, r.x), ry = sdiv(h.y, r.y);
	const float tmp = rx * rx + ry * ry + cosThetaSq;
	return sdiv(1.0f, norm * tmp * tmp);
}
// microfacet_base.hpp:227-259
inline V2 sample_slopes_ggx(float tanTheta, float u0, float u1, u64& rnd2) {
	// The reference compares against the double 0.0001; for a float x,
	// x < 0.0001 (double) <=> x <= 0.0001f.
	if(tanTheta <= 0.0001f) {
		const float r = mbmath::sqrt(sdiv(u0, 1.0f - u0));
		const float phi = 6.28318530718f * u1;
		float s, c;
		mbmath::sincos(phi, s, c);
		return { r * c, r * s };
	}
	const float a1 = 1.0f / tanTheta;
	const float g1 = 2.0f / (1.0f + mbmath::sqrt(1.0f + 1.0f / (a1 * a1)));
	const float a = 2.0f * u0 / g1 - 1.0f;
	const float tmp = sdiv(1.0f, a * a - 1.0f);
	const float d = tmp * mbmath::sqrt(tanTheta * tanTheta - (a * a - tanTheta * tanTheta) / tmp);
	const float sx1 = tanTheta * tmp - d;
	const float sx2 = tanTheta * tmp + d;
	const float slopeX = (a < 0.0f || sx2 > 1.0f / tanTheta) ? sx1 : sx2;
	float s;
	if(rnd2 & (1ull << 63)) { rnd2 *= 2; s = 1.0f; } else { rnd2 *= 2; s = -1.0f; }
	const float z = sdiv(u1 * (u1 * (u1 * 0.27385f - 0.73369f) + 0.46341f),
	                     u1 * (u1 * (u1 * 0.093073f + 0.309420f) - 1.000000f) + 0.597999f);
	const float slopeY = s * z * mbmath::sqrt(1.0f + slopeX * slopeX);
	return { slopeX, slopeY };
}
// microfacet_base.hpp:262-293
inline V3 sample_visible_normal_smith(V3 inc, V2 r, float u0, float u1, u64& rnd2) {
	V3 st = normalize(inc * V3{ r.x, r.y, 1.0f });
	if(inc.z < 0.0f) st = -st;
	const float sinTheta = mbmath::sqrt((1.0f - st.z) * (1.0f + st.z));
	const float tanTheta = sinTheta / st.z;
	const float cosPhi = sinTheta > 1e-5f ? st.x / sinTheta : 0.0f;
	const float sinPhi = sinTheta > 1e-5f ? st.y / sinTheta : 0.0f;
	V2 sl = sample_slopes_ggx(tanTheta, u0, u1, rnd2);
	const float tmp = cosPhi * sl.x - sinPhi * sl.y;
	sl.y = sinPhi * sl.x + cosPhi * sl.y;
	sl.x = tmp;
	sl.x *= r.x;
	sl.y *= r.y;
	return normalize(V3{ -sl.x, -sl.y, 1.0f });
}

// microfacet_base.hpp:73-81: V-cavity shadowing of one direction
inline float geo_vcavity(float wDotH, float wDotN, float hDotN) {
	if(wDotH * wDotN <= 0.0f) return 0.0f;
	return fmin_(1.0f, 2.0f * std::fabs(sdiv(hDotN * wDotN, wDotH)));
}
// microfacet_base.hpp:116-142: the multi-bounce compensation applied to
// min(Gi, Ge) for reflection. The eighth power is three squarings.
inline float vcavity_reflection(float gi, float ge) {
	const float g = fmin_(gi, ge);
	if(g < 0.11f) {
		const float x = g + 0.74299714456847f;
		const float x2 = x * x, x4 = x2 * x2;
		return x4 * x4 - 0.092874643071059f;
	}
	return ((1.139400367544197f * g - 3.317658394008854f) * g + 3.317115685385115f) * g - 0.13885765892046f;
}
// microfacet_base.hpp:323-343: a microfacet normal drawn from the GGX
// distribution itself (slope space), with its pdf
inline V3 sample_ndf_ggx(V2 r, float u0, float u1, float& pdf) {
	const float phi = 2.0f * PI * u0;
	const float e = mbmath::sqrt(u1 / (1.0f - u1));
	float s, c;
	mbmath::sincos(phi, s, c);
	float slopeX = e * c, slopeY = e * s;
	const float norm = PI * r.x * r.y;
	const float tmp = 1.0f + slopeX * slopeX + slopeY * slopeY;
	slopeX *= r.x;
	slopeY *= r.y;
	const V3 dir = normalize(V3{ -slopeX, -slopeY, 1.0f });
	pdf = 1.0f / fmax_(norm * tmp * tmp * dir.z * dir.z * dir.z, 1e-20f);
	return dir;
}
// microfacet_base.hpp:149-170: the cavity normal or its mirror image, chosen
// in proportion to their visibility from the incident direction
inline V3 sample_visible_normal_vcavity(V3 inc, V3 cav, u64 rnd, float& iDotH) {
	const V3 adj = { -cav.x, -cav.y, cav.z };
	const float dOut = dot(inc, cav), dAdj = dot(inc, adj);
	const float t = inc.z > 0.0f ? fmax_(0.0f, dAdj) / (fmax_(0.0f, dOut) + fmax_(0.0f, dAdj))
	                             : fmax_(0.0f, -dAdj) / (fmax_(0.0f, -dOut) + fmax_(0.0f, -dAdj));
	if(rnd < percentage_of(~0ull, t)) { iDotH = dAdj; return adj; }
	iDotH = dOut;
	return cav;
}

// half vector for vacuum on both sides (microfacet_base.hpp:15-27)
inline V3 half_vector(V3 inTS, V3 exTS) {
	const V3 h = 1.0f * inTS + 1.0f * exTS;
	const float l = len(h) * sgn(h.z);
	return { sdiv(h.x, l), sdiv(h.y, l), sdiv(h.z, l) };
}

// material_sampling.hpp:77-141 with the Lambert / Torrance(Smith, GGX) / Emissive samplers;
// adjoint: a light sub-path vertex (the shading-normal correction of :132-135)
PathSample material_sample(const TangentSpace& ts, const Params& p, V3 incident, float u0, float u1, u64 i0,
                           bool adjoint = false) {
	PathSample none = { { 0, 0, 0 }, false, { 0, 0, 0 }, 0, 0 };
	const float iDotG = -dot(incident, ts.geoN);
	const float iDotN = -dot(incident, ts.shadingN);
	if(iDotG * iDotN <= 0.0f) return none;
	const V3 inTS = { -dot(incident, ts.shadingTX), -dot(incident, ts.shadingTY), iDotN };
	PathSample res = none;
	if(p.type == OR_MAT_LAMBERT) {
		float cosT;
		const V3 e = sample_dir_cosine(u0, u1, cosT);
		res = { p.albedo, true, e * sgn(inTS.z), e.z / PI, std::fabs(inTS.z) / PI };
	} else if(p.type == OR_MAT_TORRANCE) {
		// microfacet_specular.hpp:26-79
		u64 rnd = i0;
		V3 h;
		float cavityPdf, iDotH;
		if(p.shadowing == 1) {
			h = sample_visible_normal_smith(inTS, p.roughness, u0, u1, rnd);
			cavityPdf = eval_ggx(p.roughness, h);
			cavityPdf *= h.z;
			iDotH = dot(inTS, h);
		} else {
			const V3 cav = sample_ndf_ggx(p.roughness, u0, u1, cavityPdf);
			h = sample_visible_normal_vcavity(inTS, cav, rnd, iDotH);
		}
		const V3 exTS = (2.0f * iDotH) * h - inTS;
		float ge, gi, g;
		if(p.shadowing == 1) {
			ge = geo_smith(iDotH, exTS, p.roughness);
			gi = geo_smith(iDotH, inTS, p.roughness);
			g = gi * ge;
		} else {
			ge = geo_vcavity(iDotH, exTS.z, h.z);
			gi = geo_vcavity(iDotH, inTS.z, h.z);
			g = vcavity_reflection(gi, ge);
		}
		if(ge == 0.0f || gi == 0.0f) return none;
		res = { p.albedo * sdiv(g, gi), true, exTS,
		        cavityPdf * sdiv(gi, std::fabs(4.0f * inTS.z * h.z)),
		        cavityPdf * sdiv(ge, std::fabs(4.0f * exTS.z * h.z)) };
	} else {
		return none;
	}
	if(!nonzero(res.throughput)) return none;
	V3 g = (res.excident.x * ts.shadingTX + res.excident.y * ts.shadingTY) + res.excident.z * ts.shadingN;
	g = normalize(g);
	const float eDotG = dot(g, ts.geoN);
	const float eDotN = res.excident.z;
	if(eDotG * eDotN <= 0.0f) return none;
	res.excident = g;
	res.pdfF = fmin_(res.pdfF, 1e9f);
	res.pdfB = fmin_(res.pdfB, 1e9f);
	if(adjoint)
		res.throughput = res.throughput * ((SHADING_NORMAL_EPS + std::fabs(iDotN * eDotG))
		                                   / (SHADING_NORMAL_EPS + std::fabs(iDotG * eDotN)));
	return res;
}

// material_sampling.hpp:156-237. adjoint: a light sub-path vertex; the
// tangent-space directions are swapped for the BSDF, the value gets the
// shading-normal correction and the pdfs are swapped back. lightNormal: a
// merge; the photon's geometric normal replaces the vertex's in the
// shadow-masking test and the value gets |cos| at the shading over the
// geometric normal (:173, 217-220).
EvalValue material_evaluate(const TangentSpace& ts, const Params& p, V3 incident, V3 excident, bool adjoint = false,
                            const V3* lightNormal = nullptr) {
	EvalValue none = { { 0, 0, 0 }, 0, 0, 0 };
	const float iDotN = -dot(incident, ts.shadingN);
	const float eDotN = dot(excident, ts.shadingN);
	if(p.type == OR_MAT_EMISSIVE) {
		// Emissive materials are neither reflective nor refractive
		if(iDotN * eDotN > 0.0f) return none;
		if(iDotN * eDotN < 0.0f) return none;
	} else {
		if(iDotN * eDotN < 0.0f) return none; // not refractive
	}
	const V3 geoN = lightNormal ? *lightNormal : ts.geoN;
	const float iDotG = -dot(incident, geoN);
	const float eDotG = dot(excident, geoN);
	if(eDotG * eDotN <= 0.0f || iDotG * iDotN <= 0.0f) return none;
	V3 inTS = { -dot(incident, ts.shadingTX), -dot(incident, ts.shadingTY), iDotN };
	V3 exTS = { dot(excident, ts.shadingTX), dot(excident, ts.shadingTY), eDotN };
	if(adjoint) std::swap(inTS, exTS);
	V3 value; float pf, pb;
	if(p.type == OR_MAT_LAMBERT) {
		if(inTS.z * exTS.z < 0.0f) return none;
		value = p.albedo / PI;
		pf = std::fabs(exTS.z) / PI;
		pb = std::fabs(inTS.z) / PI;
	} else if(p.type == OR_MAT_TORRANCE) {
		const V3 h = half_vector(inTS, exTS);
		if(inTS.z * exTS.z < 0.0f) return none;
		const float iDotH = dot(inTS, h);
		float ge, gi, g;
		if(p.shadowing == 1) {
			ge = geo_smith(iDotH, exTS, p.roughness);
			gi = geo_smith(iDotH, inTS, p.roughness);
			g = gi * ge;
		} else {
			ge = geo_vcavity(iDotH, exTS.z, h.z);
			gi = geo_vcavity(iDotH, inTS.z, h.z);
			g = vcavity_reflection(gi, ge);
		}
		if(ge == 0.0f || gi == 0.0f) return none;
		const float dd = eval_ggx(p.roughness, h);
		value = p.albedo * sdiv(g * dd, std::fabs(4.0f * inTS.z * exTS.z));
		pf = sdiv(gi * dd, std::fabs(4.0f * inTS.z));
		pb = sdiv(ge * dd, std::fabs(4.0f * exTS.z));
	} else {
		return none;
	}
	if(!nonzero(value)) return none;
	if(lightNormal) {
		value = value * ((SHADING_NORMAL_EPS + std::fabs(eDotN)) / (SHADING_NORMAL_EPS + std::fabs(eDotG)));
		return { value, std::fabs(eDotN), fmin_(pf, 1e9f), fmin_(pb, 1e9f) };
	}
	if(adjoint) {
		value = value * ((SHADING_NORMAL_EPS + std::fabs(iDotN * eDotG)) / (SHADING_NORMAL_EPS + std::fabs(iDotG * eDotN)));
		return { value, std::fabs(eDotN), fmin_(pb, 1e9f), fmin_(pf, 1e9f) };
	}
	return { value, std::fabs(eDotN), fmin_(pf, 1e9f), fmin_(pb, 1e9f) };
}

// ---------------------------------------------------------------- lights
inline V3 quad_light_center(const PosLight& l) {
	return (l.posV[0] + (l.posV[1] + l.posV[2]) * 0.5f) + l.posV[3] * 0.25f;
}
inline V3 light_center(const PosLight& l) {
	if(l.type == LT_QUAD) return quad_light_center(l);
	if(l.type == LT_TRI) return l.posV[0] + (l.posV[1] + l.posV[2]) / 3.0f; // lights.hpp:216-220
	return l.position;
}
inline float light_flux(const Scene& S, const PosLight& l) {
	if(l.type == LT_POINT) {
		const V3 f = l.intensity * 4.0f * PI;
		return (f.x + f.y) + f.z;
	}
	if(l.type == LT_SPHERE) {
		// lights.cpp:63-80: the mean of 128 radiance samples (constant here)
		// times the sphere's area times 2 pi
		const Material& m = S.materials[l.material];
		const V3 rad = m.radiance * m.scale;
		const float area = ((4.0f * PI) * l.radius) * l.radius;
		V3 sum = { 0, 0, 0 };
		for(int i = 0; i < 128; ++i) sum = sum + rad;
		sum = sum / 128.0f;
		const V3 f = sum * area * 2.0f * PI;
		return (f.x + f.y) + f.z;
	}
	if(l.type == LT_TRI) {
		// lights.cpp:24-40: the mean of 128 radiance samples (a constant emission
		// adds the same value every time) times area times 2 pi
		const Material& m = S.materials[l.material];
		const V3 rad = m.radiance * m.scale;
		const float area = len(cross(l.posV[1], l.posV[2])) / 2.0f;
		V3 sum = { 0, 0, 0 };
		for(int i = 0; i < 128; ++i) sum = sum + rad;
		sum = sum / 128.0f;
		const V3 f = sum * area * 2.0f * PI;
		return (f.x + f.y) + f.z;
	}
	// lights.cpp:43-62: for constant emission textures every one of the 128
	// samples adds the same value; the per-sample area is the local
	// parallelogram area at a low-discrepancy sample point.
	const Material& m = S.materials[l.material];
	const V3 rad = m.radiance * m.scale;
	// GoldenRatio2D seeded from the light's address in the reference; here
	// seeded from its index in the light list (deterministic).
	u64 state = scramble_seed(u32(l.primId) * 2654435761u + u32(l.primInst)); // GoldenRatio2D(seed)
	V3 sum = { 0, 0, 0 };
	for(int i = 0; i < 128; ++i) {
		const u64 s = golden_ratio2d_next(state);
		const float ux = sample_uniform(u32(s & 0xffffffffull));
		const float uy = sample_uniform(u32(s >> 32ull));
		const V3 tx = l.posV[1] + ux * l.posV[3];
		const V3 ty = l.posV[2] + uy * l.posV[3];
		const float area = len(cross(ty, tx));
		sum = sum + area * rad;
	}
	sum = sum / 128.0f;
	const V3 f = sum * 2.0f * PI;
	return (f.x + f.y) + f.z;
}

// light_tree.cpp:120-330 (positional sub-tree) and fill_map
void build_pos_tree(const Scene& S, LightTree& T) {
	auto& lights = T.lights;
	const size_t n = lights.size();
	T.nodes.clear();
	T.primToNodePath.clear();
	if(n == 0) { T.rootFlux = 0.0f; T.rootType = INTERNAL_NODE; return; }
	std::vector<float> flux(n);
	for(size_t i = 0; i < n; ++i) flux[i] = light_flux(S, lights[i]);
	if(n == 1) {
		T.rootType = lights[0].type;
		T.rootIndex = 0;
		T.rootFlux = flux[0];
		if(lights[0].primInst != -1) T.primToNodePath[{ lights[0].primInst, lights[0].primId }] = 0u;
		return;
	}
	size_t height = 0;
	while((size_t(1) << (height + 1)) <= n) ++height;
	const size_t extra = n - (size_t(1) << height);
	const size_t internalCount = ((size_t(1) << height) - 1) + extra;
	T.nodes.assign(internalCount, LightNode{});
	auto lightRef = [&](size_t i) { return LightNodeRef{ flux[i], i32(i), lights[i].type }; };
	auto nodeRef = [&](size_t i) {
		const LightNode& nd = T.nodes[i];
		return LightNodeRef{ nd.left.flux + nd.right.flux, i32(i), INTERNAL_NODE };
	};
	auto refCenter = [&](const LightNodeRef& r) {
		if(r.type == INTERNAL_NODE) return T.nodes[r.index].center;
		return light_center(lights[r.index]);
	};
	auto makeNode = [&](size_t at, LightNodeRef l, LightNodeRef r) {
		LightNode nd;
		nd.left = l;
		nd.right = r;
		nd.center = (refCenter(l) + refCenter(r)) / 2.0f;
		T.nodes[at] = nd;
	};
	if(extra > 0) {
		const size_t startNode = (size_t(1) << height) - 1;
		const size_t startLight = n - 2 * extra;
		for(size_t i = 0; i < extra; ++i) makeNode(startNode + i, lightRef(startLight + 2 * i), lightRef(startLight + 2 * i + 1));
		const size_t startInner = (size_t(1) << (height - 1)) - 1;
		for(size_t i = 0; i < extra / 2; ++i) makeNode(startInner + i, nodeRef(startNode + 2 * i), nodeRef(startNode + 2 * i + 1));
		if(extra % 2 != 0) makeNode(startInner + extra / 2, nodeRef(startNode + extra - 1), lightRef(0));
	}
	const size_t startLight = (extra % 2 == 0) ? 0 : 1;
	const size_t levelNodeCount = n - 2 * extra - startLight;
	const size_t nodeCount = levelNodeCount / 2;
	const size_t startNodeIndex = (size_t(1) << height) - nodeCount - 1;
	for(size_t i = 0; i < nodeCount; ++i) makeNode(startNodeIndex + i, lightRef(startLight + 2 * i), lightRef(startLight + 2 * i + 1));
	if(height > 1) {
		for(size_t level = height - 1; level >= 1; --level) {
			const size_t nodes = size_t(1) << level;
			const size_t inner = nodes / 2 - 1;
			for(size_t i = 0; i < nodes / 2; ++i) makeNode(inner + i, nodeRef(nodes - 1 + 2 * i), nodeRef(nodes - 1 + 2 * i + 1));
		}
	}
	T.rootType = INTERNAL_NODE;
	T.rootIndex = 0;
	T.rootFlux = T.nodes[0].left.flux + T.nodes[0].right.flux;
	// fill_map
	int h = int(height);
	const u32 lowerLightCount = u32(1u << h) - u32(extra);
	u32 i = 0;
	if(extra > 0) {
		for(; i < lowerLightCount; ++i) {
			if(lights[i].primInst != -1) {
				u32 code = ((1u << h) - 1) - (lowerLightCount - i - 1);
				code <<= (32 - h);
				T.primToNodePath[{ lights[i].primInst, lights[i].primId }] = code;
			}
		}
		h += 1;
	}
	for(; i < n; ++i) {
		if(lights[i].primInst != -1) {
			const u32 code = (i - lowerLightCount) << (32 - h);
			T.primToNodePath[{ lights[i].primInst, lights[i].primId }] = code;
		}
	}
}

struct Nee {
	V3 position;
	float creationPdf;
	V3 dir;
	float dirPdf;
	float cosOut;
	V3 diffIrradiance;
	float dist;
	V3 geoNormal;
	float distSq;
	bool valid;
	i32 emitMat = -1; // material of the sampled area light (-1: point light, background)
};

// light_sampling.hpp:143-171 + 369-390
Nee connect_quad(const Scene& S, const PosLight& l, V3 pos, float u0, float u1) {
	const V3 tx = l.posV[1] + u0 * l.posV[3];
	const V3 ty = l.posV[2] + u1 * l.posV[3];
	V3 normal = cross(ty, tx);
	const float area = len(normal);
	normal = normal / area;
	const V3 position = (l.posV[0] + tx * u1) + l.posV[2] * u0;
	const V2 uv = ((l.uvV[0] + l.uvV[1] * u1) + l.uvV[2] * u0) + l.uvV[3] * (u0 * u1);
	(void)uv;
	const Material& m = S.materials[l.material];
	const V3 radiance = m.type == OR_MAT_EMISSIVE ? m.radiance * m.scale : V3{ 0, 0, 0 };
	const V3 intensity = radiance * area;
	const float pdf = 1.0f / area;
	V3 direction = position - pos;
	const float distSq = lensq(direction) + DISTANCESQ_EPSILON;
	const float dist = mbmath::sqrt(distSq);
	direction = direction / dist;
	// evaluate_area(-direction, intensity, normal)
	const float cosOut = dot(normal, -direction);
	V3 value = { 0, 0, 0 }; float vcos = 0.0f, vpdf = 0.0f;
	if(cosOut > 0.0f) { value = intensity; vcos = cosOut; vpdf = cosOut / PI; }
	const V3 diff = value / distSq;
	return { position, pdf, direction, vpdf, vcos, diff, dist, normal, distSq, true, i32(l.material) };
}

// light_sampling.hpp:117-140 + 347-368; sampling.hpp:123-128 (barycentric sample)
Nee connect_tri(const Scene& S, const PosLight& l, V3 pos, float u0, float u1) {
	V3 normal = cross(l.posV[1], l.posV[2]);
	const float area2 = len(normal);
	normal = normal / area2;
	const float area = area2 * 0.5f;
	const float bs = 1.0f - mbmath::sqrt(1.0f - u0);
	const float bt = (1.0f - bs) * u1;
	const V3 position = (l.posV[0] + l.posV[1] * bs) + l.posV[2] * bt;
	const Material& m = S.materials[l.material];
	const V3 radiance = m.type == OR_MAT_EMISSIVE ? m.radiance * m.scale : V3{ 0, 0, 0 };
	const V3 intensity = radiance * area;
	const float pdf = 1.0f / area;
	V3 direction = position - pos;
	const float distSq = lensq(direction) + DISTANCESQ_EPSILON;
	const float dist = mbmath::sqrt(distSq);
	direction = direction / dist;
	const float cosOut = dot(normal, -direction);
	V3 value = { 0, 0, 0 }; float vcos = 0.0f, vpdf = 0.0f;
	if(cosOut > 0.0f) { value = intensity; vcos = cosOut; vpdf = cosOut / PI; }
	const V3 diff = value / distSq;
	return { position, pdf, direction, vpdf, vcos, diff, dist, normal, distSq, true, i32(l.material) };
}

inline V3 perpendicular(V3 n);

// sampling.hpp:112-119: a direction in the cone cos theta >= maxCos about +z
inline V3 sample_cone_uniform(float maxCos, float u0, float u1, float& pdf) {
	const float cosTheta = (1.0f - u0) + u0 * maxCos;
	const float sinTheta = mbmath::sqrt(1.0f - cosTheta * cosTheta);
	const float phi = (2.0f * u1) * PI;
	float s, c;
	mbmath::sincos(phi, s, c);
	pdf = 1.0f / ((2.0f * PI) * (1.0f - maxCos));
	return { c * sinTheta, s * sinTheta, cosTheta };
}

// light_sampling.hpp:389-430: the cap of the sphere seen from pos, sampled
// uniformly by solid angle; from inside the sphere an empty sample (valid,
// without irradiance)
Nee connect_sphere(const Scene& S, const PosLight& l, V3 pos, float u0, float u1) {
	Nee n{};
	n.valid = true;
	n.emitMat = i32(l.material);
	V3 centerDir = pos - l.position;
	const float dist = len(centerDir);
	if(dist <= l.radius) return n;
	centerDir = centerDir / dist;
	const float cosSphere = l.radius / dist;
	float conePdf;
	const V3 d = sample_cone_uniform(cosSphere, u0, u1, conePdf);
	const V3 tx = normalize(perpendicular(centerDir));
	const V3 ty = cross(centerDir, tx);
	const V3 globalDir = (tx * d.x + ty * d.y) + centerDir * d.z;
	const V3 surfPos = l.position + globalDir * l.radius;
	V3 connection = surfPos - pos;
	const float cDistSq = lensq(connection) + DISTANCESQ_EPSILON;
	const float cDist = mbmath::sqrt(cDistSq);
	connection = connection / cDist;
	const Material& m = S.materials[l.material];
	const V3 radiance = m.type == OR_MAT_EMISSIVE ? m.radiance * m.scale : V3{ 0, 0, 0 };
	const float sampleArea = (l.radius * l.radius) / conePdf;
	const float cosOut = std::fmax(0.0f, -dot(globalDir, connection));
	return { surfPos, 1.0f / sampleArea, connection, cosOut / PI, cosOut, radiance * (sampleArea / cDistSq), cDist,
	         globalDir, cDistSq, true, i32(l.material) };
}

// light_sampling.hpp:308-325
Nee connect_point(const PosLight& l, V3 pos) {
	V3 direction = l.position - pos;
	const float distSq = lensq(direction) + DISTANCESQ_EPSILON;
	const float dist = mbmath::sqrt(distSq);
	direction = direction / dist;
	const V3 diff = l.intensity / distSq;
	return { l.position, INF_PDF, direction, 1.0f / (4.0f * PI), 0.0f, diff, dist, { 0, 0, 0 }, distSq, true };
}

// light_sampling.hpp:447-462
Nee connect_background(const LightTree& T, V3 pos, Box bounds, float u0, float u1) {
	const V3 dir = sample_dir_sphere_uniform(u0, u1);
	const float dirPdf = 1.0f / (4.0f * PI);
	const V3 radiance = T.bgColor * T.bgScale;
	const float posPdf = 1.0f / projected_area(dir, bounds);
	const V3 diff = radiance / dirPdf;
	const float creation = dirPdf * std::fabs(1.0f) / (MAX_SCENE_SIZE * MAX_SCENE_SIZE);
	return { pos + dir * len(bounds.mx - bounds.mn), creation, dir, posPdf, 1.0f, diff,
	         MAX_SCENE_SIZE, { 0, 0, 0 }, MAX_SCENE_SIZE * MAX_SCENE_SIZE, true };
}

inline Nee adjust(Nee n, float chance) {
	n.creationPdf *= chance;
	n.diffIrradiance = n.diffIrradiance / chance;
	return n;
}

Nee connect_pos_light(const Scene& S, const PosLight& l, V3 pos, float u0, float u1) {
	if(l.type == LT_QUAD) return connect_quad(S, l, pos, u0, u1);
	if(l.type == LT_TRI) return connect_tri(S, l, pos, u0, u1);
	if(l.type == LT_SPHERE) return connect_sphere(S, l, pos, u0, u1);
	return connect_point(l, pos);
}

// light_tree_sampling.hpp:278-329 and 195-259
Nee lights_connect(const Scene& S, u64 index, u64 numIndices, u64 seed, V3 position, float u0, float u1) {
	const LightTree& T = S.lightTree;
	u64 rndChoice = numIndices > 0 ? seed + index * (~0ull / numIndices) : seed;
	if(rndChoice == ~0ull) --rndChoice;
	const float bgSum = (T.bgFlux.x + T.bgFlux.y) + T.bgFlux.z;
	const float fluxSum = (bgSum + T.dirFlux) + T.rootFlux;
	Nee none{};
	none.valid = false;
	if(!(fluxSum > 0.0f)) return none;
	const float envProb = bgSum / fluxSum;
	const float dirProb = T.dirFlux / fluxSum;
	const float posProb = T.rootFlux / fluxSum;
	const u64 rightEnv = percentage_of(~0ull, envProb);
	if(rndChoice < rightEnv) return adjust(connect_background(T, position, S.aabb, u0, u1), envProb);
	u64 right = percentage_of(~0ull, envProb + dirProb);
	u64 left = rightEnv;
	float p = dirProb;
	if(rndChoice < right) {
		return none; // no directional lights are supported
	}
	left = right;
	right = ~0ull;
	p = posProb;
	// traverse the positional tree
	u16 type = T.rootType;
	i32 index2 = T.rootIndex;
	u64 iL = left, iR = right;
	float lightProb = p;
	i32 nodeIdx = 0;
	while(type == INTERNAL_NODE) {
		const LightNode& nd = T.nodes[nodeIdx];
		const float probLeft = nd.left.flux / (nd.left.flux + nd.right.flux);
		const u64 boundary = iL + percentage_of(iR - iL, probLeft);
		if(rndChoice < boundary) {
			type = nd.left.type; index2 = nd.left.index; iR = boundary; lightProb *= probLeft;
		} else {
			type = nd.right.type; index2 = nd.right.index; iL = boundary; lightProb *= (1.0f - probLeft);
		}
		nodeIdx = index2;
	}
	return adjust(connect_pos_light(S, T.lights[index2], position, u0, u1), lightProb);
}

// light_tree_sampling.hpp:340-412: the area pdfs of a hit on an area light,
// for starting a light path there (emit) and for a next-event sample of it
// from refPos (connect); they differ for spheres.
struct LightPdfs { float emit, connect; };
LightPdfs light_pdfs(const Scene& S, i32 inst, i32 prim, V2 sp, V3 refPos) {
	const LightTree& T = S.lightTree;
	const float bgSum = (T.bgFlux.x + T.bgFlux.y) + T.bgFlux.z;
	float p = T.rootFlux / ((T.dirFlux + T.rootFlux) + bgSum);
	auto it = T.primToNodePath.find({ inst, prim });
	if(it == T.primToNodePath.end()) return { 0.0f, 0.0f };
	u32 code = it->second;
	u16 type = T.rootType;
	i32 idx = T.rootIndex;
	i32 nodeIdx = 0;
	while(type == INTERNAL_NODE) {
		const LightNode& nd = T.nodes[nodeIdx];
		const float pLeft = nd.left.flux / (nd.left.flux + nd.right.flux);
		if(code & 0x80000000u) { p *= (1.0f - pLeft); type = nd.right.type; idx = nd.right.index; }
		else { p *= pLeft; type = nd.left.type; idx = nd.left.index; }
		nodeIdx = idx;
		code <<= 1;
	}
	const PosLight& l = T.lights[idx];
	if(l.type == LT_QUAD) {
		const V3 tx = l.posV[1] + sp.x * l.posV[3];
		const V3 ty = l.posV[2] + sp.y * l.posV[3];
		const float a = p / len(cross(ty, tx));
		return { a, a };
	}
	if(l.type == LT_TRI) {
		const float a = p / (len(cross(l.posV[1], l.posV[2])) / 2.0f);
		return { a, a };
	}
	if(l.type == LT_SPHERE) {
		const float cosSphere = l.radius / len(refPos - l.position);
		const float solidAngle = (2.0f * PI) * (1.0f - cosSphere);
		const float rsq = l.radius * l.radius;
		return { p / ((4.0f * PI) * rsq), p / (solidAngle * rsq) };
	}
	return { 0.0f, 0.0f };
}

// ---------------------------------------------------------------- path tracer
enum VType { V_CAMERA, V_SURFACE, V_VOID };

struct Vertex {
	VType type;
	V3 position;
	V3 incidentEncoded;
	i32 pathLen;
	float incidentPdf;
	TangentSpace ts;
	i32 inst, prim;
	V2 surfaceParams;
	Params mat;
};

// render_target.hpp:64-75: a NaN channel of a contribution is replaced by 0
inline float nan_to_zero(float x) { return std::isnan(x) ? 0.0f : x; }
inline V3 contribute(V3 acc, V3 c) { return { acc.x + nan_to_zero(c.x), acc.y + nan_to_zero(c.y), acc.z + nan_to_zero(c.z) }; }

inline V3 incident_direction(const Vertex& v) {
	const V3 e = v.incidentEncoded;
	float t = 1.0f - e.x * e.x - e.y * e.y;
	t = std::fmin(std::fmax(t, 0.0f), 1.0f);
	return { e.x, e.y, sgn(e.z) * mbmath::sqrt(t) };
}

// The path tracer's auxiliary targets (pt_params.hpp:16-26, pt_common.hpp:
// 146-152): per pixel and iteration 13 channels, position 3, depth 1, normal 3,
// uv 2, albedo 3, lightness 1.
enum { AUX_POS = 0, AUX_DEPTH = 3, AUX_NORMAL = 4, AUX_UV = 7, AUX_ALBEDO = 9, AUX_LIGHT = 12, AUX_CHANNELS = 13 };

struct PtState {
	const Scene* scene;
	OrPtParams params;
	std::vector<Pcg64> rngs;
	std::vector<float> radiance, hitId;       // cumulative
	std::vector<float> radianceVar, hitIdVar; // their variances
	std::vector<float> aux, auxVar;           // AUX_CHANNELS per pixel: cumulative means, variances
	i32 iteration = -1;
	Counters stats;
};

// output_handler_variance.hpp:7-31, one channel of a target: the running mean
// and its variance (UpdateIter<T, false>) ...
inline void update_moments(float iter, float& cum, float& var, float iteration) {
	const float diff = iter - cum;
	cum += diff / std::fmax(1.0f, iteration + 1.0f);
	const float varIter = diff * (iter - cum);
	const float varDiff = varIter - var;
	var += varDiff / std::fmax(1.0f, iteration);
}
// ... or, for a target that reduces moments (the light tracer's Density,
// render_targets.hpp:68-74), the iteration's value and the running mean in
// the variance slot (UpdateIter<T, true>).
inline void update_reduced(float iter, float& cum, float& mean, float iteration) {
	cum = iter;
	const float diff = iter - mean;
	mean += diff / std::fmax(1.0f, iteration + 1.0f);
}

// pinhole.hpp:58-81
inline V3 pinhole_ray(const Camera& c, i32 px, i32 py, float u0, float u1, float& pdf) {
	const V2 sub = { float(px) + u0, float(py) + u1 };
	V2 cp = { sub.x / float(c.resX), sub.y / float(c.resY) };
	cp = { cp.x * 2.0f - 1.0f, cp.y * 2.0f - 1.0f };
	cp = { cp.x * c.tanVFov, cp.y * c.tanVFov };
	const float aspect = float(c.resX) / float(c.resY);
	const V3 nPos = { cp.x * aspect, cp.y, 1.0f };
	const V3 xAxis = cross(c.viewDir, c.up);
	const V3 dir = normalize((xAxis * nPos.x + c.up * nPos.y) + c.viewDir * nPos.z);
	const float t2 = 2.0f * c.tanVFov;
	const float pixelArea = (t2 * t2) * aspect;
	const float cosOut = dot(c.viewDir, dir);
	pdf = 1.0f / (((pixelArea * cosOut) * cosOut) * cosOut);
	return dir;
}

// Records, in pt_sample's order, the terms a path sample adds to its radiance
// and its Lambert vertices that look up albedo texture texIndex, and keeps in
// double precision, per such vertex, the sum of the terms added after it
// (its own next-event terms included). With Russian roulette off each of
// those terms contains the vertex's albedo once, so the derivative of the
// sample with respect to that albedo is suffix / albedo. This is the CPU
// reference of the GPU path-replay adjoint (test infrastructure).
// The same replay also gives the derivative of the sample with respect to
// the emitted radiance L (radiance x scale) of one emissive material
// (emissionMat >= 0): every term that material emits, at an emitter hit or
// through next-event estimation, is linear in L, so it adds term / L
// (Russian roulette may stay on: its probabilities do not depend on L).
struct AlbedoAdjoint {
	i32 texIndex = -1;
	int n = 0;
	i32 texel[64];
	double alb[64][3], suf[64][3];
	i32 emissionMat = -1;
	V3 emissionL = { 0, 0, 0 };
	double emis[3] = { 0, 0, 0 };
	void add_all(const V3& c) {
		for(int k = 0; k < n; ++k) { suf[k][0] += c.x; suf[k][1] += c.y; suf[k][2] += c.z; }
	}
	void emitted(const V3& c, i32 mat) {
		if(emissionMat < 0 || mat != emissionMat) return;
		const float L[3] = { emissionL.x, emissionL.y, emissionL.z }, t[3] = { c.x, c.y, c.z };
		for(int k = 0; k < 3; ++k) if(L[k] > 0.0f) emis[k] += double(t[k]) / double(L[k]);
	}
	void vertex(const Scene& S, const V3& e, bool surface, i32 type, i32 mat, V2 uv, V3 albedo);
};

// FootprintV0::add_segment (footprint.hpp:137-165) of a camera path: the
// camera vertex starts with m_a = 0 and pChoice 1 (path_util.hpp:553), every
// sampled direction adds 1 / sqrt(its pdf), roulette passes 1; the guide
// weight of the vertex reached is 1 / (1 + solid angle), solid angle = m_a^2
// (pt_common.hpp:49-61).
inline float guide_after_segment(float& ma, float pdf) {
	ma = ma + 1.0f / mbmath::sqrt(pdf);
	return 1.0f / (1.0f + ma * ma);
}
// ei::avg of the emission (the mean of the three channels)
inline float avg3(V3 v) { return ((v.x + v.y) + v.z) / 3.0f; }

// pt_common.hpp:75-156
void pt_sample(PtState& st, i32 px, i32 py, Pcg64& rng, V3& radianceOut, V2& hitOut, Counters& cnt,
               AlbedoAdjoint* adj = nullptr, float* aux = nullptr) {
	const Scene& S = *st.scene;
	const OrPtParams& P = st.params;
	V3 throughput = { 1, 1, 1 };
	V3 radiance = { 0, 0, 0 };
	V2 hitAcc = { 0, 0 };
	Vertex v{};
	v.type = V_CAMERA;
	v.position = S.cam.position;
	v.incidentEncoded = { float(px), float(py), 0.0f };
	v.pathLen = 0;
	v.incidentPdf = 1.0f;
	v.inst = v.prim = -1;
	(void)rng.next(); // create_camera consumes one number (unused by the pinhole camera)
	int pathLen = 0;
	float guideA = 0.0f, guideWeight = 1.0f;
	auto aux_add = [&](int c, float x) { if(aux) aux[c] += nan_to_zero(x); };
	do {
		if(pathLen > 0 && pathLen + 1 >= P.minPathLength && pathLen + 1 <= P.maxPathLength) {
			const u64 neeSeed = rng.next();
			for(int i = 0; i < P.neeCount; ++i) {
				const u64 r = rng.next();
				const float nu0 = sample_uniform(u32(r)), nu1 = sample_uniform(u32(r >> 32));
				Nee nee = lights_connect(S, u64(i), u64(P.neeCount), neeSeed, v.position, nu0, nu1);
				if(!nee.valid) continue;
				EvalValue val = material_evaluate(v.ts, v.mat, incident_direction(v), nee.dir);
				if(nee.cosOut != 0.0f) val.cosOut *= nee.cosOut;
				const V3 rad = val.value * nee.diffIrradiance;
				if(any_pos(rad) && val.cosOut > 0.0f) {
					const bool occ = any_intersection(S, v.position, nee.position, v.ts.geoN, nee.geoNormal, nee.dir, cnt);
					if(!occ) {
						const float hitPdf = val.pdfF * std::fabs(nee.cosOut) / nee.distSq;
						const float mis = 1.0f / (float(P.neeCount) + hitPdf / nee.creationPdf);
						radiance = contribute(radiance, ((throughput * val.cosOut) * rad) * mis);
						if(adj) {
							const V3 term = contribute(V3{ 0, 0, 0 }, ((throughput * val.cosOut) * rad) * mis);
							adj->add_all(term);
							adj->emitted(term, nee.emitMat);
						}
						aux_add(AUX_LIGHT, guideWeight * val.cosOut);
					}
				}
			}
		}
		// walk (random_walk.hpp:38-113)
		const u64 x0 = rng.next(), x1 = rng.next();
		const float ru0 = sample_uniform(u32(x0)), ru1 = sample_uniform(u32(x0 >> 32));
		const float rr = sample_uniform(u32(rng.next()));
		V3 origin, excident;
		V3 sThroughput;
		float pdfF;
		if(v.type == V_CAMERA) {
			excident = pinhole_ray(S.cam, px, py, ru0, ru1, pdfF);
			sThroughput = { 1, 1, 1 };
			origin = v.position;
		} else {
			PathSample s = material_sample(v.ts, v.mat, incident_direction(v), ru0, ru1, x1);
			if(!s.valid) break;
			excident = s.excident;
			sThroughput = s.throughput;
			pdfF = s.pdfF;
			origin = v.position;
		}
		throughput = throughput * sThroughput;
		if(pathLen >= P.rrStartDepth) {
			const float cp = fmin_(maxc(throughput) + 0.1f, 1.0f);
			if(rr >= cp) break;
			throughput = throughput / cp;
		}
		const V3 geoN = (v.type == V_SURFACE) ? v.ts.geoN : V3{ 0, 0, 0 };
		const V3 lastPosition = v.position; // pt_common.hpp:126
		Intersection hit = first_intersection(S, origin, excident, geoN, MAX_SCENE_SIZE, cnt);
		i32 vMat = -1;
		const V2 vUv = hit.uv;
		if(hit.inst < 0) {
			v.type = V_VOID;
			v.incidentEncoded = excident;
			v.position = { 0, 0, 0 };
			v.incidentPdf = pdfF * 1.0f;
		} else {
			const V3 position = origin + excident * hit.distance;
			const TangentSpace ts = tangent_space(S, hit);
			v.type = V_SURFACE;
			v.position = position;
			v.incidentEncoded = { excident.x, excident.y, hit.distance * sgn(excident.z) };
			v.ts = ts;
			v.inst = hit.inst;
			v.prim = hit.prim;
			v.surfaceParams = hit.sp;
			vMat = material_index(S, hit.inst, hit.prim);
			v.mat = fetch_material(S, u16(vMat), hit.uv);
			const float inCosAbs = std::fabs(dot(excident, ts.shadingN));
			v.incidentPdf = pdfF * std::fabs(inCosAbs) / (hit.distance * hit.distance);
		}
		if(pathLen == 0) hitAcc = { float(v.type == V_SURFACE ? v.inst : -1), float(v.type == V_SURFACE ? v.prim : -1) };
		guideWeight = guide_after_segment(guideA, pdfF);
		++pathLen;
		if(pathLen >= P.minPathLength) {
			V3 emission = { 0, 0, 0 };
			float connectPdf = 0.0f;
			if(v.type == V_VOID) {
				if(S.lightTree.hasBackground) {
					emission = S.lightTree.bgColor * S.lightTree.bgScale;
					if(nonzero(emission)) {
						const LightTree& T = S.lightTree;
						const float bgFlux = (T.bgFlux.x + T.bgFlux.y) + T.bgFlux.z;
						const float p = bgFlux / ((T.dirFlux + T.rootFlux) + bgFlux);
						connectPdf = (1.0f / (4.0f * PI)) * p;
					}
				}
			} else if(v.mat.type == OR_MAT_EMISSIVE) {
				const V3 ex = -incident_direction(v);
				const float cosOut = dot(v.ts.geoN, ex);
				if(cosOut > 0.0f) {
					emission = v.mat.radiance;
					if(nonzero(emission)) connectPdf = light_pdfs(S, v.inst, v.prim, v.surfaceParams, lastPosition).connect;
				}
			}
			if(nonzero(emission) && pathLen > 1) {
				const float misWeight = 1.0f / (1.0f + float(P.neeCount) * (connectPdf / v.incidentPdf));
				emission = emission * misWeight;
			}
			radiance = contribute(radiance, throughput * emission);
			if(adj) adj->vertex(S, contribute(V3{ 0, 0, 0 }, throughput * emission), v.type == V_SURFACE, v.mat.type, vMat, vUv, v.mat.albedo);
			if(aux) {
				// pt_common.hpp:146-152: position, incident distance, shading normal, uv, albedo
				// (Lambert and Torrance; 0 for emitters) and lightness, each times the guide weight
				const bool surf = v.type == V_SURFACE;
				const V3 pos = surf ? v.position : V3{ 0, 0, 0 };
				const V3 nrm = surf ? v.ts.shadingN : V3{ 0, 0, 0 };
				const V3 alb = surf && v.mat.type != OR_MAT_EMISSIVE ? v.mat.albedo : V3{ 0, 0, 0 };
				const float depth = surf ? std::fabs(v.incidentEncoded.z) : 0.0f;
				const V2 uv = surf ? vUv : V2{ 0, 0 };
				aux_add(AUX_POS, guideWeight * pos.x); aux_add(AUX_POS + 1, guideWeight * pos.y); aux_add(AUX_POS + 2, guideWeight * pos.z);
				aux_add(AUX_DEPTH, guideWeight * depth);
				aux_add(AUX_NORMAL, guideWeight * nrm.x); aux_add(AUX_NORMAL + 1, guideWeight * nrm.y); aux_add(AUX_NORMAL + 2, guideWeight * nrm.z);
				aux_add(AUX_UV, guideWeight * uv.x); aux_add(AUX_UV + 1, guideWeight * uv.y);
				aux_add(AUX_ALBEDO, guideWeight * alb.x); aux_add(AUX_ALBEDO + 1, guideWeight * alb.y); aux_add(AUX_ALBEDO + 2, guideWeight * alb.z);
				aux_add(AUX_LIGHT, guideWeight * avg3(emission));
			}
		} else if(adj) {
			adj->vertex(S, V3{ 0, 0, 0 }, v.type == V_SURFACE, v.mat.type, vMat, vUv, v.mat.albedo);
		}
		if(v.type != V_SURFACE) break;
	} while(pathLen < P.maxPathLength);
	radianceOut = radiance;
	hitOut = hitAcc;
}

void AlbedoAdjoint::vertex(const Scene& S, const V3& e, bool surface, i32 type, i32 mat, V2 uv, V3 albedo) {
	add_all(e);
	if(surface && type == OR_MAT_EMISSIVE) emitted(e, mat);
	if(texIndex < 0 || !surface || type != OR_MAT_LAMBERT || n >= 64 || mat < 0 || S.materials[size_t(mat)].albedoTex != texIndex) return;
	const Texture& t = S.textures[size_t(texIndex)];
	const float fx = uv.x - std::floor(uv.x), fy = uv.y - std::floor(uv.y);
	i32 x = i32(fx * float(t.w)), y = i32(fy * float(t.h));
	if(x >= i32(t.w)) x = i32(t.w) - 1;
	if(y >= i32(t.h)) y = i32(t.h) - 1;
	texel[n] = y * i32(t.w) + x;
	alb[n][0] = albedo.x; alb[n][1] = albedo.y; alb[n][2] = albedo.z;
	suf[n][0] = suf[n][1] = suf[n][2] = 0.0;
	++n;
}

void pt_iterate(PtState& st, int numThreads, u32 y0, u32 y1, bool accumulate) {
	const Scene& S = *st.scene;
	const i32 W = i32(S.width), H = i32(S.height);
	if(accumulate) ++st.iteration;
	const float it = float(st.iteration);
	const i32 p0 = i32(y0) * W, p1 = i32(y1) * W;
	(void)H;
	Counters total;
#pragma omp parallel num_threads(numThreads)
	{
		Counters local;
#pragma omp for schedule(static, 1000)
		for(i32 pixel = p0; pixel < p1; ++pixel) {
			V3 rad; V2 hid;
			float aux[AUX_CHANNELS] = {};
			pt_sample(st, pixel % W, pixel / W, st.rngs[pixel], rad, hid, local, nullptr, aux);
			if(accumulate) {
				const float iter[5] = { rad.x, rad.y, rad.z, hid.x, hid.y };
				for(int c = 0; c < 3; ++c)
					update_moments(iter[c], st.radiance[size_t(pixel) * 3 + size_t(c)], st.radianceVar[size_t(pixel) * 3 + size_t(c)], it);
				for(int c = 0; c < 2; ++c)
					update_moments(iter[3 + c], st.hitId[size_t(pixel) * 2 + size_t(c)], st.hitIdVar[size_t(pixel) * 2 + size_t(c)], it);
				for(int c = 0; c < AUX_CHANNELS; ++c)
					update_moments(aux[c], st.aux[size_t(pixel) * AUX_CHANNELS + size_t(c)],
					               st.auxVar[size_t(pixel) * AUX_CHANNELS + size_t(c)], it);
			}
		}
#pragma omp critical
		total.add(local);
	}
	st.stats.add(total);
}

// ---------------------------------------------------------------- light tracer
enum LtKind { LV_POINT, LV_AREA, LV_SURFACE, LV_ENV };

// A photon's start on a light (light_sampling.hpp:20-49 Emitter): the
// position, the intensity divided by the probability of choosing the light
// (light_tree_sampling.hpp:12-16) and, for an area light, its normal; for
// the environment, the direction the photon travels (in `normal`) and the
// irradiance.
struct Emitter { V3 position, intensity, normal; LtKind kind; bool valid; float pChoice, pdf; };

// A vector perpendicular to n (not normalised): n crossed with the coordinate
// axis of n's smallest component. The reference takes `perpendicular` from
// its math library (epsilon, absent); the emission lobe it orients is
// rotationally symmetric about n, so the choice of axis changes which
// direction a random number pair maps to, not the image's expectation.
inline V3 perpendicular(V3 n) {
	const float ax = std::fabs(n.x), ay = std::fabs(n.y), az = std::fabs(n.z);
	if(ax <= ay && ax <= az) return { 0.0f, n.z, -n.y };
	if(ay <= az) return { -n.z, 0.0f, n.x };
	return { n.y, -n.x, 0.0f };
}

// light_sampling.hpp:80-84 (point), 117-140 (triangle), 143-171 (quad), 173-194 (sphere)
Emitter sample_light_pos(const Scene& S, const PosLight& l, float u0, float u1, float lightProb) {
	Emitter e{};
	e.valid = true;
	if(l.type == LT_POINT) {
		e.position = l.position;
		e.intensity = l.intensity / lightProb;
		e.normal = { 0, 0, 0 };
		e.kind = LV_POINT;
		e.pChoice = lightProb;
		e.pdf = INF_PDF;
		return e;
	}
	const Material& m = S.materials[l.material];
	const V3 radiance = m.type == OR_MAT_EMISSIVE ? m.radiance * m.scale : V3{ 0, 0, 0 };
	if(l.type == LT_SPHERE) {
		// light_sampling.hpp:173-194: a uniformly chosen point of the sphere,
		// its area pdf the direction pdf 1 / (4 pi) over r^2
		const float r = l.radius;
		const V3 normal = sample_dir_sphere_uniform(u0, u1);
		const float area = ((4.0f * PI) * r) * r;
		e.position = l.position + normal * r;
		e.intensity = (radiance * area) / lightProb;
		e.normal = normal;
		e.kind = LV_AREA;
		e.pChoice = lightProb;
		e.pdf = ((1.0f / (4.0f * PI)) * 1.0f) / (r * r);
		return e;
	}
	V3 normal, position;
	float area;
	if(l.type == LT_TRI) {
		normal = cross(l.posV[1], l.posV[2]);
		const float area2 = len(normal);
		normal = normal / area2;
		area = area2 * 0.5f;
		const float bs = 1.0f - mbmath::sqrt(1.0f - u0);
		const float bt = (1.0f - bs) * u1;
		position = (l.posV[0] + l.posV[1] * bs) + l.posV[2] * bt;
	} else {
		const V3 tx = l.posV[1] + u0 * l.posV[3];
		const V3 ty = l.posV[2] + u1 * l.posV[3];
		normal = cross(ty, tx);
		area = len(normal);
		normal = normal / area;
		position = (l.posV[0] + tx * u1) + l.posV[2] * u0;
	}
	e.position = position;
	e.intensity = (radiance * area) / lightProb;
	e.normal = normal;
	e.kind = LV_AREA;
	e.pChoice = lightProb;
	e.pdf = 1.0f / area;
	return e;
}

// light_sampling.hpp:226-232 and 292-306 (a colored background), scaled by
// the environment's choice probability (light_tree_sampling.hpp:158-167): a
// direction drawn uniformly on the sphere; the photon travels against it.
Emitter sample_background(const LightTree& T, float u0, float u1, float envProb) {
	const V3 dir = sample_dir_sphere_uniform(u0, u1);
	const float dirPdf = 1.0f / (4.0f * PI);
	const V3 irradiance = (T.bgColor * T.bgScale) / dirPdf;
	Emitter e{};
	e.valid = true;
	e.kind = LV_ENV;
	e.position = { 0, 0, 0 };
	e.normal = -dir;
	e.intensity = irradiance / envProb;
	e.pChoice = envProb;
	e.pdf = dirPdf;
	return e;
}

// math/sampling.hpp:132-158: a start point for a photon of direction dir on
// the faces of the scene box it enters through, and the inverse of the
// box's projected area (the position pdf).
V3 sample_position(const Box& b, V3 dir, float u0, float u1, float& pdf) {
	const V3 sides = b.mx - b.mn;
	const float projAx = (sides.y * sides.z) * std::fabs(dir.x);
	const float projAy = (sides.x * sides.z) * std::fabs(dir.y);
	const float projAz = (sides.x * sides.y) * std::fabs(dir.z);
	const float area = (projAx + projAy) + projAz;
	float x = u0 * area;
	V3 p;
	if(x < projAx) {
		x = (x - 0.0f) / (projAx - 0.0f);
		p = { dir.x < 0.0f ? 1.0f : 0.0f, u1, x };
	} else if(x < projAx + projAy) {
		x = (x - projAx) / ((projAx + projAy) - projAx);
		p = { u1, dir.y < 0.0f ? 1.0f : 0.0f, x };
	} else {
		x = (x - (projAx + projAy)) / (area - (projAx + projAy));
		p = { u1, x, dir.z < 0.0f ? 1.0f : 0.0f };
	}
	pdf = 1.0f / area;
	return (b.mn + p * sides) - dir * 1e-3f;
}

// light_tree_sampling.hpp:141-188 with the sub-tree descent of :81-131. The
// photon index spreads the photons over the flux interval before the seed's
// random offset. There are no directional lights.
Emitter lights_emit(const Scene& S, u64 index, u64 numIndices, u64 seed, float u0, float u1) {
	const LightTree& T = S.lightTree;
	u64 rndChoice = numIndices > 0 ? seed + index * (~0ull / numIndices) : seed;
	if(rndChoice == ~0ull) --rndChoice;
	const float bgSum = (T.bgFlux.x + T.bgFlux.y) + T.bgFlux.z;
	const float fluxSum = (bgSum + T.dirFlux) + T.rootFlux;
	Emitter none{};
	none.valid = false;
	if(!(fluxSum > 0.0f)) return none;
	const float envProb = bgSum / fluxSum;
	const float dirProb = T.dirFlux / fluxSum;
	const float posProb = T.rootFlux / fluxSum;
	if(rndChoice < percentage_of(~0ull, envProb)) return sample_background(T, u0, u1, envProb);
	const u64 right = percentage_of(~0ull, envProb + dirProb);
	if(rndChoice < right) return none;
	u64 iL = right, iR = ~0ull;
	float lightProb = posProb;
	u16 type = T.rootType;
	i32 idx = T.rootIndex;
	i32 nodeIdx = 0;
	while(type == INTERNAL_NODE) {
		const LightNode& nd = T.nodes[nodeIdx];
		const float probLeft = nd.left.flux / (nd.left.flux + nd.right.flux);
		const u64 boundary = iL + percentage_of(iR - iL, probLeft);
		if(rndChoice < boundary) { type = nd.left.type; idx = nd.left.index; iR = boundary; lightProb *= probLeft; }
		else { type = nd.right.type; idx = nd.right.index; iL = boundary; lightProb *= (1.0f - probLeft); }
		nodeIdx = idx;
	}
	return sample_light_pos(S, T.lights[idx], u0, u1, lightProb);
}

// pinhole.hpp:86-116: the pixel a direction leaving the camera falls in and
// the sensor response w (equal to the sampling pdf); false when the direction
// points behind the camera or off the image.
inline bool pinhole_project(const Camera& c, V3 excident, i32& px, i32& py, float& w) {
	const float cosOut = dot(c.viewDir, excident);
	if(cosOut < 0.0f) return false;
	const V3 xAxis = cross(c.viewDir, c.up);
	const float d = cosOut * c.tanVFov;
	float ux = dot(xAxis, excident) / d;
	const float uy = dot(c.up, excident) / d;
	const float aspect = float(c.resX) / float(c.resY);
	ux = ux / aspect;
	if(!(ux > -1.0f && ux <= 1.0f && uy > -1.0f && uy <= 1.0f)) return false;
	px = i32(std::floor((ux * 0.5f + 0.5f) * float(c.resX)));
	py = i32(std::floor((uy * 0.5f + 0.5f) * float(c.resY)));
	if(px >= i32(c.resX)) px = i32(c.resX) - 1;
	if(py >= i32(c.resY)) py = i32(c.resY) - 1;
	const float t2 = 2.0f * c.tanVFov;
	const float pixelArea = (t2 * t2) * aspect;
	w = 1.0f / (((pixelArea * cosOut) * cosOut) * cosOut);
	return true;
}

inline V3 decode_incident(V3 e) {
	float t = 1.0f - e.x * e.x - e.y * e.y;
	t = std::fmin(std::fmax(t, 0.0f), 1.0f);
	return { e.x, e.y, sgn(e.z) * mbmath::sqrt(t) };
}

struct LtState {
	const Scene* scene;
	OrLtParams params;
	std::vector<Pcg64> rngs;
	std::vector<float> radiance, lightness, density; // cumulative means (density: the last iteration's)
	std::vector<float> radianceVar, lightnessVar, densityMean; // variances (density: its running mean)
	std::vector<i32> recPixel;   // last iteration, per photon and path length: pixel or -1
	std::vector<float> recValue; // ... radiance rgb, lightness, density as added
	i32 iteration = -1;
	Counters stats;
};

// lt_common.hpp:19-77: one photon's random walk from a light, every vertex
// (the light vertex included) connected to the camera. The connections are
// written to rec (one slot per path length).
void lt_sample(const LtState& st, u32 photon, u32 numPhotons, Pcg64& rng, i32* recPixel, float* recValue, Counters& cnt) {
	const Scene& S = *st.scene;
	const OrLtParams& P = st.params;
	V3 throughput = { 1, 1, 1 };
	const u64 r0 = rng.next();
	const float su0 = sample_uniform(u32(r0)), su1 = sample_uniform(u32(r0 >> 32));
	const u64 treeSeed = rng.next();
	const Emitter em = lights_emit(S, photon, numPhotons, treeSeed, su0, su1);
	(void)rng.next(); // create_camera consumes one number (unused by the pinhole camera)
	if(!em.valid) return;
	LtKind kind = em.kind;
	V3 position = em.position;
	const V3 normal = em.normal, intensity = em.intensity;
	TangentSpace ts{};
	Params mat{};
	V3 incEnc = { 0, 0, 0 };
	const V3 camPos = S.cam.position;
	i32 pathLen = 0;
	do {
		if(pathLen + 1 >= P.minPathLength && pathLen + 1 <= P.maxPathLength) {
			// get_connection(camera, vertex) (path_util.hpp:384-403); an
			// environment vertex has no position: the connection is its
			// direction at distance 1
			V3 dir;
			float distSq;
			if(kind == LV_ENV) {
				dir = -normal;
				distSq = 1.0f;
			} else {
				const V3 c = position - camPos;
				distSq = lensq(c);
				const float dist = mbmath::sqrt(distSq);
				dir = { sdiv(c.x, dist), sdiv(c.y, dist), sdiv(c.z, dist) };
			}
			i32 px = -1, py = -1;
			float w = 0.0f;
			if(pinhole_project(S.cam, dir, px, py, w)) {
				// vertex.evaluate(-dir, adjoint) (path_util.hpp:245-293, lights.hpp:263-293)
				const V3 ex = -dir;
				V3 lvalue = { 0, 0, 0 };
				float lcos = 0.0f;
				if(kind == LV_POINT || kind == LV_ENV) { lvalue = intensity; lcos = 1.0f; }
				else if(kind == LV_AREA) { const float co = dot(normal, ex); if(co > 0.0f) { lvalue = intensity; lcos = co; } }
				else { const EvalValue ev = material_evaluate(ts, mat, decode_incident(incEnc), ex, true); lvalue = ev.value; lcos = ev.cosOut; }
				V3 bxdfProd = V3{ w, w, w } * lvalue;
				const float cosProd = 1.0f * lcos;
				if(P.density || (any_pos(bxdfProd) && cosProd > 0.0f)) {
					const V3 vGeo = kind == LV_SURFACE ? ts.geoN : (kind == LV_AREA ? normal : V3{ 0, 0, 0 });
					// the environment vertex is placed the maximum scene size away (path_util.hpp:130-137)
					const V3 vpos = kind == LV_ENV ? camPos - decode_incident(normal) * MAX_SCENE_SIZE : position;
					if(!any_intersection(S, camPos, vpos, V3{ 0, 0, 0 }, vGeo, dir, cnt)) {
						bxdfProd = bxdfProd / distSq;
						const V3 rad = (throughput * cosProd) * bxdfProd;
						const float light = (((throughput.x + throughput.y) + throughput.z) / 3.0f) * cosProd;
						float dens = 0.0f;
						if(P.density) {
							dens = (w * 1.0f) / distSq;
							const float gf = kind == LV_SURFACE ? dot(dir, ts.shadingN)
							               : kind == LV_AREA ? dot(dir, normal) : kind == LV_ENV ? 1.0f : 0.0f;
							dens *= std::fabs(gf);
						}
						recPixel[pathLen] = py * i32(S.width) + px;
						float* v = recValue + 5 * size_t(pathLen);
						v[0] = nan_to_zero(rad.x); v[1] = nan_to_zero(rad.y); v[2] = nan_to_zero(rad.z);
						v[3] = nan_to_zero(light);
						v[4] = nan_to_zero(dens);
					}
				}
			}
		}
		// walk (random_walk.hpp:38-113), Russian roulette always on
		const u64 x0 = rng.next(), x1 = rng.next();
		const float ru0 = sample_uniform(u32(x0)), ru1 = sample_uniform(u32(x0 >> 32));
		const float rr = sample_uniform(u32(rng.next()));
		V3 excident, sThroughput;
		V3 start = position;
		if(kind == LV_POINT) {
			// sample_light_dir_point (light_sampling.hpp:85-89)
			excident = sample_dir_sphere_uniform(ru0, ru1);
			sThroughput = (intensity * 4.0f) * PI;
		} else if(kind == LV_AREA) {
			// sample_light_dir_area (light_sampling.hpp:197-210)
			float cosT;
			const V3 d = sample_dir_cosine(ru0, ru1, cosT);
			const V3 tx = normalize(perpendicular(normal));
			const V3 ty = cross(normal, tx);
			excident = (d.x * tx + d.y * ty) + d.z * normal;
			sThroughput = intensity * PI;
		} else if(kind == LV_ENV) {
			// path_util.hpp:312-320: a start point on the scene box, travelling along the photon's direction
			float pdf;
			start = sample_position(S.aabb, normal, ru0, ru1, pdf);
			excident = normal;
			sThroughput = intensity / pdf;
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
		const V3 geoN = kind == LV_SURFACE ? ts.geoN : (kind == LV_AREA ? normal : V3{ 0, 0, 0 });
		V3 origin = start;
		const Intersection hit = first_intersection(S, origin, excident, geoN, MAX_SCENE_SIZE, cnt);
		if(hit.inst < 0) break;
		position = origin + excident * hit.distance;
		ts = tangent_space(S, hit);
		mat = fetch_material(S, material_index(S, hit.inst, hit.prim), hit.uv);
		incEnc = { excident.x, excident.y, hit.distance * sgn(excident.z) };
		kind = LV_SURFACE;
		++pathLen;
	} while(pathLen < P.maxPathLength);
}

// cpu_lt.cpp:18-39: one photon per pixel index per iteration. The terms are
// added to the iteration buffer in photon order, then the running means are
// updated (output_handler_variance.hpp:7-31).
void lt_iterate(LtState& st, int numThreads) {
	const Scene& S = *st.scene;
	const u32 n = S.width * S.height;
	const size_t maxL = size_t(std::max(1, st.params.maxPathLength));
	++st.iteration;
	st.recPixel.assign(size_t(n) * maxL, -1);
	st.recValue.assign(size_t(n) * maxL * 5, 0.0f);
	Counters total;
#pragma omp parallel num_threads(numThreads)
	{
		Counters local;
#pragma omp for schedule(dynamic, 256)
		for(i32 photon = 0; photon < i32(n); ++photon)
			lt_sample(st, u32(photon), n, st.rngs[size_t(photon)], &st.recPixel[size_t(photon) * maxL],
			          &st.recValue[size_t(photon) * maxL * 5], local);
#pragma omp critical
		total.add(local);
	}
	st.stats.add(total);
	std::vector<float> iter(size_t(n) * 5, 0.0f);
	for(size_t k = 0; k < st.recPixel.size(); ++k) {
		if(st.recPixel[k] < 0) continue;
		float* d = &iter[size_t(st.recPixel[k]) * 5];
		for(int c = 0; c < 5; ++c) d[c] += st.recValue[5 * k + size_t(c)];
	}
	const float itf = float(st.iteration);
	for(size_t p = 0; p < n; ++p) {
		for(int c = 0; c < 3; ++c) update_moments(iter[5 * p + size_t(c)], st.radiance[3 * p + size_t(c)], st.radianceVar[3 * p + size_t(c)], itf);
		update_moments(iter[5 * p + 3], st.lightness[p], st.lightnessVar[p], itf);
		update_reduced(iter[5 * p + 4], st.density[p], st.densityMean[p], itf);
	}
}

// ---------------------------------------------------------------- bidirectional path tracer
// cpu_bpt.cpp:1-247 with the vertex machinery of path_util.hpp it uses. A
// vertex keeps what the reference's PathVertex<BptVertexExt> keeps: its kind,
// position, encoded incident direction (surfaces: x, y of the direction and
// the distance with the sign of z; a miss: the direction; an area light: its
// normal; a point light: its intensity; the environment: the photon's
// direction), surface data, and the MIS extension (incident area pdf, cached
// sum of relative probabilities of the earlier events, subpath throughput).
enum BKind { BV_VIRTUAL, BV_CAMERA, BV_SURFACE, BV_VOID, BV_POINT, BV_AREA, BV_ENV };

struct BVertex {
	BKind kind;
	V3 position;
	V3 incEnc;
	V3 intensity;       // area light intensity / environment irradiance
	float projSceneArea; // environment
	TangentSpace ts;
	Params mat;
	i32 inst, prim;
	V2 sp;
	i32 prev;           // index of the previous vertex in its subpath, or -1
	float incidentPdf;  // BptVertexExt::incidentPdf
	float prevRelSum;   // BptVertexExt::prevRelativeProbabilitySum
	V3 throughput;      // BptVertexExt::throughput
	i32 pathLen;        // PathVertex::m_pathLen
	float prevConv;     // VcmVertexExt::prevConversionFactor
};

inline bool bv_ortho(BKind k) { return k == BV_VOID || k == BV_ENV; }           // path_util.hpp:41-46
inline bool bv_camera(BKind k) { return k == BV_CAMERA; }
inline bool bv_end(BKind k) { return k != BV_SURFACE; }                          // path_util.hpp:33-35

// path_util.hpp:160-176
inline float bv_geo_factor(const BVertex& v, V3 dir) {
	if(v.kind == BV_AREA) return dot(dir, v.incEnc);
	if(v.kind == BV_SURFACE) return dot(dir, v.ts.shadingN);
	if(v.kind == BV_ENV || v.kind == BV_VOID) return 1.0f;
	return 0.0f;
}
inline V3 bv_geo_normal(const BVertex& v) {
	if(v.kind == BV_AREA) return v.incEnc;
	if(v.kind == BV_SURFACE) return v.ts.geoN;
	return { 0, 0, 0 };
}
inline V3 bv_incident_dir(const BVertex& v) { return decode_incident(v.incEnc); }
inline float bv_incident_dist_sq(const BVertex& v) { return bv_end(v.kind) ? 0.0f : v.incEnc.z * v.incEnc.z; }
// path_util.hpp:130-137
inline V3 bv_position(const BVertex& v, V3 ref) {
	if(v.kind == BV_ENV) return ref - bv_incident_dir(v) * MAX_SCENE_SIZE;
	return v.position;
}
// path_util.hpp:208-221: a sampling pdf converted into an area pdf at v
inline float bv_convert_pdf(const BVertex& v, BKind source, float samplePdf, V3 dir, float distSq) {
	if(source == BV_VIRTUAL) return samplePdf;
	const float geo = bv_geo_factor(v, dir);
	if(bv_ortho(source) || bv_ortho(v.kind)) return samplePdf * std::fabs(geo);
	return samplePdf * std::fabs(geo) / distSq;
}

// path_util.hpp:245-293: value, cosine and pdfs of leaving v along excident;
// a camera also yields the pixel (-1 off the image)
EvalValue bv_evaluate(const Scene& S, const BVertex& v, V3 excident, bool adjoint, i32& px, i32& py) {
	EvalValue none = { { 0, 0, 0 }, 0, 0, 0 };
	switch(v.kind) {
		case BV_POINT: return { v.incEnc, 1.0f, 1.0f / (4.0f * PI), 0.0f };
		case BV_AREA: {
			const float cosOut = dot(v.incEnc, excident);
			if(cosOut <= 0.0f) return none;
			return { v.intensity, cosOut, cosOut / PI, 0.0f };
		}
		case BV_ENV: return { v.intensity, 1.0f, 1.0f / v.projSceneArea, 0.0f };
		case BV_CAMERA: {
			float w = 0.0f;
			if(!pinhole_project(S.cam, excident, px, py, w)) { px = -1; py = -1; return { { 0, 0, 0 }, 1.0f, 0.0f, 0.0f }; }
			return { { w, w, w }, 1.0f, w, 0.0f };
		}
		case BV_SURFACE: return material_evaluate(v.ts, v.mat, bv_incident_dir(v), excident, adjoint);
		default: return none;
	}
}

// cpu_bpt.cpp:68-88
float bpt_mis_part(const std::vector<BVertex>& path, const BVertex& v, float vertexPdfBack, float nextPdfBack,
                   BKind nextType, V3 dir, float distSq) {
	float reversePdf = bv_convert_pdf(v, nextType, nextPdfBack, dir, distSq);
	const float relPdf = reversePdf / v.incidentPdf;
	if(v.prev >= 0) {
		const BVertex& p = path[size_t(v.prev)];
		reversePdf = bv_convert_pdf(p, v.kind, vertexPdfBack, bv_incident_dir(v), bv_incident_dist_sq(v));
		const float prevRelPdf = reversePdf / p.incidentPdf;
		return relPdf + relPdf * (prevRelPdf + prevRelPdf * p.prevRelSum);
	}
	return relPdf;
}

struct BptState {
	const Scene* scene;
	OrLtParams params;
	std::vector<Pcg64> rngs;
	std::vector<float> radiance, lightness; // cumulative means
	std::vector<float> radianceVar, lightnessVar;
	std::vector<i32> recPixel;               // last iteration, per pixel: connections [view length][light index], then hits [view length]
	std::vector<float> recValue;             // radiance rgb, lightness as added
	i32 iteration = -1;
	Counters stats;
};

inline size_t bpt_slots(i32 maxPath) { return size_t(maxPath) * size_t(maxPath) + size_t(maxPath); }

inline bool bv_hitable(BKind k) { return k == BV_SURFACE || k == BV_AREA || k == BV_ENV || k == BV_VOID; } // path_util.hpp:53-58

// cpu_vcm.cpp:21-32: the relative probabilities of the events before v
// (connections and merges) for the reverse sampling pdf pdfBack at v.
float vcm_prev_rel_sum(const std::vector<BVertex>& path, const BVertex& v, float pdfBack, float nPhotons, float area) {
	if(v.prev < 0) return 0.0f;
	const BVertex& p = path[size_t(v.prev)];
	const float pdfBackA = pdfBack * v.prevConv;
	const float relMerge = p.prev >= 0 ? pdfBackA * nPhotons * area : 0.0f; // no merges at start points
	const float relConn = pdfBackA / p.incidentPdf;
	return relConn + relMerge + relConn * p.prevRelSum;
}

// random_walk.hpp:38-113 for a BPT vertex: samples v (updating its MIS
// extension), applies Russian roulette and traces; out gets the next vertex.
// Returns 0: cancelled, 1: hit, 2: miss (out is a void vertex).
// vcm: null for the bidirectional path tracer; for vertex connection and
// merging the number of light subpaths and the merge area (VcmVertexExt's
// updates, cpu_vcm.cpp:117-146).
int bpt_walk(const Scene& S, std::vector<BVertex>& path, i32 vi, const OrLtParams& P, i32 px, i32 py, Pcg64& rng,
             bool adjoint, V3& throughput, BVertex& out, Counters& cnt, const float* vcm = nullptr) {
	BVertex& v = path[size_t(vi)];
	const u64 x0 = rng.next(), x1 = rng.next();
	const float ru0 = sample_uniform(u32(x0)), ru1 = sample_uniform(u32(x0 >> 32));
	const float rr = sample_uniform(u32(rng.next()));
	(void)P;
	V3 excident, sThroughput, origin = v.position;
	float pdfF = 0.0f, pdfB = 0.0f;
	switch(v.kind) {
		case BV_POINT:
			excident = sample_dir_sphere_uniform(ru0, ru1);
			sThroughput = (v.incEnc * 4.0f) * PI;
			pdfF = 1.0f / (4.0f * PI);
			break;
		case BV_AREA: {
			float cosT;
			const V3 d = sample_dir_cosine(ru0, ru1, cosT);
			const V3 tx = normalize(perpendicular(v.incEnc));
			const V3 ty = cross(v.incEnc, tx);
			excident = (d.x * tx + d.y * ty) + d.z * v.incEnc;
			sThroughput = v.intensity * PI;
			pdfF = d.z / PI;
			break;
		}
		case BV_ENV: {
			float pdf;
			origin = sample_position(S.aabb, v.incEnc, ru0, ru1, pdf);
			excident = v.incEnc;
			sThroughput = v.intensity / pdf;
			pdfF = pdf;
			break;
		}
		case BV_CAMERA:
			excident = pinhole_ray(S.cam, px, py, ru0, ru1, pdfF);
			sThroughput = { 1, 1, 1 };
			break;
		case BV_SURFACE: {
			const PathSample smp = material_sample(v.ts, v.mat, bv_incident_dir(v), ru0, ru1, x1, adjoint);
			if(!smp.valid) { throughput = { 0, 0, 0 }; return 0; }
			excident = smp.excident;
			sThroughput = smp.throughput;
			pdfF = smp.pdfF;
			pdfB = smp.pdfB;
			break;
		}
		default: return 0;
	}
	// BptVertexExt::update after sampling (cpu_bpt.cpp:49-58), or VcmVertexExt's
	if(vcm) v.prevRelSum = vcm_prev_rel_sum(path, v, pdfB, vcm[0], vcm[1]);
	else if(v.prev >= 0) {
		const BVertex& p = path[size_t(v.prev)];
		const float prevReversePdf = bv_convert_pdf(p, v.kind, pdfB, bv_incident_dir(v), bv_incident_dist_sq(v));
		const float relToPrev = prevReversePdf / p.incidentPdf;
		v.prevRelSum = relToPrev + relToPrev * p.prevRelSum;
	}
	throughput = throughput * sThroughput;
	const float cp = fmin_(maxc(throughput) + 0.1f, 1.0f);
	if(rr >= cp) { throughput = { 0, 0, 0 }; return 0; }
	throughput = throughput / cp;
	const Intersection hit = first_intersection(S, origin, excident, bv_geo_normal(v), MAX_SCENE_SIZE, cnt);
	out = BVertex{};
	out.prev = vi;
	out.pathLen = v.pathLen + 1;
	out.prevRelSum = 0.0f;
	out.inst = out.prim = -1;
	if(hit.inst < 0) {
		out.kind = BV_VOID;
		out.position = { 0, 0, 0 };
		out.incEnc = excident;
	} else {
		out.kind = BV_SURFACE;
		out.position = origin + excident * hit.distance;
		out.incEnc = { excident.x, excident.y, hit.distance * sgn(excident.z) };
		out.ts = tangent_space(S, hit);
		out.inst = hit.inst;
		out.prim = hit.prim;
		out.sp = hit.sp;
		out.mat = fetch_material(S, material_index(S, hit.inst, hit.prim), hit.uv);
	}
	// BptVertexExt::update after the segment (cpu_bpt.cpp:36-47)
	const float inCosAbs = std::fabs(bv_geo_factor(out, excident));
	const bool ortho = bv_ortho(v.kind) || bv_ortho(out.kind);
	out.incidentPdf = ortho ? pdfF * inCosAbs : pdfF * std::fabs(inCosAbs) / (hit.distance * hit.distance);
	out.throughput = throughput;
	if(vcm && bv_hitable(v.kind)) {
		const float outCosAbs = std::fabs(bv_geo_factor(v, excident));
		out.prevConv = ortho ? outCosAbs : outCosAbs / (hit.distance * hit.distance);
	}
	return hit.inst < 0 ? 2 : 1;
}

// cpu_bpt.cpp:170-232: one light subpath and one view subpath for a pixel,
// every view vertex connected to every light vertex, random emitter hits
// weighted by the balance heuristic.
void bpt_sample(const BptState& st, i32 px, i32 py, u32 idx, u32 numPixels, Pcg64& rng, i32* recPixel, float* recValue,
                Counters& cnt) {
	const Scene& S = *st.scene;
	const OrLtParams& P = st.params;
	const i32 maxP = std::max(1, P.maxPathLength);
	const i32 pixel = py * i32(S.width) + px;
	std::vector<BVertex> lpath(size_t(maxP) + 1), vpath(size_t(maxP) + 1);
	// light subpath
	const u64 r0 = rng.next();
	const float su0 = sample_uniform(u32(r0)), su1 = sample_uniform(u32(r0 >> 32));
	const u64 treeSeed = rng.next();
	const Emitter em = lights_emit(S, idx, numPixels, treeSeed, su0, su1);
	i32 lightPathLen = -1;
	if(em.valid) {
		BVertex& l0 = lpath[0];
		l0 = BVertex{};
		l0.prev = -1;
		l0.position = em.position;
		l0.throughput = { 1, 1, 1 };
		l0.prevRelSum = 0.0f;
		if(em.kind == LV_POINT) { l0.kind = BV_POINT; l0.incEnc = em.intensity; l0.incidentPdf = em.pChoice; }
		else if(em.kind == LV_AREA) { l0.kind = BV_AREA; l0.incEnc = em.normal; l0.intensity = em.intensity; l0.incidentPdf = em.pdf * em.pChoice; }
		else {
			l0.kind = BV_ENV; l0.incEnc = em.normal; l0.intensity = em.intensity; l0.incidentPdf = em.pdf * em.pChoice;
			l0.position = { 0, 0, 0 };
			l0.projSceneArea = projected_area(-em.normal, S.aabb);
		}
		lightPathLen = 0;
		V3 thr = { 1, 1, 1 };
		if(maxP > 1) do {
			if(bpt_walk(S, lpath, lightPathLen, P, px, py, rng, true, thr, lpath[size_t(lightPathLen) + 1], cnt) != 1) break;
			++lightPathLen;
		} while(lightPathLen < maxP - 1);
	}
	// view subpath
	BVertex& c = vpath[0];
	c = BVertex{};
	c.kind = BV_CAMERA;
	c.prev = -1;
	c.position = S.cam.position;
	c.incEnc = { float(px), float(py), 0.0f };
	c.incidentPdf = 1.0f;
	c.prevRelSum = 0.0f;
	c.throughput = { 1, 1, 1 };
	(void)rng.next(); // create_camera consumes one number (unused by the pinhole camera)
	V3 throughput = { 1, 1, 1 };
	i32 viewPathLen = 0;
	const size_t hitBase = size_t(maxP) * size_t(maxP);
	do {
		const BVertex& v = vpath[size_t(viewPathLen)];
		const i32 maxL = std::min(lightPathLen + 1, maxP - viewPathLen);
		for(i32 l = std::max(0, P.minPathLength - viewPathLen - 1); l < maxL; ++l) {
			const BVertex& w = lpath[size_t(l)];
			// connect (cpu_bpt.cpp:120-148)
			i32 ox = px, oy = py;
			V3 bxdfs = { 0, 0, 0 };
			float cosines = 0.0f;
			if(!((bv_ortho(v.kind) && bv_ortho(w.kind)) || (bv_ortho(v.kind) && bv_camera(w.kind)) ||
			     (bv_camera(v.kind) && bv_ortho(w.kind)))) {
				V3 dir, v0;
				float distSq;
				if(bv_ortho(w.kind)) { dir = -w.incEnc; distSq = 1.0f; v0 = v.position; }
				else {
					const V3 cv = w.position - v.position;
					distSq = lensq(cv);
					const float dist = mbmath::sqrt(distSq);
					dir = { sdiv(cv.x, dist), sdiv(cv.y, dist), sdiv(cv.z, dist) };
					v0 = v.position;
				}
				const EvalValue val0 = bv_evaluate(S, v, dir, false, ox, oy);
				const EvalValue val1 = bv_evaluate(S, w, -dir, true, ox, oy);
				if(ox != -1) {
					const V3 bxdfProd = val0.value * val1.value;
					const float cosProd = val0.cosOut * val1.cosOut;
					if(any_pos(bxdfProd) && cosProd > 0.0f &&
					   !any_intersection(S, v0, bv_position(w, v0), bv_geo_normal(v), bv_geo_normal(w), dir, cnt)) {
						const float rp0 = bpt_mis_part(vpath, v, val0.pdfB, val1.pdfF, w.kind, dir, distSq);
						const float rp1 = bpt_mis_part(lpath, w, val1.pdfB, val0.pdfF, v.kind, dir, distSq);
						const float mis = 1.0f / ((1.0f + rp0) + rp1);
						bxdfs = bxdfProd * (mis / distSq);
						cosines = cosProd;
					}
				}
			}
			if(ox != -1) {
				const V3 full = throughput * w.throughput;
				const V3 rad = (full * cosines) * bxdfs;
				const float light = (((full.x + full.y) + full.z) / 3.0f) * cosines;
				const size_t slot = size_t(viewPathLen) * size_t(maxP) + size_t(l);
				recPixel[slot] = oy * i32(S.width) + ox;
				float* o = recValue + 4 * slot;
				o[0] = nan_to_zero(rad.x); o[1] = nan_to_zero(rad.y); o[2] = nan_to_zero(rad.z); o[3] = nan_to_zero(light);
			}
		}
		// walk (view subpath, not adjoint)
		const i32 r = bpt_walk(S, vpath, viewPathLen, P, px, py, rng, false, throughput, vpath[size_t(viewPathLen) + 1], cnt);
		if(r == 0) break;
		++viewPathLen;
		const BVertex& h = vpath[size_t(viewPathLen)];
		if(viewPathLen >= P.minPathLength) {
			// get_emission (path_util.hpp:410-458) and the random-hit weight (cpu_bpt.cpp:104-115)
			V3 value = { 0, 0, 0 };
			float backPdf = 0.0f, startPdf = 0.0f;
			if(h.kind == BV_VOID) {
				const LightTree& T = S.lightTree;
				if(T.hasBackground) {
					value = T.bgColor * T.bgScale;
					if(nonzero(value)) {
						backPdf = 1.0f / projected_area(h.incEnc, S.aabb);
						const float bgFlux = (T.bgFlux.x + T.bgFlux.y) + T.bgFlux.z;
						const float p = bgFlux / ((T.dirFlux + T.rootFlux) + bgFlux);
						startPdf = (1.0f / (4.0f * PI)) * p;
					}
				}
			} else if(h.mat.type == OR_MAT_EMISSIVE) {
				const float cosOut = dot(h.ts.geoN, -bv_incident_dir(h));
				if(cosOut > 0.0f) {
					value = h.mat.radiance;
					backPdf = cosOut / PI;
					// the bidirectional weight counts the light's emission pdf (cpu_bpt.cpp:228)
					if(nonzero(value)) startPdf = light_pdfs(S, h.inst, h.prim, h.sp, V3{ 0, 0, 0 }).emit;
				}
			}
			if(nonzero(value)) {
				const float sum = bpt_mis_part(vpath, h, backPdf, startPdf, BV_VIRTUAL, { 0, 0, 0 }, 0.0f);
				value = value * (1.0f / (1.0f + sum));
			}
			const V3 rad = throughput * value;
			const float light = ((throughput.x + throughput.y) + throughput.z) / 3.0f * (((value.x + value.y) + value.z) / 3.0f);
			const size_t slot = hitBase + size_t(viewPathLen - 1);
			recPixel[slot] = pixel;
			float* o = recValue + 4 * slot;
			o[0] = nan_to_zero(rad.x); o[1] = nan_to_zero(rad.y); o[2] = nan_to_zero(rad.z); o[3] = nan_to_zero(light);
		}
		if(bv_end(h.kind)) break;
	} while(viewPathLen < maxP);
}

void bpt_iterate(BptState& st, int numThreads) {
	const Scene& S = *st.scene;
	const u32 n = S.width * S.height;
	const i32 maxP = std::max(1, st.params.maxPathLength);
	const size_t slots = bpt_slots(maxP);
	++st.iteration;
	st.recPixel.assign(size_t(n) * slots, -1);
	st.recValue.assign(size_t(n) * slots * 4, 0.0f);
	Counters total;
#pragma omp parallel num_threads(numThreads)
	{
		Counters local;
#pragma omp for schedule(dynamic, 256)
		for(i32 pixel = 0; pixel < i32(n); ++pixel)
			bpt_sample(st, pixel % i32(S.width), pixel / i32(S.width), u32(pixel), n, st.rngs[size_t(pixel)],
			           &st.recPixel[size_t(pixel) * slots], &st.recValue[size_t(pixel) * slots * 4], local);
#pragma omp critical
		total.add(local);
	}
	st.stats.add(total);
	std::vector<float> iter(size_t(n) * 4, 0.0f);
	for(size_t k = 0; k < st.recPixel.size(); ++k) {
		if(st.recPixel[k] < 0) continue;
		float* d = &iter[size_t(st.recPixel[k]) * 4];
		for(int c = 0; c < 4; ++c) d[c] += st.recValue[4 * k + size_t(c)];
	}
	const float itf = float(st.iteration);
	for(size_t p = 0; p < n; ++p) {
		for(int c = 0; c < 3; ++c) update_moments(iter[4 * p + size_t(c)], st.radiance[3 * p + size_t(c)], st.radianceVar[3 * p + size_t(c)], itf);
		update_moments(iter[4 * p + 3], st.lightness[p], st.lightnessVar[p], itf);
	}
}

// ---------------------------------------------------------------- vertex connection and merging
// cpu_vcm.cpp:1-298: one light subpath per pixel, all of them stored as
// photons in a hash grid (data_structs/photon_map.hpp); then per pixel a view
// subpath whose vertices connect to every vertex of one light subpath (chosen
// by a hash of the pixel index), count the emitters they hit, and merge with
// the photons within the merge radius. All estimates share one balance
// heuristic over connections and merges (VcmVertexExt, cpu_vcm.cpp:17-146).
//
// The hash grid here is deterministic: the reference inserts photons from
// parallel threads at the head of each bucket's list, so its buckets hold
// them in reverse insertion order; this restatement visits a bucket's photons
// in descending (light subpath, vertex) order, the reference's order for a
// single thread.

// photon_map.hpp:29-52: the cell of a position and the hash of a cell
constexpr u32 VCM_MAGIC[3] = { 0xb286aff7u, 0x35e4a487u, 0x75a9c18fu };
// An integral float as the grid's unsigned coordinate (two's complement wrap
// for negative cells, as the conversion does on the reference's x86 hosts).
inline u32 vcm_cell_coord(float x) { return u32(int64_t(x)); }
inline u32 vcm_cell_hash(u32 x, u32 y, u32 z) { return x * VCM_MAGIC[0] + y * VCM_MAGIC[1] + z * VCM_MAGIC[2]; }
// HashGrid::insert: the cell is ceil(position / cell edge)
inline u32 vcm_insert_hash(V3 p, float density) {
	return vcm_cell_hash(vcm_cell_coord(std::ceil(p.x * density)), vcm_cell_coord(std::ceil(p.y * density)),
	                     vcm_cell_coord(std::ceil(p.z * density)));
}
// HashGrid::find_first: the query's base cell is round(position / cell edge);
// the 8 cells base + {0, 1}^3 cover a disc of half the cell edge
inline u32 vcm_query_hash(V3 p, float density) {
	return vcm_cell_hash(vcm_cell_coord(std::round(p.x * density)), vcm_cell_coord(std::round(p.y * density)),
	                     vcm_cell_coord(std::round(p.z * density)));
}
inline u32 vcm_query_bucket(u32 baseHash, int cell, u32 mapSize) {
	u32 h = baseHash;
	if(cell & 1) h += VCM_MAGIC[0];
	if(cell & 2) h += VCM_MAGIC[1];
	if(cell & 4) h += VCM_MAGIC[2];
	return h % mapSize;
}
// HashGridManager::resize (photon_map.hpp:216-229): the next prime above
// 1.15 x the capacity that is 3 mod 4
u32 vcm_map_size(u32 capacity) {
	auto prime = [](u32 v) {
		if(v < 2) return false;
		for(u32 d = 2; u64(d) * d <= v; ++d) if(v % d == 0) return false;
		return true;
	};
	u32 v = u32(float(capacity) * 1.15f);
	do { ++v; while(!prime(v)) ++v; } while((v & 3u) != 3u);
	return v;
}
// Thomas Wang's 32-bit integer hash (cn::WangHash of the reference's
// cn/rnd.hpp, a dependency the reference does not vendor)
inline u32 wang_hash(u32 x) {
	x = (x ^ 61u) ^ (x >> 16);
	x = x * 9u;
	x = x ^ (x >> 4);
	x = x * 0x27d4eb2du;
	x = x ^ (x >> 15);
	return x;
}

struct VcmState {
	const Scene* scene;
	OrLtParams params;
	float mergeRadius;      // "Relative merge radius": of the scene's diagonal
	bool progressive;       // "Progressive": the radius shrinks with iteration^(-1/6)
	std::vector<Pcg64> rngs;
	std::vector<float> radiance, lightness, radianceVar, lightnessVar;
	std::vector<i32> recPixel; // per pixel: connections [view length][light vertex], hits [view length - 1], merges [view length - 1]
	std::vector<float> recValue;
	i32 iteration = -1;
	Counters stats;
};

inline size_t vcm_slots(i32 maxPath) { return size_t(maxPath) * size_t(maxPath) + 2 * size_t(maxPath); }

// path_util.hpp:568-625 create_light and mis_start_pdf (:763-771)
BVertex vcm_light_vertex(const Scene& S, const Emitter& em) {
	BVertex l0 = BVertex{};
	l0.prev = -1;
	l0.position = em.position;
	l0.throughput = { 1, 1, 1 };
	if(em.kind == LV_POINT) { l0.kind = BV_POINT; l0.incEnc = em.intensity; l0.incidentPdf = em.pChoice; }
	else if(em.kind == LV_AREA) { l0.kind = BV_AREA; l0.incEnc = em.normal; l0.intensity = em.intensity; l0.incidentPdf = em.pdf * em.pChoice; }
	else {
		l0.kind = BV_ENV; l0.incEnc = em.normal; l0.intensity = em.intensity; l0.incidentPdf = em.pdf * em.pChoice;
		l0.position = { 0, 0, 0 };
		l0.projSceneArea = projected_area(-em.normal, S.aabb);
	}
	return l0;
}

// cpu_vcm.cpp:50-68: the weight of a connection of view vertex v with light vertex w
float vcm_connection_weight(const std::vector<BVertex>& vpath, const BVertex& v, const EvalValue& vPdf,
                            const std::vector<BVertex>& lpath, const BVertex& w, const EvalValue& lPdf, V3 dir,
                            float distSq, float nPhotons, float area) {
	float relSumV = 1.0f + vcm_prev_rel_sum(vpath, v, vPdf.pdfB, nPhotons, area);
	float relSumL = 1.0f + vcm_prev_rel_sum(lpath, w, lPdf.pdfB, nPhotons, area);
	const float lightToView = bv_convert_pdf(v, w.kind, lPdf.pdfF, dir, distSq);
	relSumV *= lightToView / v.incidentPdf;
	if(v.prev >= 0) relSumV += lightToView * nPhotons * area;
	const float viewToLight = bv_convert_pdf(w, v.kind, vPdf.pdfF, dir, distSq);
	relSumL *= viewToLight / w.incidentPdf;
	if(w.prev >= 0) relSumL += viewToLight * nPhotons * area;
	return 1.0f / (1.0f + relSumV + relSumL);
}

// cpu_vcm.cpp:35-47: the weight of a merge of view vertex v with photon w
float vcm_merge_weight(const std::vector<BVertex>& vpath, const BVertex& v, const EvalValue& pdf,
                       const std::vector<BVertex>& lpath, const BVertex& w, float nPhotons, float area) {
	float relSumV = 1.0f + vcm_prev_rel_sum(vpath, v, pdf.pdfB, nPhotons, area);
	float relSumL = 1.0f + vcm_prev_rel_sum(lpath, w, pdf.pdfF, nPhotons, area);
	relSumV /= v.incidentPdf * nPhotons * area;
	relSumL /= w.incidentPdf * nPhotons * area;
	return 1.0f / (1.0f + relSumV + relSumL);
}

// cpu_vcm.cpp:71-78: the weight of an emitter or the background hit at v
float vcm_hit_weight(const std::vector<BVertex>& vpath, const BVertex& v, float pdfBack, float startPdf, float nPhotons,
                     float area) {
	float relSum = 1.0f + vcm_prev_rel_sum(vpath, v, pdfBack, nPhotons, area);
	const float relRndHit = startPdf / v.incidentPdf;
	relSum *= relRndHit;
	return 1.0f / (1.0f + relSum);
}

struct VcmGrid {
	float density = 1.0f;        // 1 / cell edge
	u32 mapSize = 1;
	std::vector<u32> start, end; // per bucket: range in keys
	std::vector<u32> keys;       // light subpath * max. path length + vertex, by bucket then ascending
};

void vcm_iterate(VcmState& st, int numThreads) {
	const Scene& S = *st.scene;
	const OrLtParams& P = st.params;
	const u32 n = S.width * S.height;
	const i32 maxP = std::max(1, P.maxPathLength);
	const size_t slots = vcm_slots(maxP);
	++st.iteration;
	st.recPixel.assign(size_t(n) * slots, -1);
	st.recValue.assign(size_t(n) * slots * 4, 0.0f);
	// CpuVcm::iterate (cpu_vcm.cpp:148-172)
	const float diag = len(S.aabb.mx - S.aabb.mn); // SceneDescriptor::diagSize (scene.cpp:377)
	float radius = st.mergeRadius * diag;
	if(st.progressive) radius *= std::pow(float(st.iteration + 1), -1.0f / 6.0f);
	const float nPhotons = float(n);
	const float lightArea[2] = { nPhotons, PI * radius * radius };     // trace_photon's merge area
	const float radiusSq = radius * radius;
	const float viewArea[2] = { nPhotons, PI * radiusSq };             // sample's merge area
	const u64 photonSeed = st.rngs[0].next();
	std::vector<std::vector<BVertex>> lpaths(n);
	std::vector<i32> lightLen(n, -1);
	Counters total;
	// first pass: one light subpath per pixel (CpuVcm::trace_photon, :191-218)
#pragma omp parallel num_threads(numThreads)
	{
		Counters local;
#pragma omp for schedule(dynamic, 256)
		for(i32 i = 0; i < i32(n); ++i) {
			Pcg64& rng = st.rngs[size_t(i)];
			const u64 r0 = rng.next();
			const Emitter em = lights_emit(S, u64(i), n, photonSeed, sample_uniform(u32(r0)), sample_uniform(u32(r0 >> 32)));
			if(!em.valid) continue; // no light in the scene at all
			std::vector<BVertex>& lp = lpaths[size_t(i)];
			lp.assign(size_t(maxP) + 1, BVertex{});
			lp[0] = vcm_light_vertex(S, em);
			V3 thr = { 1, 1, 1 };
			i32 len = 0;
			while(len < maxP - 1) {
				if(bpt_walk(S, lp, len, P, 0, 0, rng, true, thr, lp[size_t(len) + 1], local, lightArea) != 1) break;
				++len;
			}
			lightLen[size_t(i)] = len;
		}
#pragma omp critical
		total.add(local);
	}
	// the photon map: every light vertex after the start (vertex 0 is never merged)
	VcmGrid G;
	G.density = 1.0f / (radius * 2.0001f);
	G.mapSize = vcm_map_size(n * u32(maxP));
	{
		std::vector<std::pair<u32, u32>> e;
		for(u32 i = 0; i < n; ++i)
			for(i32 l = 1; l <= lightLen[i]; ++l)
				e.push_back({ vcm_insert_hash(lpaths[i][size_t(l)].position, G.density) % G.mapSize, i * u32(maxP) + u32(l) });
		std::sort(e.begin(), e.end());
		G.start.assign(G.mapSize, 0);
		G.end.assign(G.mapSize, 0);
		G.keys.resize(e.size());
		for(size_t k = 0; k < e.size(); ++k) {
			G.keys[k] = e[k].second;
			if(k == 0 || e[k - 1].first != e[k].first) G.start[e[k].first] = u32(k);
			G.end[e[k].first] = u32(k + 1);
		}
	}
	// second pass: view subpaths (CpuVcm::sample, :220-290)
#pragma omp parallel num_threads(numThreads)
	{
		Counters local;
#pragma omp for schedule(dynamic, 256)
		for(i32 pixel = 0; pixel < i32(n); ++pixel) {
			const i32 px = pixel % i32(S.width), py = pixel / i32(S.width);
			Pcg64& rng = st.rngs[size_t(pixel)];
			i32* recPixel = &st.recPixel[size_t(pixel) * slots];
			float* recValue = &st.recValue[size_t(pixel) * slots * 4];
			auto put = [&](size_t slot, i32 pix, V3 rad, float light) {
				recPixel[slot] = pix;
				float* o = recValue + 4 * slot;
				o[0] = nan_to_zero(rad.x); o[1] = nan_to_zero(rad.y); o[2] = nan_to_zero(rad.z); o[3] = nan_to_zero(light);
			};
			const u32 lightPath = wang_hash(u32(pixel)) % n;
			const std::vector<BVertex>& lp = lpaths[lightPath];
			const i32 lLen = lightLen[lightPath];
			std::vector<BVertex> vpath(size_t(maxP) + 1);
			BVertex& c = vpath[0];
			c = BVertex{};
			c.kind = BV_CAMERA;
			c.prev = -1;
			c.position = S.cam.position;
			c.incEnc = { float(px), float(py), 0.0f };
			c.incidentPdf = 1.0f;
			c.throughput = { 1, 1, 1 };
			(void)rng.next(); // create_camera consumes one number (unused by the pinhole camera)
			V3 throughput = { 1, 1, 1 };
			i32 viewLen = 0;
			do {
				// connections to every vertex of the light subpath, from its end (:232-246)
				const BVertex& v = vpath[size_t(viewLen)];
				for(i32 l = lLen; l >= 0; --l) {
					const i32 pathLen = l + 1 + viewLen;
					if(pathLen < P.minPathLength || pathLen > P.maxPathLength) continue;
					const BVertex& w = lp[size_t(l)];
					i32 ox = px, oy = py;
					V3 bxdfs = { 0, 0, 0 };
					float cosines = 0.0f;
					if(!((bv_ortho(v.kind) && bv_ortho(w.kind)) || (bv_ortho(v.kind) && bv_camera(w.kind)) ||
					     (bv_camera(v.kind) && bv_ortho(w.kind)))) {
						V3 dir;
						float distSq;
						if(bv_ortho(w.kind)) { dir = -w.incEnc; distSq = 1.0f; }
						else {
							const V3 cv = w.position - v.position;
							distSq = lensq(cv);
							const float dist = mbmath::sqrt(distSq);
							dir = { sdiv(cv.x, dist), sdiv(cv.y, dist), sdiv(cv.z, dist) };
						}
						const EvalValue val0 = bv_evaluate(S, v, dir, false, ox, oy);
						const EvalValue val1 = bv_evaluate(S, w, -dir, true, ox, oy);
						if(ox != -1) {
							const V3 bxdfProd = val0.value * val1.value;
							const float cosProd = val0.cosOut * val1.cosOut;
							if(any_pos(bxdfProd) && cosProd > 0.0f &&
							   !any_intersection(S, v.position, bv_position(w, v.position), bv_geo_normal(v), bv_geo_normal(w), dir, local)) {
								const float mis = vcm_connection_weight(vpath, v, val0, lp, w, val1, dir, distSq, viewArea[0], viewArea[1]);
								bxdfs = bxdfProd * (mis / distSq);
								cosines = cosProd;
							}
						}
					}
					if(ox != -1)
						put(size_t(viewLen) * size_t(maxP) + size_t(l), oy * i32(S.width) + ox,
						    ((throughput * w.throughput) * cosines) * bxdfs, (((throughput.x + throughput.y) + throughput.z) / 3.0f) * cosines);
				}
				// walk (:249-256)
				if(bpt_walk(S, vpath, viewLen, P, px, py, rng, false, throughput, vpath[size_t(viewLen) + 1], local, viewArea) == 0) break;
				++viewLen;
				const BVertex& h = vpath[size_t(viewLen)];
				// emitters and the background (:259-268)
				if(viewLen >= P.minPathLength) {
					V3 value = { 0, 0, 0 };
					float backPdf = 0.0f, startPdf = 0.0f;
					if(h.kind == BV_VOID) {
						const LightTree& T = S.lightTree;
						if(T.hasBackground) {
							value = T.bgColor * T.bgScale;
							if(nonzero(value)) {
								backPdf = 1.0f / projected_area(h.incEnc, S.aabb);
								const float bgFlux = (T.bgFlux.x + T.bgFlux.y) + T.bgFlux.z;
								const float p = bgFlux / ((T.dirFlux + T.rootFlux) + bgFlux);
								startPdf = (1.0f / (4.0f * PI)) * p;
							}
						}
					} else if(h.mat.type == OR_MAT_EMISSIVE) {
						const float cosOut = dot(h.ts.geoN, -bv_incident_dir(h));
						if(cosOut > 0.0f) {
							value = h.mat.radiance;
							backPdf = cosOut / PI;
							if(nonzero(value)) startPdf = light_pdfs(S, h.inst, h.prim, h.sp, V3{ 0, 0, 0 }).emit;
						}
					}
					if(nonzero(value)) value = value * vcm_hit_weight(vpath, h, backPdf, startPdf, viewArea[0], viewArea[1]);
					put(size_t(maxP) * size_t(maxP) + size_t(viewLen - 1), pixel, throughput * value,
					    (((throughput.x + throughput.y) + throughput.z) / 3.0f) * (((value.x + value.y) + value.z) / 3.0f));
				}
				if(bv_end(h.kind)) break;
				// merges with the photons within the radius (:271-288)
				V3 rad = { 0, 0, 0 };
				const u32 base = vcm_query_hash(h.position, G.density);
				for(int cell = 0; cell < 8; ++cell) {
					const u32 b = vcm_query_bucket(base, cell, G.mapSize);
					for(u32 k = G.end[b]; k > G.start[b];) {
						--k;
						const u32 key = G.keys[k];
						const std::vector<BVertex>& ph = lpaths[key / u32(maxP)];
						const i32 l = i32(key % u32(maxP));
						const BVertex& w = ph[size_t(l)];
						const i32 pathLen = viewLen + l;
						if(l > 0 && pathLen >= P.minPathLength && pathLen <= P.maxPathLength && lensq(w.position - h.position) < radiusSq) {
							const V3 geoN = w.ts.geoN;
							const EvalValue bsdf = material_evaluate(h.ts, h.mat, bv_incident_dir(h), -bv_incident_dir(w), false, &geoN);
							const float mis = vcm_merge_weight(vpath, h, bsdf, ph, w, viewArea[0], viewArea[1]);
							rad = rad + (bsdf.value * w.throughput) * mis;
						}
					}
				}
				const float norm = viewArea[1] * viewArea[0];
				rad = { rad.x / norm, rad.y / norm, rad.z / norm };
				put(size_t(maxP) * size_t(maxP) + size_t(maxP) + size_t(viewLen - 1), pixel, throughput * rad,
				    (((throughput.x + throughput.y) + throughput.z) / 3.0f) * (((rad.x + rad.y) + rad.z) / 3.0f));
			} while(viewLen < maxP);
		}
#pragma omp critical
		total.add(local);
	}
	st.stats.add(total);
	std::vector<float> iter(size_t(n) * 4, 0.0f);
	for(size_t k = 0; k < st.recPixel.size(); ++k) {
		if(st.recPixel[k] < 0) continue;
		float* dd = &iter[size_t(st.recPixel[k]) * 4];
		for(int ch = 0; ch < 4; ++ch) dd[ch] += st.recValue[4 * k + size_t(ch)];
	}
	const float itf = float(st.iteration);
	for(size_t p = 0; p < n; ++p) {
		for(int ch = 0; ch < 3; ++ch) update_moments(iter[4 * p + size_t(ch)], st.radiance[3 * p + size_t(ch)], st.radianceVar[3 * p + size_t(ch)], itf);
		update_moments(iter[4 * p + 3], st.lightness[p], st.lightnessVar[p], itf);
	}
}

// ---------------------------------------------------------------- wireframe renderer
// wireframe_common.hpp:15-180 and cpu_wireframe.cpp:18-38: one camera ray per
// pixel and iteration, walked through the surfaces until it passes within
// "Line width" pixels of an edge (white) or leaves the scene (background).
struct WireState {
	const Scene* scene;
	float lineWidth;
	i32 maxTraceDepth;
	std::vector<Pcg64> rngs;
	std::vector<float> border;    // cumulative mean, 3 per pixel
	std::vector<float> borderVar; // its variance
	i32 iteration = -1;
	Counters stats;
};

// wireframe_common.hpp:15-78: the point on the closest edge line (triangle
// AB, AC, BC; quad AB, AC, BD, CD with (A, B, C, D) = (v0, v1, v3, v2)).
// The choice is the reference's chain (:36-41, :70-77): edge k wins if its
// distance is <= every other's, tried in order, else the last edge; so with a
// NaN distance (a zero-length edge) the chain falls through to the last edge.
V3 closest_line_point(const V3* c, int n, V3 hit) {
	const int e0[4] = { 0, 0, 1, 2 };
	const int e1[4] = { 1, 2, n == 3 ? 2 : 3, 3 };
	const int ne = n == 3 ? 3 : 4;
	V3 on[4];
	float d[4];
	for(int k = 0; k < ne; ++k) {
		const V3 a = c[e0[k]], e = c[e1[k]] - a, ap = hit - a;
		on[k] = a + e * (dot(ap, e) / lensq(e));
		d[k] = lensq(on[k] - hit);
	}
	for(int k = 0; k + 1 < ne; ++k) {
		bool closest = true;
		for(int j = 0; j < ne; ++j)
			if(j != k && !(d[k] <= d[j])) closest = false;
		if(closest) return on[k];
	}
	return on[ne - 1];
}

V3 wireframe_sample(const WireState& st, i32 px, i32 py, Pcg64& rng, Counters& cnt) {
	const Scene& S = *st.scene;
	(void)rng.next(); // create_camera consumes one number (unused by the pinhole camera)
	const u64 x0 = rng.next();
	(void)rng.next();
	float pdf;
	const V3 dir = pinhole_ray(S.cam, px, py, sample_uniform(u32(x0)), sample_uniform(u32(x0 >> 32)), pdf);
	const V3 cam = S.cam.position;
	V3 origin = cam;
	float total = 0.0f;
	for(i32 i = 0; i < st.maxTraceDepth; ++i) {
		const Intersection hit = first_intersection(S, origin, dir, V3{ 0, 0, 0 }, MAX_SCENE_SIZE, cnt, false);
		if(hit.inst < 0) {
			const LightTree& T = S.lightTree;
			if(T.hasBackground) {
				const V3 bg = T.bgColor * T.bgScale;
				if(any_pos(bg)) return bg;
			}
			return { 0, 0, 0 };
		}
		const float hitDist = hit.distance < 0.001f ? 0.001f : hit.distance;
		const V3 p = origin + dir * hitDist;
		total += hitDist;
		const float pixelSize = total * S.cam.tanVFov / float(S.cam.resY);
		const Mat34 m = instance_to_world(S.w2i[size_t(hit.inst)]);
		const Lod& l = S.lods[S.instLod[size_t(hit.inst)]];
		float rim;
		if(u32(hit.prim) < l.nT + l.nQ) {
			V3 c[4];
			int n;
			if(u32(hit.prim) < l.nT) {
				for(int k = 0; k < 3; ++k) c[k] = xform_point(m, l.verts[l.idx[3 * size_t(hit.prim) + size_t(k)]]);
				n = 3;
			} else {
				const size_t o = 3 * size_t(l.nT) + 4 * (size_t(hit.prim) - l.nT);
				c[0] = xform_point(m, l.verts[l.idx[o]]);
				c[1] = xform_point(m, l.verts[l.idx[o + 1]]);
				c[2] = xform_point(m, l.verts[l.idx[o + 3]]);
				c[3] = xform_point(m, l.verts[l.idx[o + 2]]);
				n = 4;
			}
			const V3 seg = closest_line_point(c, n, p) - cam;
			const V3 proj = seg - dir * dot(seg, dir);
			rim = len(proj);
		} else {
			const i32 sidx = hit.prim - i32(l.nT + l.nQ);
			const V3 center = xform_point(m, sphere_center(l, sidx));
			const V3 toCenter = normalize(center - p);
			rim = 0.05f * (sphere_radius(l, sidx) * dot(toCenter, dir));
		}
		if(rim > st.lineWidth * pixelSize) origin = origin + dir * hitDist;
		else return { 1.0f, 1.0f, 1.0f };
	}
	return { 0, 0, 0 };
}

void wireframe_iterate(WireState& st, int numThreads) {
	const Scene& S = *st.scene;
	const i32 n = i32(S.width * S.height);
	++st.iteration;
	const float itf = float(st.iteration);
	Counters total;
#pragma omp parallel num_threads(numThreads)
	{
		Counters local;
#pragma omp for schedule(dynamic, 256)
		for(i32 pixel = 0; pixel < n; ++pixel) {
			const V3 v = wireframe_sample(st, pixel % i32(S.width), pixel / i32(S.width), st.rngs[size_t(pixel)], local);
			const float it[3] = { v.x, v.y, v.z };
			for(int c = 0; c < 3; ++c)
				update_moments(it[c], st.border[3 * size_t(pixel) + size_t(c)], st.borderVar[3 * size_t(pixel) + size_t(c)], itf);
		}
#pragma omp critical
		total.add(local);
	}
	st.stats.add(total);
}

// ---------------------------------------------------------------- scene setup
Scene* create_scene(const OrSceneDesc* d) {
	auto S = std::make_unique<Scene>();
	S->width = d->width; S->height = d->height;
	for(u32 i = 0; i < d->numMaterials; ++i) {
		const OrMaterial& m = d->materials[i];
		Material mm;
		mm.type = m.type;
		mm.albedo = { m.albedo[0], m.albedo[1], m.albedo[2] };
		mm.roughness = { m.roughness[0], m.roughness[1] };
		mm.shadowing = m.shadowing; mm.ndf = m.ndf;
		mm.radiance = { m.radiance[0], m.radiance[1], m.radiance[2] };
		mm.scale = { m.scale[0], m.scale[1], m.scale[2] };
		mm.albedoTex = m.albedoTexture;
		mm.alphaTex = m.alphaTexture;
		S->hasAlpha = S->hasAlpha || m.alphaTexture >= 0;
		S->materials.push_back(mm);
	}
	for(u32 i = 0; i < d->numTextures; ++i) {
		Texture t;
		t.w = d->textures[i].width; t.h = d->textures[i].height;
		t.texels.assign(d->textures[i].texels, d->textures[i].texels + size_t(t.w) * t.h * 4);
		S->textures.push_back(std::move(t));
	}
	S->lods.resize(d->numLods);
	for(u32 i = 0; i < d->numLods; ++i) {
		const OrLod& s = d->lods[i];
		Lod& l = S->lods[i];
		l.nV = s.numVertices; l.nT = s.numTriangles; l.nQ = s.numQuads; l.nS = s.numSpheres;
		l.verts.resize(l.nV); l.normals.resize(l.nV); l.uvs.resize(l.nV);
		for(u32 v = 0; v < l.nV; ++v) {
			l.verts[v] = { s.vertices[3 * v], s.vertices[3 * v + 1], s.vertices[3 * v + 2] };
			l.normals[v] = s.normals ? V3{ s.normals[3 * v], s.normals[3 * v + 1], s.normals[3 * v + 2] } : V3{ 0, 0, 0 };
			l.uvs[v] = s.uvs ? V2{ s.uvs[2 * v], s.uvs[2 * v + 1] } : V2{ 0, 0 };
		}
		l.idx.assign(s.indices, s.indices + (size_t(l.nT) * 3 + size_t(l.nQ) * 4));
		l.faceMat.assign(s.faceMaterials, s.faceMaterials + (l.nT + l.nQ));
		l.spheres.assign(s.spheres, s.spheres + size_t(l.nS) * 4);
		l.sphereMat.assign(s.sphereMaterials, s.sphereMaterials + l.nS);
		l.numPrims = i32(l.nT + l.nQ + l.nS);
		Box b = empty_box();
		for(u32 v = 0; v < l.nV; ++v) { b.mn = vmin(b.mn, l.verts[v]); b.mx = vmax(b.mx, l.verts[v]); }
		for(u32 k = 0; k < l.nS; ++k) {
			const V3 c = sphere_center(l, k); const float r = sphere_radius(l, k);
			b.mn = vmin(b.mn, c - V3{ r, r, r }); b.mx = vmax(b.mx, c + V3{ r, r, r });
		}
		l.aabb = b;
	}
	// LoD BVHs (lod.cpp:16-38)
	S->lodBvh.resize(d->numLods);
	for(u32 i = 0; i < d->numLods; ++i) {
		BuildDesc bd;
		bd.isScene = false; bd.scene = S.get(); bd.lod = &S->lods[i];
		bd.numPrims = S->lods[i].numPrims; bd.bb = S->lods[i].aabb;
		build_lbvh(bd, bd.numPrims, bd.numPrims, S->lodBvh[i]);
	}
	// Instances (scene.cpp:111-419)
	S->w2i.resize(d->numInstances);
	S->instLod.assign(d->instanceLod, d->instanceLod + d->numInstances);
	std::vector<Box> instBoxes(d->numInstances, empty_box());
	std::vector<V3> instCentroids(d->numInstances, V3{ 0, 0, 0 });
	S->activeInstances = 0;
	S->validInstance = 0xFFFFFFFFu;
	Box sceneBox = empty_box();
	for(u32 i = 0; i < d->numInstances; ++i) {
		std::memcpy(S->w2i[i].m, d->worldToInstance + 12 * i, sizeof(float) * 12);
		if(S->instLod[i] == 0xFFFFFFFFu) continue;
		++S->activeInstances;
		if(S->validInstance == 0xFFFFFFFFu) S->validInstance = i;
		const Mat34 i2w = instance_to_world(S->w2i[i]);
		const Box lb = S->lods[S->instLod[i]].aabb;
		instBoxes[i] = xform_box(i2w, lb);
		instCentroids[i] = xform_point(i2w, center(lb));
		sceneBox = merge(sceneBox, instBoxes[i]);
	}
	S->aabb = sceneBox;
	{
		BuildDesc bd;
		bd.isScene = true; bd.scene = S.get(); bd.lod = nullptr;
		bd.numPrims = i32(d->numInstances); bd.bb = sceneBox;
		bd.instBoxes = instBoxes; bd.instCentroids = instCentroids;
		build_lbvh(bd, i32(d->numInstances), S->activeInstances, S->tlas);
	}
	// Camera (camera.hpp:81-96, pinhole.hpp:22)
	{
		V3 dir = { d->camDir[0], d->camDir[1], d->camDir[2] };
		V3 up = { d->camUp[0], d->camUp[1], d->camUp[2] };
		dir = normalize(dir);
		up = normalize(up);
		const float zDotY = dot(dir, up);
		up = normalize(up - zDotY * dir);
		S->cam.position = { d->camPos[0], d->camPos[1], d->camPos[2] };
		S->cam.viewDir = dir;
		S->cam.up = up;
		S->cam.tanVFov = std::tan(d->vFov / 2.0f);
		S->cam.nearP = d->nearPlane; S->cam.farP = d->farPlane;
		S->cam.resX = u16(d->width); S->cam.resY = u16(d->height);
	}
	// Lights (world_container.cpp:869-990, light_tree.cpp:340-447)
	const auto tLights = std::chrono::steady_clock::now();
	LightTree& T = S->lightTree;
	for(u32 inst = 0; inst < d->numInstances; ++inst) {
		if(S->instLod[inst] == 0xFFFFFFFFu) continue;
		const Lod& l = S->lods[S->instLod[inst]];
		const Mat34 i2w = instance_to_world(S->w2i[inst]);
		const float* m = i2w.m;
		const float det3 = m[0] * (m[5] * m[10] - m[9] * m[6]) - m[1] * (m[4] * m[10] - m[8] * m[6]) + m[2] * (m[4] * m[9] - m[8] * m[5]);
		const bool mirroring = det3 < 0.0f;
		// world_container.cpp:929-948: emissive triangles first, then quads
		for(u32 t = 0; t < l.nT; ++t) {
			const u16 mi = l.faceMat[t];
			if(S->materials[mi].type != OR_MAT_EMISSIVE) continue;
			V3 pts[3]; V2 uvs[3];
			for(int k = 0; k < 3; ++k) { pts[k] = xform_point(i2w, l.verts[l.idx[3 * t + k]]); uvs[k] = l.uvs[l.idx[3 * t + k]]; }
			if(mirroring) { std::swap(pts[1], pts[2]); std::swap(uvs[1], uvs[2]); }
			PosLight pl{};
			pl.type = LT_TRI;
			pl.posV[0] = pts[0];
			pl.posV[1] = pts[1] - pts[0];
			pl.posV[2] = pts[2] - pts[0];
			pl.uvV[0] = uvs[0];
			pl.uvV[1] = uvs[1] - uvs[0];
			pl.uvV[2] = uvs[2] - uvs[0];
			pl.material = mi;
			pl.primInst = i32(inst);
			pl.primId = i32(t);
			T.lights.push_back(pl);
		}
		for(u32 q = 0; q < l.nQ; ++q) {
			const u16 mi = l.faceMat[l.nT + q];
			if(S->materials[mi].type != OR_MAT_EMISSIVE) continue;
			V3 pts[4]; V2 uvs[4];
			const u32 o = l.nT * 3 + q * 4;
			for(int k = 0; k < 4; ++k) { pts[k] = xform_point(i2w, l.verts[l.idx[o + k]]); uvs[k] = l.uvs[l.idx[o + k]]; }
			if(mirroring) { std::swap(pts[1], pts[3]); std::swap(uvs[1], uvs[3]); }
			PosLight pl{};
			pl.type = LT_QUAD;
			pl.posV[0] = pts[0];
			pl.posV[1] = pts[3] - pts[0];
			pl.posV[2] = pts[1] - pts[0];
			pl.posV[3] = (pts[2] - pts[3]) - pl.posV[2];
			pl.uvV[0] = uvs[0];
			pl.uvV[1] = uvs[3] - uvs[0];
			pl.uvV[2] = uvs[1] - uvs[0];
			pl.uvV[3] = (uvs[2] - uvs[3]) - pl.uvV[2];
			pl.material = mi;
			pl.primInst = i32(inst);
			pl.primId = i32(l.nT + q);
			T.lights.push_back(pl);
		}
		// world_container.cpp:966-990: then spheres, the centre transformed and
		// the radius scaled by the length of the instance's first axis
		for(u32 k = 0; k < l.nS; ++k) {
			const u16 mi = l.sphereMat[k];
			if(S->materials[mi].type != OR_MAT_EMISSIVE) continue;
			PosLight pl{};
			pl.type = LT_SPHERE;
			pl.position = xform_point(i2w, sphere_center(l, k));
			pl.radius = len(V3{ m[0], m[4], m[8] }) * sphere_radius(l, k);
			pl.material = mi;
			pl.primInst = i32(inst);
			pl.primId = i32(l.nT + l.nQ + k);
			T.lights.push_back(pl);
		}
	}
	for(u32 i = 0; i < d->numPointLights; ++i) {
		PosLight pl{};
		pl.type = LT_POINT;
		pl.position = { d->pointLights[6 * i], d->pointLights[6 * i + 1], d->pointLights[6 * i + 2] };
		pl.intensity = { d->pointLights[6 * i + 3], d->pointLights[6 * i + 4], d->pointLights[6 * i + 5] };
		T.lights.push_back(pl);
	}
	if(T.lights.size() > 1) {
		const V3 scale = sceneBox.mx - sceneBox.mn;
		auto conv = [](float v) { return v <= 0.0f ? 0u : (v >= 4294967040.0f ? 0xFFFFFF00u : u32(v)); };
		auto hilbert = [](u32 a, u32 b, u32 c) { return hilbert_code16(a, b, c); };
		std::stable_sort(T.lights.begin(), T.lights.end(), [&](const PosLight& a, const PosLight& b) {
			const V3 ca = light_center(a) * scale, cb = light_center(b) * scale;
			const u32 ax = conv(ca.x), ay = conv(ca.y), az = conv(ca.z);
			const u32 bx = conv(cb.x), by = conv(cb.y), bz = conv(cb.z);
			u64 A = hilbert(ax >> 16, ay >> 16, az >> 16), B = hilbert(bx >> 16, by >> 16, bz >> 16);
			if(A == B) { A = hilbert(ax & 0xffff, ay & 0xffff, az & 0xffff); B = hilbert(bx & 0xffff, by & 0xffff, bz & 0xffff); }
			return A < B;
		});
	}
	build_pos_tree(*S, T);
	S->lightBuildMs = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - tLights).count();
	T.hasBackground = d->hasBackground != 0;
	if(T.hasBackground) {
		T.bgColor = { d->backgroundColor[0], d->backgroundColor[1], d->backgroundColor[2] };
		T.bgScale = { d->backgroundScale[0], d->backgroundScale[1], d->backgroundScale[2] };
		// background.cpp:125-135
		const V3 diag = sceneBox.mx - sceneBox.mn;
		const float solidAngle = 4.0f * PI;
		const float area = 2.0f * PI * ((diag.x * diag.y + diag.x * diag.z) + diag.y * diag.z);
		const float f = solidAngle * area;
		T.bgFlux = T.bgColor * f;
	}
	return S.release();
}

} // namespace

// ================================================================= C ABI
extern "C" {

void* oracle_scene_create(const OrSceneDesc* desc) {
	if(!desc) return nullptr;
	return create_scene(desc);
}

void oracle_scene_destroy(void* s) { delete static_cast<Scene*>(s); }

static const Bvh* pick_bvh(Scene* S, int32_t which) {
	if(which < 0) return &S->tlas;
	if(u32(which) >= S->lodBvh.size()) return nullptr;
	return &S->lodBvh[which];
}

int oracle_bvh_info(void* s, int32_t which, int32_t* numPrims, int32_t* numInternal) {
	const Bvh* b = pick_bvh(static_cast<Scene*>(s), which);
	if(!b) return 0;
	if(numPrims) *numPrims = b->numPrims;
	if(numInternal) *numInternal = b->numInternal;
	return 1;
}

int oracle_bvh_get(void* s, int32_t which, uint64_t* morton, int32_t* parents, float* nodes, int32_t* primIds) {
	const Bvh* b = pick_bvh(static_cast<Scene*>(s), which);
	if(!b) return 0;
	if(morton && !b->mortonSorted.empty()) std::memcpy(morton, b->mortonSorted.data(), b->mortonSorted.size() * 8);
	if(parents && !b->parents.empty()) std::memcpy(parents, b->parents.data(), b->parents.size() * 4);
	if(nodes && !b->nodes.empty()) std::memcpy(nodes, b->nodes.data(), b->nodes.size() * sizeof(BvhNode));
	if(primIds && !b->primIds.empty()) std::memcpy(primIds, b->primIds.data(), b->primIds.size() * 4);
	return 1;
}

// Rebuilds every LoD hierarchy of the scene with 63- or 30-bit Morton codes
// (build_lbvh.cu:59-86); bvh(which) then returns those.
int oracle_scene_rebuild_lod_bvhs(void* s, int32_t mortonBits) {
	Scene* S = static_cast<Scene*>(s);
	if(mortonBits != 63 && mortonBits != 30) return 0;
	for(size_t i = 0; i < S->lods.size(); ++i) {
		BuildDesc bd;
		bd.isScene = false; bd.scene = S; bd.lod = &S->lods[i];
		bd.numPrims = S->lods[i].numPrims; bd.bb = S->lods[i].aabb;
		bd.mortonBits = mortonBits;
		build_lbvh(bd, bd.numPrims, bd.numPrims, S->lodBvh[i]);
	}
	return 1;
}

int oracle_scene_aabb(void* s, float* a) {
	Scene* S = static_cast<Scene*>(s);
	a[0] = S->aabb.mn.x; a[1] = S->aabb.mn.y; a[2] = S->aabb.mn.z;
	a[3] = S->aabb.mx.x; a[4] = S->aabb.mx.y; a[5] = S->aabb.mx.z;
	return 1;
}

// The light list and tree in the core's device layout (scene_types.hpp
// DLight 108 bytes, DLightNode 20 bytes) so tests compare them byte for byte.
double oracle_light_build_ms(void* s) { return static_cast<const Scene*>(s)->lightBuildMs; }

int oracle_light_tree(void* s, uint32_t* numLights, uint32_t* numNodes, uint32_t* numCodes, void* lightsOut,
                      void* nodesOut, uint64_t* keysOut, uint32_t* codesOut, float* rootFlux) {
	const Scene* S = static_cast<const Scene*>(s);
	const LightTree& T = S->lightTree;
	if(numLights) *numLights = u32(T.lights.size());
	if(numNodes) *numNodes = u32(T.nodes.size());
	if(numCodes) *numCodes = u32(T.primToNodePath.size());
	if(rootFlux) *rootFlux = T.rootFlux;
	if(lightsOut) {
		unsigned char* o = static_cast<unsigned char*>(lightsOut);
		for(const PosLight& l : T.lights) {
			float f[27] = { l.position.x, l.position.y, l.position.z, l.intensity.x, l.intensity.y, l.intensity.z };
			for(int k = 0; k < 4; ++k) { f[6 + 3 * k] = l.posV[k].x; f[7 + 3 * k] = l.posV[k].y; f[8 + 3 * k] = l.posV[k].z; }
			for(int k = 0; k < 4; ++k) { f[18 + 2 * k] = l.uvV[k].x; f[19 + 2 * k] = l.uvV[k].y; }
			f[26] = l.radius;
			std::memcpy(o, &l.type, 2);
			std::memcpy(o + 2, &l.material, 2);
			std::memcpy(o + 4, f, sizeof(f));
			o += 112;
		}
	}
	if(nodesOut) {
		unsigned char* o = static_cast<unsigned char*>(nodesOut);
		for(const LightNode& n : T.nodes) {
			std::memcpy(o, &n.left.flux, 4); std::memcpy(o + 4, &n.right.flux, 4);
			std::memcpy(o + 8, &n.left.index, 4); std::memcpy(o + 12, &n.right.index, 4);
			std::memcpy(o + 16, &n.left.type, 2); std::memcpy(o + 18, &n.right.type, 2);
			o += 20;
		}
	}
	size_t k = 0;
	for(const auto& [prim, code] : T.primToNodePath) {
		if(keysOut) keysOut[k] = (u64(u32(prim.first)) << 32) | u32(prim.second);
		if(codesOut) codesOut[k] = code;
		++k;
	}
	return 1;
}

int oracle_trace_first(void* s, const float* rays, const float* geoNormals, float tmax, uint32_t n,
                       float* tOut, int32_t* instOut, int32_t* primOut, float* spOut) {
	Scene* S = static_cast<Scene*>(s);
#pragma omp parallel for schedule(static, 256)
	for(int64_t i = 0; i < int64_t(n); ++i) {
		Counters c;
		V3 o = { rays[6 * i], rays[6 * i + 1], rays[6 * i + 2] };
		const V3 d = { rays[6 * i + 3], rays[6 * i + 4], rays[6 * i + 5] };
		const V3 g = geoNormals ? V3{ geoNormals[3 * i], geoNormals[3 * i + 1], geoNormals[3 * i + 2] } : V3{ 0, 0, 0 };
		const Intersection h = first_intersection(*S, o, d, g, tmax, c);
		tOut[i] = h.distance; instOut[i] = h.inst; primOut[i] = h.prim;
		if(spOut) { spOut[2 * i] = h.sp.x; spOut[2 * i + 1] = h.sp.y; }
	}
	return 1;
}

int oracle_trace_any(void* s, const float* a, const float* b, uint32_t n, uint8_t* occ) {
	Scene* S = static_cast<Scene*>(s);
#pragma omp parallel for schedule(static, 256)
	for(int64_t i = 0; i < int64_t(n); ++i) {
		Counters c;
		const V3 pa = { a[3 * i], a[3 * i + 1], a[3 * i + 2] };
		const V3 pb = { b[3 * i], b[3 * i + 1], b[3 * i + 2] };
		const V3 dv = pb - pa;
		const V3 dir = dv / len(dv);
		occ[i] = any_intersection(*S, pa, pb, { 0, 0, 0 }, { 0, 0, 0 }, dir, c) ? 1 : 0;
	}
	return 1;
}

void* oracle_pt_create(void* s, const OrPtParams* params) {
	Scene* S = static_cast<Scene*>(s);
	auto* st = new PtState();
	st->scene = S;
	st->params = *params;
	const i32 num = i32(S->width * S->height);
	st->rngs.resize(num);
	// cpu_pt.cpp:40-45
	const i32 seed = i32(u32(params->seed) * u32(num + 1));
	for(i32 i = 0; i < num; ++i) st->rngs[i] = Pcg64::seeded(u32(i32(u32(i) + u32(seed))));
	st->radiance.assign(size_t(num) * 3, 0.0f);
	st->hitId.assign(size_t(num) * 2, 0.0f);
	st->radianceVar.assign(size_t(num) * 3, 0.0f);
	st->hitIdVar.assign(size_t(num) * 2, 0.0f);
	st->aux.assign(size_t(num) * AUX_CHANNELS, 0.0f);
	st->auxVar.assign(size_t(num) * AUX_CHANNELS, 0.0f);
	return st;
}

void oracle_pt_destroy(void* p) { delete static_cast<PtState*>(p); }

int oracle_albedo_gradient(void* p, int32_t texIndex, uint32_t spp, const float* imageGrad, double* gradOut, int32_t nt) {
	PtState& st = *static_cast<PtState*>(p);
	const Scene& S = *st.scene;
	if(texIndex < 0 || size_t(texIndex) >= S.textures.size() || spp == 0) return 0;
	if(st.params.rrStartDepth < st.params.maxPathLength) return 0; // Russian roulette must be off
	const i32 num = i32(S.width * S.height);
	const Texture& t = S.textures[size_t(texIndex)];
	const size_t nt3 = size_t(t.w) * t.h * 3;
	const i32 seed = i32(u32(st.params.seed) * u32(num + 1));
	if(nt <= 0) nt = 1;
	std::vector<std::vector<double>> part(size_t(nt), std::vector<double>(nt3, 0.0));
#pragma omp parallel num_threads(nt)
	{
		int tid = 0;
#ifdef _OPENMP
		tid = omp_get_thread_num();
#endif
		std::vector<double>& g = part[size_t(tid)];
		Counters cnt;
		AlbedoAdjoint adj;
		adj.texIndex = texIndex;
#pragma omp for schedule(static, 64)
		for(i32 pixel = 0; pixel < num; ++pixel) {
			Pcg64 rng = Pcg64::seeded(u32(i32(u32(pixel) + u32(seed))));
			const double w[3] = { double(imageGrad[3 * size_t(pixel)]) / spp, double(imageGrad[3 * size_t(pixel) + 1]) / spp,
			                      double(imageGrad[3 * size_t(pixel) + 2]) / spp };
			for(u32 s = 0; s < spp; ++s) {
				adj.n = 0;
				V3 rad; V2 hid;
				pt_sample(st, pixel % i32(S.width), pixel / i32(S.width), rng, rad, hid, cnt, &adj);
				for(int k = 0; k < adj.n; ++k)
					for(int c = 0; c < 3; ++c)
						if(adj.alb[k][c] > 0.0) g[3 * size_t(adj.texel[k]) + c] += w[c] * adj.suf[k][c] / adj.alb[k][c];
			}
		}
	}
	for(size_t i = 0; i < nt3; ++i) {
		double acc = 0.0;
		for(auto& g : part) acc += g[i];
		gradOut[i] = acc;
	}
	return 1;
}

int oracle_emission_gradient(void* p, int32_t matIndex, uint32_t spp, const float* imageGrad, double* gradOut, int32_t nt) {
	PtState& st = *static_cast<PtState*>(p);
	const Scene& S = *st.scene;
	if(matIndex < 0 || size_t(matIndex) >= S.materials.size() || spp == 0) return 0;
	const Material& m = S.materials[size_t(matIndex)];
	if(m.type != OR_MAT_EMISSIVE) return 0;
	const i32 num = i32(S.width * S.height);
	const i32 seed = i32(u32(st.params.seed) * u32(num + 1));
	if(nt <= 0) nt = 1;
	std::vector<std::array<double, 3>> part(size_t(nt), std::array<double, 3>{ 0.0, 0.0, 0.0 });
#pragma omp parallel num_threads(nt)
	{
		int tid = 0;
#ifdef _OPENMP
		tid = omp_get_thread_num();
#endif
		Counters cnt;
		AlbedoAdjoint adj;
		adj.emissionMat = matIndex;
		adj.emissionL = m.radiance * m.scale;
#pragma omp for schedule(static, 64)
		for(i32 pixel = 0; pixel < num; ++pixel) {
			Pcg64 rng = Pcg64::seeded(u32(i32(u32(pixel) + u32(seed))));
			const double w[3] = { double(imageGrad[3 * size_t(pixel)]) / spp, double(imageGrad[3 * size_t(pixel) + 1]) / spp,
			                      double(imageGrad[3 * size_t(pixel) + 2]) / spp };
			for(u32 s = 0; s < spp; ++s) {
				adj.n = 0;
				adj.emis[0] = adj.emis[1] = adj.emis[2] = 0.0;
				V3 rad; V2 hid;
				pt_sample(st, pixel % i32(S.width), pixel / i32(S.width), rng, rad, hid, cnt, &adj);
				for(int c = 0; c < 3; ++c) part[size_t(tid)][size_t(c)] += w[c] * adj.emis[c];
			}
		}
	}
	for(int c = 0; c < 3; ++c) {
		double acc = 0.0;
		for(auto& g : part) acc += g[size_t(c)];
		gradOut[c] = acc;
	}
	return 1;
}

int oracle_pt_iterate(void* p, int32_t nt) {
	PtState* st = static_cast<PtState*>(p);
	pt_iterate(*st, nt > 0 ? nt : 1, 0, st->scene->height, true);
	return 1;
}

int oracle_pt_iterate_rows(void* p, int32_t nt, uint32_t y0, uint32_t y1) {
	PtState* st = static_cast<PtState*>(p);
	if(y1 > st->scene->height) y1 = st->scene->height;
	if(y0 >= y1) return 0;
	pt_iterate(*st, nt > 0 ? nt : 1, y0, y1, false);
	return 1;
}

int oracle_pt_get_target(void* p, int32_t target, float* out) {
	PtState* st = static_cast<PtState*>(p);
	// 0 Radiance, 1 Hit ID; 2 and 3 their variances; 4..9 Position, Depth,
	// Normal, UV, Albedo, Lightness and 10..15 their variances
	const std::vector<float>* v = target == 0 ? &st->radiance : target == 1 ? &st->hitId
	                            : target == 2 ? &st->radianceVar : target == 3 ? &st->hitIdVar : nullptr;
	if(v) { std::memcpy(out, v->data(), v->size() * 4); return 1; }
	if(target < 4 || target > 15) return 0;
	static const int first[6] = { AUX_POS, AUX_DEPTH, AUX_NORMAL, AUX_UV, AUX_ALBEDO, AUX_LIGHT };
	static const int count[6] = { 3, 1, 3, 2, 3, 1 };
	const int a = (target - 4) % 6;
	const std::vector<float>& src = target < 10 ? st->aux : st->auxVar;
	const size_t num = src.size() / AUX_CHANNELS;
	for(size_t p = 0; p < num; ++p)
		for(int c = 0; c < count[a]; ++c) out[p * size_t(count[a]) + size_t(c)] = src[p * AUX_CHANNELS + size_t(first[a] + c)];
	return 1;
}

int oracle_pt_stats(void* p, OrStats* o) {
	PtState* st = static_cast<PtState*>(p);
	o->rays = st->stats.rays; o->shadowRays = st->stats.shadowRays;
	o->nodeVisits = st->stats.nodeVisits; o->instanceVisits = st->stats.instanceVisits;
	o->triTests = st->stats.tri; o->quadTests = st->stats.quad; o->sphereTests = st->stats.sphere;
	return 1;
}

void* oracle_lt_create(void* s, const OrLtParams* params) {
	Scene* S = static_cast<Scene*>(s);
	auto* st = new LtState();
	st->scene = S;
	st->params = *params;
	const i32 num = i32(S->width * S->height);
	st->rngs.resize(size_t(num));
	// cpu_lt.cpp:33-38
	const i32 seed = i32(u32(params->seed) * u32(num + 1));
	for(i32 i = 0; i < num; ++i) st->rngs[size_t(i)] = Pcg64::seeded(u32(i32(u32(i) + u32(seed))));
	st->radiance.assign(size_t(num) * 3, 0.0f);
	st->lightness.assign(size_t(num), 0.0f);
	st->density.assign(size_t(num), 0.0f);
	st->radianceVar.assign(size_t(num) * 3, 0.0f);
	st->lightnessVar.assign(size_t(num), 0.0f);
	st->densityMean.assign(size_t(num), 0.0f);
	return st;
}

void oracle_lt_destroy(void* p) { delete static_cast<LtState*>(p); }

int oracle_lt_iterate(void* p, int32_t nt) {
	lt_iterate(*static_cast<LtState*>(p), nt > 0 ? nt : 1);
	return 1;
}

int oracle_lt_get_target(void* p, int32_t target, float* out) {
	const LtState* st = static_cast<const LtState*>(p);
	// 0 Radiance, 1 Lightness, 2 Density; 3, 4, 5 their variance buffers
	const std::vector<float>* v = target == 0 ? &st->radiance : target == 1 ? &st->lightness : target == 2 ? &st->density
	                            : target == 3 ? &st->radianceVar : target == 4 ? &st->lightnessVar
	                            : target == 5 ? &st->densityMean : nullptr;
	if(!v) return 0;
	std::memcpy(out, v->data(), v->size() * 4);
	return 1;
}

int oracle_lt_records(void* p, int32_t* pixels, float* values) {
	const LtState* st = static_cast<const LtState*>(p);
	if(st->iteration < 0) return 0;
	std::memcpy(pixels, st->recPixel.data(), st->recPixel.size() * 4);
	std::memcpy(values, st->recValue.data(), st->recValue.size() * 4);
	return 1;
}

int oracle_lt_stats(void* p, OrStats* o) {
	const LtState* st = static_cast<const LtState*>(p);
	o->rays = st->stats.rays; o->shadowRays = st->stats.shadowRays;
	o->nodeVisits = st->stats.nodeVisits; o->instanceVisits = st->stats.instanceVisits;
	o->triTests = st->stats.tri; o->quadTests = st->stats.quad; o->sphereTests = st->stats.sphere;
	return 1;
}

void* oracle_bpt_create(void* s, const OrLtParams* params) {
	Scene* S = static_cast<Scene*>(s);
	auto* st = new BptState();
	st->scene = S;
	st->params = *params;
	const i32 num = i32(S->width * S->height);
	st->rngs.resize(size_t(num));
	// cpu_bpt.cpp:239-244
	const i32 seed = i32(u32(params->seed) * u32(num + 1));
	for(i32 i = 0; i < num; ++i) st->rngs[size_t(i)] = Pcg64::seeded(u32(i32(u32(i) + u32(seed))));
	st->radiance.assign(size_t(num) * 3, 0.0f);
	st->lightness.assign(size_t(num), 0.0f);
	st->radianceVar.assign(size_t(num) * 3, 0.0f);
	st->lightnessVar.assign(size_t(num), 0.0f);
	return st;
}

void oracle_bpt_destroy(void* p) { delete static_cast<BptState*>(p); }

int oracle_bpt_iterate(void* p, int32_t nt) {
	bpt_iterate(*static_cast<BptState*>(p), nt > 0 ? nt : 1);
	return 1;
}

int oracle_bpt_get_target(void* p, int32_t target, float* out) {
	const BptState* st = static_cast<const BptState*>(p);
	// 0 Radiance, 1 Lightness; 2, 3 their variances
	const std::vector<float>* v = target == 0 ? &st->radiance : target == 1 ? &st->lightness
	                            : target == 2 ? &st->radianceVar : target == 3 ? &st->lightnessVar : nullptr;
	if(!v) return 0;
	std::memcpy(out, v->data(), v->size() * 4);
	return 1;
}

int oracle_bpt_records(void* p, int32_t* pixels, float* values) {
	const BptState* st = static_cast<const BptState*>(p);
	if(st->iteration < 0) return 0;
	std::memcpy(pixels, st->recPixel.data(), st->recPixel.size() * 4);
	std::memcpy(values, st->recValue.data(), st->recValue.size() * 4);
	return 1;
}

int oracle_bpt_stats(void* p, OrStats* o) {
	const BptState* st = static_cast<const BptState*>(p);
	o->rays = st->stats.rays; o->shadowRays = st->stats.shadowRays;
	o->nodeVisits = st->stats.nodeVisits; o->instanceVisits = st->stats.instanceVisits;
	o->triTests = st->stats.tri; o->quadTests = st->stats.quad; o->sphereTests = st->stats.sphere;
	return 1;
}

void* oracle_vcm_create(void* s, const OrLtParams* params, float mergeRadius, int32_t progressive) {
	Scene* S = static_cast<Scene*>(s);
	auto* st = new VcmState();
	st->scene = S;
	st->params = *params;
	st->mergeRadius = mergeRadius;
	st->progressive = progressive != 0;
	const i32 num = i32(S->width * S->height);
	st->rngs.resize(size_t(num));
	// cpu_vcm.cpp:292-297
	const i32 seed = i32(u32(params->seed) * u32(num + 1));
	for(i32 i = 0; i < num; ++i) st->rngs[size_t(i)] = Pcg64::seeded(u32(i32(u32(i) + u32(seed))));
	st->radiance.assign(size_t(num) * 3, 0.0f);
	st->lightness.assign(size_t(num), 0.0f);
	st->radianceVar.assign(size_t(num) * 3, 0.0f);
	st->lightnessVar.assign(size_t(num), 0.0f);
	return st;
}

void oracle_vcm_destroy(void* p) { delete static_cast<VcmState*>(p); }

int oracle_vcm_iterate(void* p, int32_t nt) {
	vcm_iterate(*static_cast<VcmState*>(p), nt > 0 ? nt : 1);
	return 1;
}

int oracle_vcm_get_target(void* p, int32_t target, float* out) {
	const VcmState* st = static_cast<const VcmState*>(p);
	const std::vector<float>* v = target == 0 ? &st->radiance : target == 1 ? &st->lightness
	                            : target == 2 ? &st->radianceVar : target == 3 ? &st->lightnessVar : nullptr;
	if(!v) return 0;
	std::memcpy(out, v->data(), v->size() * 4);
	return 1;
}

int oracle_vcm_records(void* p, int32_t* pixels, float* values) {
	const VcmState* st = static_cast<const VcmState*>(p);
	if(st->iteration < 0) return 0;
	std::memcpy(pixels, st->recPixel.data(), st->recPixel.size() * 4);
	std::memcpy(values, st->recValue.data(), st->recValue.size() * 4);
	return 1;
}

int oracle_vcm_stats(void* p, OrStats* o) {
	const VcmState* st = static_cast<const VcmState*>(p);
	o->rays = st->stats.rays; o->shadowRays = st->stats.shadowRays;
	o->nodeVisits = st->stats.nodeVisits; o->instanceVisits = st->stats.instanceVisits;
	o->triTests = st->stats.tri; o->quadTests = st->stats.quad; o->sphereTests = st->stats.sphere;
	return 1;
}

uint32_t oracle_vcm_map_size(uint32_t capacity) { return vcm_map_size(capacity); }
uint32_t oracle_wang_hash(uint32_t x) { return wang_hash(x); }

void* oracle_wireframe_create(void* s, float lineWidth, int32_t maxTraceDepth) {
	Scene* S = static_cast<Scene*>(s);
	auto* st = new WireState();
	st->scene = S;
	st->lineWidth = lineWidth;
	st->maxTraceDepth = maxTraceDepth;
	const i32 num = i32(S->width * S->height);
	st->rngs.resize(size_t(num));
	for(i32 i = 0; i < num; ++i) st->rngs[size_t(i)] = Pcg64::seeded(u32(i)); // cpu_wireframe.cpp:31-36
	st->border.assign(size_t(num) * 3, 0.0f);
	st->borderVar.assign(size_t(num) * 3, 0.0f);
	return st;
}
void oracle_wireframe_destroy(void* p) { delete static_cast<WireState*>(p); }
int oracle_wireframe_iterate(void* p, int32_t nt) { wireframe_iterate(*static_cast<WireState*>(p), nt > 0 ? nt : 1); return 1; }
int oracle_wireframe_get_target(void* p, float* out) {
	const WireState* st = static_cast<const WireState*>(p);
	std::memcpy(out, st->border.data(), st->border.size() * 4);
	return 1;
}
int oracle_wireframe_get_variance(void* p, float* out) {
	const WireState* st = static_cast<const WireState*>(p);
	std::memcpy(out, st->borderVar.data(), st->borderVar.size() * 4);
	return 1;
}

int oracle_karras(const uint64_t* keys, int32_t n, int32_t* parents) {
	if(n < 2) return 0;
	std::vector<u64> k(keys, keys + n);
	std::vector<i32> p(size_t(2 * n - 1), 0);
	for(i32 i = 0; i < n - 1; ++i) karras_node(k, n, p, i);
	std::memcpy(parents, p.data(), p.size() * 4);
	return 1;
}

uint64_t oracle_pcg64_seed(uint32_t seed) { return Pcg64::seeded(seed).state; }
uint64_t oracle_pcg64_next(uint64_t* state) { Pcg64 r; r.state = *state; u64 v = r.next(); *state = r.state; return v; }
uint64_t oracle_part_by_two21(uint32_t x) { return part_by_two21(x); }
uint32_t oracle_part_by_two10(uint32_t x) { return part_by_two10(x); }
uint64_t oracle_scramble_seed(uint32_t x) { return scramble_seed(x); }
void oracle_golden_ratio2d(uint32_t seed, uint32_t n, uint64_t* out) {
	u64 state = scramble_seed(seed);
	for(uint32_t i = 0; i < n; ++i) out[i] = golden_ratio2d_next(state);
}
uint64_t oracle_part_by_two16(uint32_t x) { return part_by_two16(x); }
uint64_t oracle_morton_code16(uint32_t a, uint32_t b, uint32_t c) { return morton_code16(a, b, c); }
uint64_t oracle_hilbert_code16(uint32_t a, uint32_t b, uint32_t c) { return hilbert_code16(a, b, c); }
void oracle_sincos(float x, float* s, float* c) { mbmath::sincos(x, *s, *c); }
float oracle_atan2(float y, float x) { return mbmath::atan2(y, x); }
float oracle_acos(float x) { return mbmath::acos(x); }

} // extern "C"
