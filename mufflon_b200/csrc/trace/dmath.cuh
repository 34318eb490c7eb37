// Device vector math for the path tracer.
//
// Every operation here is written so that its float rounding sequence is
// fixed: the file is compiled with --fmad=false (no implicit contraction) and
// FMAs appear only where written explicitly. Sums are evaluated left to right
// (dot(a, b) = (a.x*b.x + a.y*b.y) + a.z*b.z), division and square root are
// IEEE round-to-nearest. This is what makes the CUDA path tracer reproduce
// the CPU oracle bit for bit.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>
#include "../common/fmath.hpp"

namespace mb {

using u16 = uint16_t;
using u32 = uint32_t;
using u64 = uint64_t;
using i32 = int32_t;

constexpr float PI = 3.14159265358979f;
constexpr float MAX_SCENE_SIZE = 1048576.0f;
constexpr float SCENE_SCALE_EPS = 1e-4f;
constexpr float INF_PDF = 4294967296.0f;
// Box culling uses tmax * (1 + 2^-16) so that it never culls a primitive the
// exact (t, instance, primitive) ordering would accept.
constexpr float BOX_SLACK = 1.0f + 1.0f / 4096.0f;      // tmax culling slack
constexpr float BOX_FAR_SLACK = 1.0f + 1.0f / 1048576.0f; // slab interval tolerance
constexpr float DISTANCESQ_EPSILON = 1e-10f;

#define MBD __device__ __forceinline__

struct f2 { float x, y; };
struct f3 {
	float x, y, z;
	MBD float operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
};

MBD f3 make3(float x, float y, float z) { f3 r; r.x = x; r.y = y; r.z = z; return r; }
MBD f2 make2(float x, float y) { f2 r; r.x = x; r.y = y; return r; }
MBD f3 operator+(f3 a, f3 b) { return make3(a.x + b.x, a.y + b.y, a.z + b.z); }
MBD f3 operator-(f3 a, f3 b) { return make3(a.x - b.x, a.y - b.y, a.z - b.z); }
MBD f3 operator-(f3 a) { return make3(-a.x, -a.y, -a.z); }
MBD f3 operator*(f3 a, f3 b) { return make3(a.x * b.x, a.y * b.y, a.z * b.z); }
MBD f3 operator*(f3 a, float s) { return make3(a.x * s, a.y * s, a.z * s); }
MBD f3 operator*(float s, f3 a) { return make3(s * a.x, s * a.y, s * a.z); }
MBD f3 operator/(f3 a, float s) { return make3(__fdiv_rn(a.x, s), __fdiv_rn(a.y, s), __fdiv_rn(a.z, s)); }
MBD f2 operator+(f2 a, f2 b) { return make2(a.x + b.x, a.y + b.y); }
MBD f2 operator-(f2 a, f2 b) { return make2(a.x - b.x, a.y - b.y); }
MBD f2 operator*(f2 a, float s) { return make2(a.x * s, a.y * s); }
MBD f2 operator*(float s, f2 a) { return make2(s * a.x, s * a.y); }
MBD float dot(f3 a, f3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
MBD f3 cross(f3 a, f3 b) {
	return make3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
MBD float lensq(f3 a) { return dot(a, a); }
MBD float len(f3 a) { return __fsqrt_rn(lensq(a)); }
MBD f3 normalize(f3 a) { return a / len(a); }
MBD float fmin_(float a, float b) { return fminf(a, b); }
MBD float fmax_(float a, float b) { return fmaxf(a, b); }
MBD f3 vmin(f3 a, f3 b) { return make3(fmin_(a.x, b.x), fmin_(a.y, b.y), fmin_(a.z, b.z)); }
MBD f3 vmax(f3 a, f3 b) { return make3(fmax_(a.x, b.x), fmax_(a.y, b.y), fmax_(a.z, b.z)); }
MBD float maxc(f3 a) { return fmax_(fmax_(a.x, a.y), a.z); }
MBD float sgn(float x) { return x < 0.0f ? -1.0f : 1.0f; }
MBD float div_(float a, float b) { return __fdiv_rn(a, b); }
MBD float sqrt_(float a) { return __fsqrt_rn(a); }
MBD float sdiv(float x, float d) { return __fdiv_rn(x, d + 1e-20f * sgn(d)); }
MBD bool any_pos(f3 a) { return a.x > 0.0f || a.y > 0.0f || a.z > 0.0f; }
MBD bool nonzero(f3 a) { return a.x != 0.0f || a.y != 0.0f || a.z != 0.0f; }
MBD f3 load3(const float* p) { return make3(p[0], p[1], p[2]); }
MBD f3 ldg3(const float* p) { return make3(__ldg(p), __ldg(p + 1), __ldg(p + 2)); }
MBD f2 ldg2(const float* p) { return make2(__ldg(p), __ldg(p + 1)); }
MBD f3 f4to3(float4 v) { return make3(v.x, v.y, v.z); }

// ---------------------------------------------------------------- rng
// PCG64 with RXS-M-XS output (src/core/math/rng.hpp:184-207) and SplitMix64
// seeding (rng.hpp:126-131).
MBD u64 scramble_seed(u32 x) {
	u64 z = u64(x) + 0x9e3779b97f4a7c15ull;
	z = (z ^ (z >> 30u)) * 0xbf58476d1ce4e5b9ull;
	z = (z ^ (z >> 27u)) * 0x94d049bb133111ebull;
	return z ^ (z >> 31u);
}
MBD u64 pcg_next(u64& state) {
	u64 x = state;
	const u64 count = state >> 59ull;
	state = state * 6364136223846793005ull + 1442695040888963407ull;
	x ^= x >> (5 + count);
	x *= 12605985483714917081ull;
	return x ^ (x >> 43);
}
MBD u64 pcg_seed(u32 seed) {
	u64 s = scramble_seed(seed);
	pcg_next(s);
	s += seed;
	pcg_next(s);
	return s;
}
// sampling.hpp:23-29
MBD float sample_uniform(u32 u) { return __fdiv_rn(float(u), 4294967810.0f); }
// sampling.hpp:39-46
MBD u64 percentage_of(u64 num, float p) {
	u64 pfix = u64(p * 2147483648.0f);
	return ((pfix * (num & 0x7fffffff)) >> 31) + (pfix * (num >> 31));
}

} // namespace mb
