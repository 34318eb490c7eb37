// Scalar transcendental functions shared bit-for-bit between the CUDA path
// tracer and its CPU oracle.
//
// Why this exists: the path tracer's sampling routines call sin/cos
// (cosine-weighted hemisphere sampling, uniform sphere sampling, GGX slope
// sampling at normal incidence). CUDA's sinf/cosf and glibc's sinf/cosf are
// different implementations and may differ in the last bit. One differing bit
// in a sampled direction changes a later Russian-roulette decision or a hit
// on an edge, so per-image radiance would no longer be reproducible between
// the CPU oracle and the GPU. Both sides therefore call these functions,
// which are compiled from the same source with the same operation order
// (explicit fmaf, no other contraction) and so round identically on host and
// device.
//
// Method (written from the mathematics, not taken from any library):
//   * argument reduction by k = rint(x * 2/pi) and a three-part Cody-Waite
//     split of pi/2 (12 + 12 + 24 significant bits, so k * hi is exact for
//     |k| < 4096);
//   * on the reduced argument r in [-pi/4, pi/4] the Taylor series of sin
//     up to r^9 and of cos up to r^10; the first omitted terms are below
//     2e-9 relative, i.e. far below half an ulp of float;
//   * quadrant selection by k mod 4.
// Accuracy is checked against libm in tests/test_oracle_math.py (max error
// 2 ulp over [-8*pi, 8*pi]).
#pragma once

#include <cstdint>
#include <cmath>

#if defined(__CUDACC__)
#define MB_HD __host__ __device__ __forceinline__
#else
#define MB_HD inline
#endif

namespace mbmath {

// pi/2 = PIO2_A + PIO2_B + PIO2_C (+ below float precision)
constexpr float PIO2_A = 1.5703125f;              // 0x3FC90000
constexpr float PIO2_B = 4.837512969970703e-04f;  // 0x39FDA000
constexpr float PIO2_C = 7.549790126404332e-08f;  // 0x33A22169
constexpr float TWO_OVER_PI = 0.6366197466850281f;

// Taylor coefficients (-1)^n / (2n+1)!  and  (-1)^n / (2n)!
constexpr float S3 = -0.1666666716337204f;
constexpr float S5 = 0.008333333767950535f;
constexpr float S7 = -0.00019841270113829523f;
constexpr float S9 = 2.7557318844628753e-06f;
constexpr float C4 = 0.0416666679084301f;
constexpr float C6 = -0.0013888889225199819f;
constexpr float C8 = 2.4801587642286904e-05f;
constexpr float C10 = -2.755731998149713e-07f;

MB_HD float fma_(float a, float b, float c) {
#if defined(__CUDA_ARCH__)
	return __fmaf_rn(a, b, c);
#else
	return std::fmaf(a, b, c);
#endif
}

MB_HD float rint_(float x) {
#if defined(__CUDA_ARCH__)
	return rintf(x);
#else
	return std::nearbyint(x);
#endif
}

// sin(r), cos(r) for |r| <= pi/4 (slightly beyond is fine).
MB_HD void sincos_kernel(float r, float& s, float& c) {
	const float r2 = r * r;
	float p = fma_(r2, S9, S7);
	p = fma_(r2, p, S5);
	p = fma_(r2, p, S3);
	s = fma_(r * r2, p, r);
	float q = fma_(r2, C10, C8);
	q = fma_(r2, q, C6);
	q = fma_(r2, q, C4);
	q = fma_(r2, q, -0.5f);
	c = fma_(r2, q, 1.0f);
}

// Sine and cosine of x, |x| < 4096 * pi/2.
MB_HD void sincos(float x, float& s, float& c) {
	const float k = rint_(x * TWO_OVER_PI);
	float r = x - k * PIO2_A;
	r = r - k * PIO2_B;
	r = fma_(-k, PIO2_C, r);
	float sr, cr;
	sincos_kernel(r, sr, cr);
	const int q = static_cast<int>(k) & 3;
	switch(q) {
		case 0: s = sr; c = cr; break;
		case 1: s = cr; c = -sr; break;
		case 2: s = -sr; c = -cr; break;
		default: s = -cr; c = sr; break;
	}
}

MB_HD float sin(float x) { float s, c; sincos(x, s, c); return s; }
MB_HD float cos(float x) { float s, c; sincos(x, s, c); return c; }

// Correctly rounded square root on both sides (IEEE sqrtf; nvcc without
// fast-math uses the round-to-nearest form).
MB_HD float sqrt(float x) {
#if defined(__CUDA_ARCH__)
	return __fsqrt_rn(x);
#else
	return std::sqrt(x);
#endif
}

MB_HD float div(float a, float b) {
#if defined(__CUDA_ARCH__)
	return __fdiv_rn(a, b);
#else
	return a / b;
#endif
}

// arctan on [-1, 1] via two half-angle reductions
// atan(x) = 2 atan(x / (1 + sqrt(1 + x^2))) followed by the alternating
// series to x^15; used only for texture coordinates of sphere hits.
MB_HD float atan_unit(float x) {
	float y = div(x, 1.0f + sqrt(fma_(x, x, 1.0f)));
	y = div(y, 1.0f + sqrt(fma_(y, y, 1.0f)));
	// |y| <= tan(pi/16) ~ 0.199 -> y^17/17 < 7e-14
	const float y2 = y * y;
	float p = fma_(y2, -1.0f / 15.0f, 1.0f / 13.0f);
	p = fma_(y2, p, -1.0f / 11.0f);
	p = fma_(y2, p, 1.0f / 9.0f);
	p = fma_(y2, p, -1.0f / 7.0f);
	p = fma_(y2, p, 1.0f / 5.0f);
	p = fma_(y2, p, -1.0f / 3.0f);
	const float a = fma_(y * y2, p, y);
	return 4.0f * a;
}

constexpr float PI_F = 3.14159265358979f;

MB_HD float atan2(float y, float x) {
	if(x == 0.0f && y == 0.0f) return 0.0f;
	const float ax = x < 0.0f ? -x : x;
	const float ay = y < 0.0f ? -y : y;
	float a;
	if(ay <= ax) a = atan_unit(div(ay, ax));
	else a = 0.5f * PI_F - atan_unit(div(ax, ay));
	if(x < 0.0f) a = PI_F - a;
	return y < 0.0f ? -a : a;
}

// acos(x) = atan2(sqrt(1 - x^2), x)
MB_HD float acos(float x) {
	const float t = fma_(-x, x, 1.0f);
	return atan2(sqrt(t < 0.0f ? 0.0f : t), x);
}

} // namespace mbmath
