// GPU LBVH builder. See lbvh.hpp for the stage list.
//
// Semantics follow src/core/scene/accel_structs/build_lbvh.cu with these
// fixed choices (the CPU oracle makes the same ones):
//   * exact clz (the reference's Linux host path uses log2f),
//   * a stable (key, index) sort,
//   * the SAH cost of a node always adds the right child's term first, which
//     is what a sequential run of the reference's CPU loop produces; on the
//     GPU the arriving thread is arbitrary, so the order is fixed explicitly,
//   * child links are stored by the emit stage instead of being inferred from
//     the arrival flag, which removes the reference's leaf/internal ambiguity
//     for the last leaf's thread (build_lbvh.cu:365-374 compares a thread
//     index against numInternalNodes).
#include "lbvh.hpp"
#include "../trace/dmath.cuh"
#include "radix_sort.cuh"
#include "wide.hpp"

#include <algorithm>
#include <cfloat>

namespace mb {
namespace {

constexpr int32_t TREE_HEAD = 0x10000000;
constexpr int SCAN_THREADS = 1024;
// Upper bound on tree depth (63-bit codes + 32 index bits); climbs stop there.
constexpr int MAX_DEPTH = 256;
constexpr int SCAN_ITEMS = 4;
constexpr int SCAN_TILE = SCAN_THREADS * SCAN_ITEMS;

enum { MODE_LOD = 0, MODE_SCENE = 1 };

MBD float bmin(float a, float b) { return b < a ? b : a; }
MBD float bmax(float a, float b) { return a < b ? b : a; }
MBD f3 vmin3(f3 a, f3 b) { return make3(bmin(a.x, b.x), bmin(a.y, b.y), bmin(a.z, b.z)); }
MBD f3 vmax3(f3 a, f3 b) { return make3(bmax(a.x, b.x), bmax(a.y, b.y), bmax(a.z, b.z)); }

// sfcurves.hpp:35-44
MBD u64 part_by_two21(uint32_t x) {
	u64 r = x;
	r = (r | (r << 32)) & 0x001f00000000ffffull;
	r = (r | (r << 16)) & 0x001f0000ff0000ffull;
	r = (r | (r << 8)) & 0x100f00f00f00f00full;
	r = (r | (r << 4)) & 0x10c30c30c30c30c3ull;
	r = (r | (r << 2)) & 0x1249249249249249ull;
	return r;
}
MBD uint32_t disc21(float v) {
	float x = v * 2097152.0f;
	x = fminf(fmaxf(x, 0.0f), 2097151.0f);
	return uint32_t(x);
}
// build_lbvh.cu:71-85
MBD u64 morton63(f3 p, const float* mn, const float* mx) {
	const f3 lo = make3(mn[0], mn[1], mn[2]);
	const f3 span = make3(mx[0], mx[1], mx[2]) - lo;
	const f3 d = p - lo;
	const f3 n = make3(sdiv(d.x, span.x), sdiv(d.y, span.y), sdiv(d.z, span.z));
	return part_by_two21(disc21(n.x)) * 4 + part_by_two21(disc21(n.y)) * 2 + part_by_two21(disc21(n.z));
}

MBD f3 v3(const float* v, uint32_t i) { return make3(v[3 * size_t(i)], v[3 * size_t(i) + 1], v[3 * size_t(i) + 2]); }

// accel_structs_commons.hpp:56-80
MBD f3 lod_centroid(const LodBuildInput& in, int p) {
	const int sphOff = int(in.numTriangles + in.numQuads);
	if(p >= sphOff) { const float4 s = in.spheres[p - sphOff]; return make3(s.x, s.y, s.z); }
	if(p >= int(in.numTriangles)) {
		const uint32_t q = uint32_t(p - int(in.numTriangles)) * 4 + in.numTriangles * 3;
		return (((v3(in.vertices, in.indices[q]) + v3(in.vertices, in.indices[q + 1])) + v3(in.vertices, in.indices[q + 2]))
			+ v3(in.vertices, in.indices[q + 3])) / 4.0f;
	}
	const uint32_t t = uint32_t(p) * 3;
	return ((v3(in.vertices, in.indices[t]) + v3(in.vertices, in.indices[t + 1])) + v3(in.vertices, in.indices[t + 2])) / 3.0f;
}

// accel_structs_commons.hpp:85-103
MBD void lod_box(const LodBuildInput& in, int p, f3& mn, f3& mx) {
	const int sphOff = int(in.numTriangles + in.numQuads);
	if(p >= sphOff) {
		const float4 s = in.spheres[p - sphOff];
		const f3 c = make3(s.x, s.y, s.z);
		mn = c - make3(s.w, s.w, s.w);
		mx = c + make3(s.w, s.w, s.w);
		return;
	}
	mn = make3(FLT_MAX, FLT_MAX, FLT_MAX);
	mx = make3(-FLT_MAX, -FLT_MAX, -FLT_MAX);
	if(p >= int(in.numTriangles)) {
		const uint32_t q = uint32_t(p - int(in.numTriangles)) * 4 + in.numTriangles * 3;
		for(int k = 0; k < 4; ++k) { const f3 v = v3(in.vertices, in.indices[q + k]); mn = vmin3(mn, v); mx = vmax3(mx, v); }
		return;
	}
	const uint32_t t = uint32_t(p) * 3;
	for(int k = 0; k < 3; ++k) { const f3 v = v3(in.vertices, in.indices[t + k]); mn = vmin3(mn, v); mx = vmax3(mx, v); }
}

struct Counts { int c0, c1, c2; };

MBD int32_t encode_counts(int mode, Counts c) {
	if(mode == MODE_SCENE) return c.c0;
	return (min(c.c0, 0x3FF) << 20) | (min(c.c1, 0x3FF) << 10) | min(c.c2, 0x3FF);
}
MBD Counts decode_counts(int mode, int32_t v) {
	if(mode == MODE_SCENE) return { v, 0, 0 };
	return { (v & 0x3FF00000) >> 20, (v & 0x000FFC00) >> 10, v & 0x3FF };
}
// build_lbvh.cu:319-324 with the constants of build_lbvh.cu:35-48
MBD float get_cost(int mode, Counts c) {
	if(mode == MODE_SCENE) return 1.0f + float(c.c0) * 8.5f;
	return 2.0f + ((float(c.c0) * 1.2f + float(c.c1) * 4.0f) + float(c.c2) * 1.0f);
}
MBD bool count_limit(int mode, Counts c) {
	if(mode == MODE_SCENE) return c.c0 >= 1023;
	return c.c0 >= 1023 || c.c1 >= 1023 || c.c2 >= 1023;
}
// sfcurves.hpp:37-46 (10 bits to every third bit) and build_lbvh.cu:59-69:
// the 30-bit code, kept in the low bits of the 64-bit key. The hierarchy the
// Karras emit builds on it equals the one on 32-bit keys: every common-prefix
// length of two keys (and of two equal keys' indices) grows by the same 32
// bits, and the emit only compares such lengths.
MBD uint32_t part_by_two10(uint32_t x) {
	uint32_t r = x;
	r = (r * 0x00010001u) & 0xFF0000FFu;
	r = (r * 0x00000101u) & 0x0F00F00Fu;
	r = (r * 0x00000011u) & 0xC30C30C3u;
	r = (r * 0x00000005u) & 0x49249249u;
	return r;
}
MBD uint32_t disc10(float v) {
	float x = v * 1024.0f;
	x = fminf(fmaxf(x, 0.0f), 1023.0f);
	return uint32_t(x);
}
MBD u64 morton30(f3 p, const float* mn, const float* mx) {
	const f3 lo = make3(mn[0], mn[1], mn[2]);
	const f3 span = make3(mx[0], mx[1], mx[2]) - lo;
	const f3 d = p - lo;
	const f3 n = make3(sdiv(d.x, span.x), sdiv(d.y, span.y), sdiv(d.z, span.z));
	return u64(part_by_two10(disc10(n.x)) * 4u + part_by_two10(disc10(n.y)) * 2u + part_by_two10(disc10(n.z)));
}

MBD float surface(f3 mn, f3 mx) {
	const f3 d = mx - mn;
	return 2.0f * (d.x * d.y + d.x * d.z + d.y * d.z);
}

// ---------------------------------------------------------------- Morton
__global__ void k_morton_lod(LodBuildInput in, uint32_t n, u64* keys, int32_t* vals, int bits) {
	const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
	if(i >= n) return;
	const f3 c = lod_centroid(in, int(i));
	keys[i] = bits == 30 ? morton30(c, in.aabbMin, in.aabbMax) : morton63(c, in.aabbMin, in.aabbMax);
	vals[i] = int32_t(i);
}

__global__ void k_morton_scene(SceneBuildInput in, uint32_t n, u64* keys, int32_t* vals, int bits) {
	const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
	if(i >= n) return;
	if(in.instanceLod[i] == 0xFFFFFFFFu) keys[i] = bits == 30 ? u64(0xFFFFFFFFu) : ~0ull;
	else {
		const f3 c = v3(in.instCentroids, i);
		keys[i] = bits == 30 ? morton30(c, in.aabbMin, in.aabbMax) : morton63(c, in.aabbMin, in.aabbMax);
	}
	vals[i] = int32_t(i);
}

// ---------------------------------------------------------------- Karras
MBD int lcp(const u64* keys, int n, int i1, int i2, u64 key1) {
	if(i2 < 0 || i2 >= n) return -1;
	const u64 key2 = keys[i2];
	if(key1 == key2) return 64 + __clz(int(uint32_t(i1 ^ i2)));
	return __clzll((long long)(key1 ^ key2));
}

// build_lbvh.cu:180-245 (plus explicit child links and mark initialisation)
__global__ void k_karras(int n, const u64* __restrict__ keys, int32_t* parents, int32_t* children, int32_t* marks,
                         int2* ranges) {
	const int idx = blockIdx.x * blockDim.x + threadIdx.x;
	if(idx >= n - 1) return;
	const u64 key1 = keys[idx];
	const int lcp1 = lcp(keys, n, idx, idx + 1, key1);
	const int lcp2 = lcp(keys, n, idx, idx - 1, key1);
	const int direction = (lcp1 - lcp2) < 0 ? -1 : 1;
	const int minLcp = lcp(keys, n, idx, idx - direction, key1);
	int lMax = 2;
	while(lcp(keys, n, idx, idx + lMax * direction, key1) > minLcp) lMax *= 2;
	int l = 0;
	for(int t = lMax; t > 1;) {
		t = t / 2;
		if(lcp(keys, n, idx, idx + (l + t) * direction, key1) > minLcp) l += t;
	}
	const int j = idx + l * direction;
	const int nodeLcp = lcp(keys, n, idx, j, key1);
	int s = 0;
	const int maxDivisor = 1 << (32 - __clz(l));
	for(int divisor = 2; divisor <= maxDivisor; divisor *= 2) {
		const int t = (l + divisor - 1) / divisor;
		if(lcp(keys, n, idx, idx + (s + t) * direction, key1) > nodeLcp) s += t;
	}
	const int split = idx + s * direction + min(direction, 0);
	const int leftIndex = (min(idx, j) == split) ? split + n - 1 : split;
	const int rightIndex = (max(idx, j) == split + 1) ? split + n : split + 1;
	parents[leftIndex] = ~idx;
	parents[rightIndex] = idx;
	if(idx == 0) parents[0] = TREE_HEAD;
	children[2 * idx] = leftIndex;
	children[2 * idx + 1] = rightIndex;
	marks[idx] = 1;
	ranges[idx] = make_int2(min(idx, j), max(idx, j));
}

// ---------------------------------------------------------------- merge
// build_lbvh.cu:326-411: one thread per leaf climbs while it is the second
// child to arrive at a node.
// Arrival counter of the bottom-up passes: an acquire-release atomic add.
MBD unsigned arrive(unsigned int* flag) {
	unsigned prev;
	asm volatile("atom.acq_rel.gpu.global.add.u32 %0, [%1], 1;" : "=r"(prev) : "l"(flag) : "memory");
	return prev;
}

__global__ void k_bbox(int mode, LodBuildInput lod, SceneBuildInput scene, int used, int numInternal,
                       const int32_t* __restrict__ primIds, const int32_t* __restrict__ parents,
                       const int32_t* __restrict__ children, float4* nodeData, unsigned int* flags) {
	const int i = blockIdx.x * blockDim.x + threadIdx.x;
	if(i >= used) return;
	const int prim = primIds[i];
	const int leaf = numInternal + i;
	f3 mn, mx;
	Counts c;
	if(mode == MODE_SCENE) {
		const float* b = scene.instBoxes + 6 * size_t(prim);
		mn = make3(b[0], b[1], b[2]);
		mx = make3(b[3], b[4], b[5]);
		c = { 1, 0, 0 };
	} else {
		lod_box(lod, prim, mn, mx);
		const int sphOff = int(lod.numTriangles + lod.numQuads);
		if(prim >= sphOff) c = { 0, 0, 1 };
		else if(prim >= int(lod.numTriangles)) c = { 0, 1, 0 };
		else c = { 1, 0, 0 };
	}
	nodeData[2 * leaf] = make_float4(mn.x, mn.y, mn.z, __int_as_float(encode_counts(mode, c)));
	nodeData[2 * leaf + 1] = make_float4(mx.x, mx.y, mx.z, get_cost(mode, c));
	int cur = parents[leaf];
	if(cur < 0) cur = ~cur;
	const float nodeCost = mode == MODE_SCENE ? 1.0f : 2.0f;
	for(int depth = 0; depth < MAX_DEPTH; ++depth) {
		// first arrival: the sibling's thread continues; acquire-release on the
		// flag orders this thread's node writes before it and the sibling's
		// reads after it (two full fences per level measured 20 % slower)
		const unsigned prev = arrive(flags + cur);
		if(prev == 0) return;
		const int L = children[2 * cur], R = children[2 * cur + 1];
		const float4 l0 = __ldcg(&nodeData[2 * L]), l1 = __ldcg(&nodeData[2 * L + 1]);
		const float4 r0 = __ldcg(&nodeData[2 * R]), r1 = __ldcg(&nodeData[2 * R + 1]);
		const f3 lmn = make3(l0.x, l0.y, l0.z), lmx = make3(l1.x, l1.y, l1.z);
		const f3 rmn = make3(r0.x, r0.y, r0.z), rmx = make3(r1.x, r1.y, r1.z);
		const float saR = surface(rmn, rmx);
		const f3 nmn = vmin3(rmn, lmn), nmx = vmax3(rmx, lmx);
		const float newSA = surface(nmn, nmx);
		const float saL = surface(lmn, lmx);
		const Counts cR = decode_counts(mode, __float_as_int(r0.w));
		const Counts cL = decode_counts(mode, __float_as_int(l0.w));
		const float cost = (nodeCost + __fdiv_rn(saR, newSA) * get_cost(mode, cR)) + __fdiv_rn(saL, newSA) * get_cost(mode, cL);
		const Counts cn = { cR.c0 + cL.c0, cR.c1 + cL.c1, cR.c2 + cL.c2 };
		nodeData[2 * cur] = make_float4(nmn.x, nmn.y, nmn.z, __int_as_float(encode_counts(mode, cn)));
		nodeData[2 * cur + 1] = make_float4(nmx.x, nmx.y, nmx.z, cost);
		if(cur == 0) return;
		cur = parents[cur];
		if(cur < 0) cur = ~cur;
	}
}

// Refits the binary hierarchy's node boxes (xyz only; counts and costs in .w
// stay) to other leaf boxes, bottom-up as k_bbox: for the 8-wide conversion of
// the instance level, after the reference-layout nodes have been emitted.
__global__ void k_refit_boxes(int used, int numInternal, const int32_t* __restrict__ primIds,
                              const int32_t* __restrict__ parents, const int32_t* __restrict__ children,
                              const float* __restrict__ boxes, float4* nodeData, unsigned int* flags) {
	const int i = blockIdx.x * blockDim.x + threadIdx.x;
	if(i >= used) return;
	const float* b = boxes + 6 * size_t(primIds[i]);
	const int leaf = numInternal + i;
	nodeData[2 * leaf] = make_float4(b[0], b[1], b[2], nodeData[2 * leaf].w);
	nodeData[2 * leaf + 1] = make_float4(b[3], b[4], b[5], nodeData[2 * leaf + 1].w);
	int cur = parents[leaf];
	if(cur < 0) cur = ~cur;
	for(int depth = 0; depth < MAX_DEPTH; ++depth) {
		const unsigned prev = arrive(flags + cur);
		if(prev == 0) return;
		const int L = children[2 * cur], R = children[2 * cur + 1];
		const float4 l0 = __ldcg(&nodeData[2 * L]), l1 = __ldcg(&nodeData[2 * L + 1]);
		const float4 r0 = __ldcg(&nodeData[2 * R]), r1 = __ldcg(&nodeData[2 * R + 1]);
		const f3 nmn = vmin3(make3(r0.x, r0.y, r0.z), make3(l0.x, l0.y, l0.z));
		const f3 nmx = vmax3(make3(r1.x, r1.y, r1.z), make3(l1.x, l1.y, l1.z));
		nodeData[2 * cur] = make_float4(nmn.x, nmn.y, nmn.z, nodeData[2 * cur].w);
		nodeData[2 * cur + 1] = make_float4(nmx.x, nmx.y, nmx.z, nodeData[2 * cur + 1].w);
		if(cur == 0) return;
		cur = parents[cur];
		if(cur < 0) cur = ~cur;
	}
}

// build_lbvh.cu:417-463
__global__ void k_mark(int mode, int used, int numInternal, const int32_t* __restrict__ parents,
                       const float4* __restrict__ nodeData, int32_t* marks) {
	const int i = blockIdx.x * blockDim.x + threadIdx.x;
	if(i >= used) return;
	const int leaf = numInternal + i;
	int collapseNode = -1;
	int cur = parents[leaf];
	if(cur < 0) cur = ~cur;
	for(int depth = 0; cur != 0 && depth < MAX_DEPTH; ++depth) {
		const float4 d0 = nodeData[2 * cur];
		const float4 d1 = nodeData[2 * cur + 1];
		const Counts c = decode_counts(mode, __float_as_int(d0.w));
		if(count_limit(mode, c)) break;
		if(get_cost(mode, c) < d1.w) collapseNode = cur;
		cur = parents[cur];
		if(cur < 0) cur = ~cur;
	}
	if(collapseNode != -1) {
		cur = parents[leaf];
		if(cur < 0) cur = ~cur;
		for(int depth = 0; cur != collapseNode && depth < MAX_DEPTH; ++depth) {
			marks[cur] = 0;
			cur = parents[cur];
			if(cur < 0) cur = ~cur;
		}
		marks[cur] = 0;
	}
}

// ---------------------------------------------------------------- scan
__global__ void k_scan_tiles(int32_t* data, int n, int32_t* blockSums) {
	__shared__ int32_t s[SCAN_THREADS];
	const int t = threadIdx.x;
	const int base = blockIdx.x * SCAN_TILE + t * SCAN_ITEMS;
	int32_t v[SCAN_ITEMS];
	int32_t sum = 0;
#pragma unroll
	for(int k = 0; k < SCAN_ITEMS; ++k) { v[k] = base + k < n ? data[base + k] : 0; sum += v[k]; v[k] = sum; }
	s[t] = sum;
	__syncthreads();
	for(int off = 1; off < SCAN_THREADS; off <<= 1) {
		const int32_t x = t >= off ? s[t - off] : 0;
		__syncthreads();
		s[t] += x;
		__syncthreads();
	}
	const int32_t prefix = s[t] - sum;
#pragma unroll
	for(int k = 0; k < SCAN_ITEMS; ++k) if(base + k < n) data[base + k] = v[k] + prefix;
	if(t == SCAN_THREADS - 1) blockSums[blockIdx.x] = s[t];
}

__global__ void k_scan_sums(int32_t* blockSums, int numBlocks) {
	// single block, sequential chunks of SCAN_THREADS
	__shared__ int32_t s[SCAN_THREADS];
	__shared__ int32_t carry;
	if(threadIdx.x == 0) carry = 0;
	__syncthreads();
	for(int base = 0; base < numBlocks; base += SCAN_THREADS) {
		const int t = threadIdx.x;
		const int32_t own = base + t < numBlocks ? blockSums[base + t] : 0;
		s[t] = own;
		__syncthreads();
		for(int off = 1; off < SCAN_THREADS; off <<= 1) {
			const int32_t x = t >= off ? s[t - off] : 0;
			__syncthreads();
			s[t] += x;
			__syncthreads();
		}
		if(base + t < numBlocks) blockSums[base + t] = carry + s[t] - own; // exclusive
		__syncthreads();
		if(t == SCAN_THREADS - 1) carry += s[t];
		__syncthreads();
	}
}

__global__ void k_scan_add(int32_t* data, int n, const int32_t* blockSums) {
	const int i = blockIdx.x * blockDim.x + threadIdx.x;
	if(i >= n) return;
	data[i] += blockSums[i / SCAN_TILE];
}

// ---------------------------------------------------------------- compaction
MBD bool is_collapsed(const int32_t* offsets, int numInternal, int node) {
	if(node > 0 && node < numInternal) return (offsets[node] - offsets[node - 1]) == 0;
	return false;
}

// build_lbvh.cu:511-566
__global__ void k_compact(int mode, int numNodes, int numInternal, const int32_t* __restrict__ parents,
                          const int32_t* __restrict__ offsets, const float4* __restrict__ nodeData,
                          BvhNode* out) {
	const int nd = blockIdx.x * blockDim.x + threadIdx.x + 1;
	if(nd >= numNodes) return;
	if(is_collapsed(offsets, numInternal, nd)) return;
	const int after = offsets[numInternal - 1];
	int parent = parents[nd];
	int offset;
	if(parent < 0) { offset = 0; parent = ~parent; } else offset = 1;
	int finalNode = nd;
	if(finalNode >= numInternal) {
		for(int depth = 0; is_collapsed(offsets, numInternal, parent); ++depth) {
			if(depth >= MAX_DEPTH) return;
			if(offset == 1) return;
			finalNode = parent;
			parent = parents[parent];
			if(parent < 0) { offset = 0; parent = ~parent; } else offset = 1;
		}
	}
	const float4 d0 = nodeData[2 * finalNode];
	const float4 d1 = nodeData[2 * finalNode + 1];
	const Counts c = decode_counts(mode, __float_as_int(d0.w));
	const int primCount = mode == MODE_SCENE ? c.c0 : (c.c0 + c.c1 + c.c2);
	const int outIdx = (offsets[parent] - 1) * 2;
	const int outNode = (nd >= numInternal) ? nd - numInternal + after : offsets[nd] - 1;
	const f3 mn = make3(d0.x, d0.y, d0.z), mx = make3(d1.x, d1.y, d1.z);
	const f3 ctr = (mn + mx) * 0.5f;
	const f3 bmn = (mn - ctr) * 1.0001f + ctr;
	const f3 bmx = (mx - ctr) * 1.0001f + ctr;
	BvhNode node;
	node.mn[0] = bmn.x; node.mn[1] = bmn.y; node.mn[2] = bmn.z;
	node.mx[0] = bmx.x; node.mx[1] = bmx.y; node.mx[2] = bmx.z;
	node.index = outNode;
	node.primCount = primCount;
	out[outIdx + offset] = node;
}

__global__ void k_after(const int32_t* offsets, int numInternal, int32_t* out) {
	*out = offsets[numInternal - 1];
}

// Leaf-ordered triangle soup: slot k holds primitive primIds[k].
__global__ void k_soup(LodBuildInput in, int n, const int32_t* __restrict__ primIds, float4* soup) {
	const int k = blockIdx.x * blockDim.x + threadIdx.x;
	if(k >= n) return;
	const int p = primIds[k];
	if(p >= int(in.numTriangles)) return;
	const uint32_t t = uint32_t(p) * 3;
#pragma unroll
	for(int j = 0; j < 3; ++j) {
		const f3 v = v3(in.vertices, in.indices[t + j]);
		soup[3 * size_t(k) + j] = make_float4(v.x, v.y, v.z, 0.0f);
	}
}

// Soup of the wide hierarchy's primitive order: slot k holds primitive
// wprims[k]; for triangles the three vertices, and the primitive id in the
// w component of the first float4 for every primitive type.
__global__ void k_wsoup(LodBuildInput in, int n, const int32_t* __restrict__ wprims, float4* soup) {
	const int k = blockIdx.x * blockDim.x + threadIdx.x;
	if(k >= n) return;
	const int p = wprims[k];
	float4 a = make_float4(0.0f, 0.0f, 0.0f, __int_as_float(p)), b = make_float4(0, 0, 0, 0), c = b;
	if(p < int(in.numTriangles)) {
		const uint32_t t = uint32_t(p) * 3;
		const f3 v0 = v3(in.vertices, in.indices[t]), v1 = v3(in.vertices, in.indices[t + 1]), v2 = v3(in.vertices, in.indices[t + 2]);
		a = make_float4(v0.x, v0.y, v0.z, __int_as_float(p));
		b = make_float4(v1.x, v1.y, v1.z, 0.0f);
		c = make_float4(v2.x, v2.y, v2.z, 0.0f);
	}
	soup[3 * size_t(k)] = a;
	soup[3 * size_t(k) + 1] = b;
	soup[3 * size_t(k) + 2] = c;
}

inline unsigned blocks_for(size_t n, unsigned threads) { return unsigned((n + threads - 1) / threads); }

template < class T >
cudaError_t grow(T*& p, size_t count) {
	if(p) cudaFree(p);
	p = nullptr;
	return cudaMalloc(reinterpret_cast<void**>(&p), std::max<size_t>(count, 1) * sizeof(T));
}

} // namespace

void BvhBuffers::release() {
	if(nodes) cudaFree(nodes);
	if(primIds) cudaFree(primIds);
	if(triSoup) cudaFree(triSoup);
	if(wnodes) cudaFree(wnodes);
	if(wprims) cudaFree(wprims);
	if(wsoup) cudaFree(wsoup);
	nodes = nullptr; primIds = nullptr; triSoup = nullptr;
	wnodes = nullptr; wprims = nullptr; wsoup = nullptr;
	nodeCapacity = primCapacity = soupCapacity = 0;
	wideCapacity = wprimCapacity = wsoupCapacity = 0;
	numWide = 0;
}

LbvhBuilder::~LbvhBuilder() {
	cudaFree(m_keysA); cudaFree(m_keysB); cudaFree(m_valsA); cudaFree(m_valsB);
	cudaFree(m_parents); cudaFree(m_children); cudaFree(m_nodeData); cudaFree(m_flags);
	cudaFree(m_marks); cudaFree(m_blockSums); cudaFree(m_hist); cudaFree(m_status);
	cudaFree(m_tileCounter); cudaFree(m_error);
	cudaFree(m_ranges); cudaFree(m_wideCounters); cudaFree(m_wideQueueA); cudaFree(m_wideQueueB);
	if(m_hostCount) cudaFreeHost(m_hostCount);
	for(auto& e : m_ev) if(e) cudaEventDestroy(e);
	for(auto& e : m_wideEv) if(e) cudaEventDestroy(e);
	if(m_fork) cudaEventDestroy(m_fork);
	if(m_join) cudaEventDestroy(m_join);
	if(m_side) cudaStreamDestroy(m_side);
}

cudaError_t LbvhBuilder::reserve(uint32_t n) {
	cudaError_t e = cudaSuccess;
	if(!m_hist) {
		if((e = cudaMalloc(&m_hist, 8 * 256 * sizeof(uint32_t))) != cudaSuccess) return e;
		if((e = cudaMalloc(&m_tileCounter, 8 * sizeof(unsigned int))) != cudaSuccess) return e;
		if((e = cudaMalloc(&m_error, sizeof(unsigned int))) != cudaSuccess) return e;
		if((e = cudaMalloc(&m_wideCounters, WIDE_COUNTERS * sizeof(uint32_t))) != cudaSuccess) return e;
		if((e = cudaMallocHost(&m_hostCount, sizeof(int32_t))) != cudaSuccess) return e;
		if((e = cudaFuncSetAttribute(k_onesweep, cudaFuncAttributeMaxDynamicSharedMemorySize, int(SORT_SMEM))) != cudaSuccess) return e;
		for(auto& ev : m_ev) if((e = cudaEventCreate(&ev)) != cudaSuccess) return e;
		for(auto& ev : m_wideEv) if((e = cudaEventCreate(&ev)) != cudaSuccess) return e;
		if((e = cudaEventCreateWithFlags(&m_fork, cudaEventDisableTiming)) != cudaSuccess) return e;
		if((e = cudaEventCreateWithFlags(&m_join, cudaEventDisableTiming)) != cudaSuccess) return e;
		if((e = cudaStreamCreateWithFlags(&m_side, cudaStreamNonBlocking)) != cudaSuccess) return e;
	}
	if(n <= m_capacity) return cudaSuccess;
	const size_t N = n;
	if((e = grow(m_keysA, N)) != cudaSuccess) return e;
	if((e = grow(m_keysB, N)) != cudaSuccess) return e;
	if((e = grow(m_valsA, N)) != cudaSuccess) return e;
	if((e = grow(m_valsB, N)) != cudaSuccess) return e;
	if((e = grow(m_parents, 2 * N)) != cudaSuccess) return e;
	if((e = grow(m_children, 2 * N)) != cudaSuccess) return e;
	if((e = grow(m_nodeData, 4 * N)) != cudaSuccess) return e;
	if((e = grow(m_flags, N)) != cudaSuccess) return e;
	if((e = grow(m_marks, N)) != cudaSuccess) return e;
	if((e = grow(m_ranges, N)) != cudaSuccess) return e;
	m_wideQueueCapacity = uint32_t(wide_node_capacity(N, 1));
	if((e = grow(m_wideQueueA, size_t(m_wideQueueCapacity))) != cudaSuccess) return e;
	if((e = grow(m_wideQueueB, size_t(m_wideQueueCapacity))) != cudaSuccess) return e;
	if((e = grow(m_blockSums, N / SCAN_TILE + 2)) != cudaSuccess) return e;
	const uint32_t tiles = (n + SORT_TILE - 1) / SORT_TILE;
	if((e = grow(m_status, size_t(tiles) * 256)) != cudaSuccess) return e;
	m_statusCapacity = tiles;
	m_capacity = n;
	return cudaSuccess;
}

cudaError_t LbvhBuilder::sort_pairs(uint64_t* keys, int32_t* values, uint32_t n, cudaStream_t stream, int passes) {
	cudaError_t e = reserve(n);
	if(e != cudaSuccess) return e;
	// callers read the error word after the sort, also when there is nothing to sort
	cudaMemsetAsync(m_error, 0, sizeof(unsigned int), stream);
	if(n <= 1) return cudaSuccess;
	const uint32_t tiles = (n + SORT_TILE - 1) / SORT_TILE;
	cudaMemsetAsync(m_hist, 0, 8 * 256 * sizeof(uint32_t), stream);
	cudaMemsetAsync(m_tileCounter, 0, 8 * sizeof(unsigned int), stream);
	const unsigned hb = std::min<unsigned>(blocks_for(n, 256), 148u * 8u);
	k_sort_hist<<<hb, 256, 0, stream>>>(keys, n, m_hist);
	k_sort_scan<<<8, 256, 0, stream>>>(m_hist);
	u64* kin = keys; u64* kout = (keys == m_keysA) ? m_keysB : m_keysA;
	int32_t* vin = values; int32_t* vout = (values == m_valsA) ? m_valsB : m_valsA;
	// ping-pong between the caller's buffers and the builder's spare ones
	for(int pass = 0; pass < passes; ++pass) {
		cudaMemsetAsync(m_status, 0, size_t(tiles) * 256 * sizeof(uint32_t), stream);
		k_onesweep<<<tiles, SORT_THREADS, SORT_SMEM, stream>>>(kin, vin, kout, vout, n, 8 * pass,
			m_hist + 256 * pass, m_status, m_tileCounter + pass, m_error);
		std::swap(kin, kout);
		std::swap(vin, vout);
	}
	// after an even number of passes the data is back in (keys, values)
	return cudaGetLastError();
}

cudaError_t LbvhBuilder::build_common(int mode, const LodBuildInput* lod, const SceneBuildInput* scene,
                                      uint32_t numPrimitives, uint32_t used, BvhBuffers& out,
                                      cudaStream_t stream, bool withSoup) {
	cudaError_t e;
	out.numPrims = int32_t(numPrimitives);
	m_lastN = int32_t(numPrimitives);
	if(numPrimitives == 0) { out.numInternal = 0; return cudaSuccess; }
	if(out.primCapacity < numPrimitives) {
		if(out.primIds) cudaFree(out.primIds);
		out.primIds = nullptr;
		if((e = cudaMalloc(&out.primIds, sizeof(int32_t) * numPrimitives)) != cudaSuccess) return e;
		out.primCapacity = numPrimitives;
	}
	const size_t nodeCap = 2 * size_t(std::max<uint32_t>(used, 2u) - 1);
	if(out.nodeCapacity < nodeCap) {
		if(out.nodes) cudaFree(out.nodes);
		out.nodes = nullptr;
		if((e = cudaMalloc(&out.nodes, sizeof(BvhNode) * nodeCap)) != cudaSuccess) return e;
		out.nodeCapacity = nodeCap;
	}
	if(mode == MODE_LOD && withSoup && out.soupCapacity < 3 * size_t(numPrimitives)) {
		if(out.triSoup) cudaFree(out.triSoup);
		out.triSoup = nullptr;
		if((e = cudaMalloc(&out.triSoup, sizeof(float4) * 3 * size_t(numPrimitives))) != cudaSuccess) return e;
		out.soupCapacity = 3 * size_t(numPrimitives);
	}
	if((e = reserve(numPrimitives)) != cudaSuccess) return e;
	const bool wide = withSoup || mode == MODE_SCENE;
	if(wide) {
		const size_t wcap = wide_node_capacity(std::max<uint32_t>(used, 2u), mode == MODE_SCENE ? WIDE_TLAS_LEAF_MAX : WIDE_LEAF_MAX);
		if(out.wideCapacity < wcap) {
			if(out.wnodes) cudaFree(out.wnodes);
			out.wnodes = nullptr;
			if((e = cudaMalloc(&out.wnodes, sizeof(WideNode) * wcap)) != cudaSuccess) return e;
			out.wideCapacity = wcap;
		}
		if(out.wprimCapacity < numPrimitives) {
			if(out.wprims) cudaFree(out.wprims);
			out.wprims = nullptr;
			if((e = cudaMalloc(&out.wprims, sizeof(int32_t) * numPrimitives)) != cudaSuccess) return e;
			out.wprimCapacity = numPrimitives;
		}
		if(mode == MODE_LOD && out.wsoupCapacity < 3 * size_t(numPrimitives)) {
			if(out.wsoup) cudaFree(out.wsoup);
			out.wsoup = nullptr;
			if((e = cudaMalloc(&out.wsoup, sizeof(float4) * 3 * size_t(numPrimitives))) != cudaSuccess) return e;
			out.wsoupCapacity = 3 * size_t(numPrimitives);
		}
	}
	out.numWide = 0;
	if(used <= 1) {
		// build_lbvh.cu:595-602: one primitive needs no hierarchy
		cudaMemsetAsync(out.primIds, 0, sizeof(int32_t), stream);
		out.numInternal = 0;
		if(mode == MODE_LOD && withSoup) k_soup<<<1, 32, 0, stream>>>(*lod, 1, out.primIds, out.triSoup);
		if(wide) cudaMemsetAsync(out.wprims, 0, sizeof(int32_t), stream);
		if(mode == MODE_LOD && wide) k_wsoup<<<1, 32, 0, stream>>>(*lod, 1, out.wprims, out.wsoup);
		return cudaGetLastError();
	}
	const int n = int(used);
	const int numInternal = n - 1;
	const int numNodes = numInternal + n;
	if(m_timing) cudaEventRecord(m_ev[0], stream);
	if(mode == MODE_LOD) k_morton_lod<<<blocks_for(numPrimitives, 256), 256, 0, stream>>>(*lod, numPrimitives, m_keysA, m_valsA, m_mortonBits);
	else k_morton_scene<<<blocks_for(numPrimitives, 256), 256, 0, stream>>>(*scene, numPrimitives, m_keysA, m_valsA, m_mortonBits);
	if(m_timing) cudaEventRecord(m_ev[1], stream);
	// 30-bit codes: their four low bytes are the whole key
	if((e = sort_pairs(m_keysA, m_valsA, numPrimitives, stream, m_mortonBits == 30 ? 4 : 8)) != cudaSuccess) return e;
	if(m_timing) cudaEventRecord(m_ev[2], stream);
	cudaMemsetAsync(m_parents, 0, sizeof(int32_t) * numNodes, stream);
	k_karras<<<blocks_for(numInternal, 256), 256, 0, stream>>>(n, m_keysA, m_parents, m_children, m_marks, m_ranges);
	if(m_timing) cudaEventRecord(m_ev[3], stream);
	cudaMemsetAsync(m_flags, 0, sizeof(unsigned int) * numInternal, stream);
	const LodBuildInput lodIn = lod ? *lod : LodBuildInput{};
	const SceneBuildInput sceneIn = scene ? *scene : SceneBuildInput{};
	k_bbox<<<blocks_for(n, 128), 128, 0, stream>>>(mode, lodIn, sceneIn, n, numInternal, m_valsA, m_parents,
	                                               m_children, m_nodeData, m_flags);
	if(m_timing) cudaEventRecord(m_ev[4], stream);
	// An object hierarchy's 8-wide conversion reads only the merged tree
	// (children, ranges, boxes, sorted ids), as the collapse below does, so it
	// runs beside it on the side stream; the instance level's conversion waits
	// for its box refit after the collapse.
	const bool sideWide = wide && mode == MODE_LOD;
	cudaStream_t ws = stream;
	if(sideWide) {
		if((e = cudaEventRecord(m_fork, stream)) != cudaSuccess) return e;
		if((e = cudaStreamWaitEvent(m_side, m_fork, 0)) != cudaSuccess) return e;
		ws = m_side;
	}
	k_mark<<<blocks_for(n, 128), 128, 0, stream>>>(mode, n, numInternal, m_parents, m_nodeData, m_marks);
	if(m_timing) cudaEventRecord(m_ev[5], stream);
	const int scanBlocks = (numInternal + SCAN_TILE - 1) / SCAN_TILE;
	k_scan_tiles<<<scanBlocks, SCAN_THREADS, 0, stream>>>(m_marks, numInternal, m_blockSums);
	k_scan_sums<<<1, SCAN_THREADS, 0, stream>>>(m_blockSums, scanBlocks);
	k_scan_add<<<blocks_for(numInternal, 256), 256, 0, stream>>>(m_marks, numInternal, m_blockSums);
	if(m_timing) cudaEventRecord(m_ev[6], stream);
	k_compact<<<blocks_for(numNodes - 1, 256), 256, 0, stream>>>(mode, numNodes, numInternal, m_parents, m_marks,
	                                                             m_nodeData, out.nodes);
	cudaMemcpyAsync(out.primIds, m_valsA, sizeof(int32_t) * numPrimitives, cudaMemcpyDeviceToDevice, stream);
	k_after<<<1, 1, 0, stream>>>(m_marks, numInternal, m_blockSums);
	cudaMemcpyAsync(m_hostCount, m_blockSums, sizeof(int32_t), cudaMemcpyDeviceToHost, stream);
	if(m_timing) cudaEventRecord(m_ev[7], stream);
	if(mode == MODE_LOD && withSoup)
		k_soup<<<blocks_for(numPrimitives, 256), 256, 0, stream>>>(*lod, int(numPrimitives), out.primIds, out.triSoup);
	if(m_timing) cudaEventRecord(m_ev[8], stream);
	if(wide && mode == MODE_SCENE && scene && scene->wideBoxes && used > 1) {
		cudaMemsetAsync(m_flags, 0, sizeof(unsigned int) * numInternal, stream);
		k_refit_boxes<<<blocks_for(used, 128), 128, 0, stream>>>(int(used), numInternal, m_valsA, m_parents, m_children,
		                                                        scene->wideBoxes, m_nodeData, m_flags);
	}
	if(wide) {
		WideBuildArgs wa{};
		wa.n = n;
		wa.numInternal = numInternal;
		wa.leafMax = mode == MODE_SCENE ? WIDE_TLAS_LEAF_MAX : WIDE_LEAF_MAX;
		wa.children = m_children;
		wa.ranges = m_ranges;
		wa.nodeData = m_nodeData;
		wa.sortedIds = m_valsA;
		wa.nodes = out.wnodes;
		wa.prims = out.wprims;
		wa.nodeCapacity = uint32_t(std::min<size_t>(out.wideCapacity, m_wideQueueCapacity));
		wa.counters = m_wideCounters;
		wa.queueA = m_wideQueueA;
		wa.queueB = m_wideQueueB;
		int32_t numWide = 0;
		if(m_timing) cudaEventRecord(m_wideEv[0], ws);
		if((e = build_wide(wa, &numWide, ws)) != cudaSuccess) return e;
		out.numWide = numWide;
		if(mode == MODE_LOD)
			k_wsoup<<<blocks_for(n, 256), 256, 0, ws>>>(*lod, n, out.wprims, out.wsoup);
		if(m_timing) cudaEventRecord(m_wideEv[1], ws);
	}
	if(sideWide) {
		if((e = cudaEventRecord(m_join, m_side)) != cudaSuccess) return e;
		if((e = cudaStreamWaitEvent(stream, m_join, 0)) != cudaSuccess) return e;
	}
	if(m_timing) cudaEventRecord(m_ev[9], stream);
	if((e = cudaGetLastError()) != cudaSuccess) return e;
	if((e = cudaStreamSynchronize(stream)) != cudaSuccess) return e;
	unsigned int err = 0;
	if((e = cudaMemcpy(&err, m_error, sizeof(err), cudaMemcpyDeviceToHost)) != cudaSuccess) return e;
	if(err) return cudaErrorLaunchTimeout;
	out.numInternal = *m_hostCount;
	if(m_timing) {
		float t[9];
		for(int k = 0; k < 8; ++k) cudaEventElapsedTime(&t[k], m_ev[k], m_ev[k + 1]);
		// the conversion's own span (beside the collapse for object hierarchies)
		t[8] = 0.0f;
		if(wide) cudaEventElapsedTime(&t[8], m_wideEv[0], m_wideEv[1]);
		m_times = { t[0], t[1], t[2], t[3], t[4], t[5], t[6], t[7], t[8] };
	}
	return cudaSuccess;
}

cudaError_t LbvhBuilder::build_lod(const LodBuildInput& in, BvhBuffers& out, cudaStream_t stream, bool withSoup) {
	const uint32_t n = in.numTriangles + in.numQuads + in.numSpheres;
	return build_common(MODE_LOD, &in, nullptr, n, n, out, stream, withSoup);
}

cudaError_t LbvhBuilder::build_scene(const SceneBuildInput& in, BvhBuffers& out, cudaStream_t stream) {
	return build_common(MODE_SCENE, nullptr, &in, in.numInstances, in.activeInstances, out, stream, false);
}

} // namespace mb
