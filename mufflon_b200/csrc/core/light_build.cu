// GPU light list and light tree (see light_build.hpp). Compiled with
// --fmad=false like the rest of the device code: every float expression
// below has the operation order of the CPU restatement, so fluxes, keys and
// the tree are bit-identical to it.
#include "light_build.hpp"
#include "../lbvh/lbvh.hpp"

#include <algorithm>

namespace mb {
namespace {

constexpr float LB_PI = 3.14159265358979f;
constexpr int LB_THREADS = 256;

struct F3 { float x, y, z; };
__device__ __forceinline__ F3 f3(float x, float y, float z) { return F3{ x, y, z }; }
__device__ __forceinline__ F3 operator+(F3 a, F3 b) { return f3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ F3 operator-(F3 a, F3 b) { return f3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ F3 operator*(F3 a, float s) { return f3(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ F3 operator*(float s, F3 a) { return f3(s * a.x, s * a.y, s * a.z); }
__device__ __forceinline__ F3 operator*(F3 a, F3 b) { return f3(a.x * b.x, a.y * b.y, a.z * b.z); }
__device__ __forceinline__ F3 operator/(F3 a, float s) { return f3(__fdiv_rn(a.x, s), __fdiv_rn(a.y, s), __fdiv_rn(a.z, s)); }
__device__ __forceinline__ F3 cross(F3 a, F3 b) {
	return f3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ float len(F3 a) { return __fsqrt_rn(a.x * a.x + a.y * a.y + a.z * a.z); }
__device__ __forceinline__ F3 ld(const float* p) { return f3(p[0], p[1], p[2]); }
__device__ __forceinline__ void st(float* p, F3 v) { p[0] = v.x; p[1] = v.y; p[2] = v.z; }

__device__ __forceinline__ F3 xform_point(const float* m, F3 p) {
	return f3(m[0] * p.x + m[1] * p.y + m[2] * p.z + m[3],
	          m[4] * p.x + m[5] * p.y + m[6] * p.z + m[7],
	          m[8] * p.x + m[9] * p.y + m[10] * p.z + m[11]);
}

__device__ __forceinline__ F3 light_center(const DLight& l) {
	if(l.type == LT_QUAD) return (ld(l.posV[0]) + (ld(l.posV[1]) + ld(l.posV[2])) * 0.5f) + ld(l.posV[3]) * 0.25f;
	if(l.type == LT_TRI) return ld(l.posV[0]) + (ld(l.posV[1]) + ld(l.posV[2])) / 3.0f;
	return ld(l.position);
}

// Hilbert-curve code of 16-bit coordinates (light_tree.cpp ordering)
__device__ __forceinline__ uint64_t part_by_three16(uint32_t x) {
	uint64_t r = x & 0xFFFF;
	r = (r | (r << 16)) & 0x0000ff0000ffull;
	r = (r | (r << 8)) & 0x00f00f00f00full;
	r = (r | (r << 4)) & 0x0c30c30c30c3ull;
	r = (r | (r << 2)) & 0x249249249249ull;
	return r;
}
__device__ __forceinline__ uint64_t hilbert3(uint32_t a, uint32_t b, uint32_t c) {
	uint64_t num = part_by_three16(a) | (part_by_three16(b) << 1u) | (part_by_three16(c) << 2u);
	num = num ^ (num >> 32); num = num ^ (num >> 16); num = num ^ (num >> 8);
	num = num ^ (num >> 4); num = num ^ (num >> 2); num = num ^ (num >> 1);
	return num;
}
__device__ __forceinline__ uint32_t to_u32(float v) {
	return v <= 0.0f ? 0u : (v >= 4294967040.0f ? 0xFFFFFF00u : uint32_t(v));
}

__device__ __forceinline__ uint64_t scramble_seed(uint32_t x) {
	uint64_t z = uint64_t(x) + 0x9e3779b97f4a7c15ull;
	z = (z ^ (z >> 30u)) * 0xbf58476d1ce4e5b9ull;
	z = (z ^ (z >> 27u)) * 0x94d049bb133111ebull;
	return z ^ (z >> 31u);
}
__device__ __forceinline__ float sample_uniform(uint32_t u) { return __fdiv_rn(float(u), 4294967810.0f); }

// lights.cpp:16-80: a point light's flux from its intensity; a triangle's
// and a sphere's from the area and the mean emitted radiance; a quad's from
// 128 low-discrepancy samples of its area times the emitted radiance.
__device__ float light_flux(const DLight& l, int32_t primInst, int32_t primId, const DMaterial* mats) {
	if(l.type == LT_POINT) {
		const F3 f = ld(l.intensity) * 4.0f * LB_PI;
		return (f.x + f.y) + f.z;
	}
	const F3 rad = ld(mats[l.material].radiance);
	if(l.type == LT_SPHERE) {
		// lights.cpp:63-80: the mean of 128 samples of the (constant) radiance,
		// times the sphere's area times 2 pi
		const float area = ((4.0f * LB_PI) * l.radius) * l.radius;
		F3 sum = f3(0, 0, 0);
		for(int i = 0; i < 128; ++i) sum = sum + rad;
		sum = sum / 128.0f;
		const F3 f = sum * area * 2.0f * LB_PI;
		return (f.x + f.y) + f.z;
	}
	if(l.type == LT_TRI) {
		// lights.cpp:24-40: the mean of 128 samples of the (constant) radiance,
		// times area times 2 pi
		const float area = __fdiv_rn(len(cross(ld(l.posV[1]), ld(l.posV[2]))), 2.0f);
		F3 sum = f3(0, 0, 0);
		for(int i = 0; i < 128; ++i) sum = sum + rad;
		sum = sum / 128.0f;
		const F3 f = sum * area * 2.0f * LB_PI;
		return (f.x + f.y) + f.z;
	}
	uint64_t state = scramble_seed(uint32_t(primId) * 2654435761u + uint32_t(primInst));
	const F3 v1 = ld(l.posV[1]), v2 = ld(l.posV[2]), v3 = ld(l.posV[3]);
	F3 sum = f3(0, 0, 0);
	for(int i = 0; i < 128; ++i) {
		uint64_t s = state;
		state += 11400714819323198485ull;
		s = s ^ (s >> 1);
		s = ((s >> 1) & 0x2222222222222222ull) | ((s << 1) & 0x4444444444444444ull) | (s & 0x9999999999999999ull);
		s = ((s >> 2) & 0x0c0c0c0c0c0c0c0cull) | ((s << 2) & 0x3030303030303030ull) | (s & 0xc3c3c3c3c3c3c3c3ull);
		s = ((s >> 4) & 0x00f000f000f000f0ull) | ((s << 4) & 0x0f000f000f000f00ull) | (s & 0xf00ff00ff00ff00full);
		s = ((s >> 8) & 0x0000ff000000ff00ull) | ((s << 8) & 0x00ff000000ff0000ull) | (s & 0xff0000ffff0000ffull);
		s = ((s >> 16) & 0x00000000ffff0000ull) | ((s << 16) & 0x0000ffff00000000ull) | (s & 0xffff00000000ffffull);
		const float ux = sample_uniform(uint32_t(s & 0xffffffffull));
		const float uy = sample_uniform(uint32_t(s >> 32ull));
		const F3 tx = v1 + ux * v3;
		const F3 ty = v2 + uy * v3;
		const float area = len(cross(ty, tx));
		sum = sum + area * rad;
	}
	sum = sum / 128.0f;
	const F3 f = sum * 2.0f * LB_PI;
	return (f.x + f.y) + f.z;
}

__global__ void k_make_lights(const LightBuildInput in, uint32_t n, DLight* lights, int32_t* primInst, int32_t* primId,
                              uint64_t* keyHi, uint64_t* keyLo, int32_t* order) {
	const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
	if(t >= n) return;
	DLight L{};
	int32_t inst = -1, prim = -1;
	if(t < in.numArea) {
		// the instance whose range of light indices holds t
		uint32_t lo = 0, hi = in.numInstances;
		while(hi - lo > 1) {
			const uint32_t mid = (lo + hi) >> 1;
			if(in.instFirstLight[mid] <= t) lo = mid; else hi = mid;
		}
		const uint32_t i = lo;
		const LightLodInfo lod = in.lods[in.instLod[i]];
		const uint32_t entry = lod.faceListStart + (t - in.instFirstLight[i]);
		const uint32_t f = in.emissiveFaces[entry];
		const float* m = in.instToWorld + 12 * size_t(i);
		if(f >= lod.numTriangles + lod.numQuads) {
			// world_container.cpp:966-990: the centre transformed, the radius
			// scaled by the length of the instance's first axis
			const float4 sp = lod.spheres[f - lod.numTriangles - lod.numQuads];
			const F3 col0 = f3(m[0], m[4], m[8]);
			L.type = LT_SPHERE;
			L.material = in.faceMaterial[entry];
			st(L.position, xform_point(m, f3(sp.x, sp.y, sp.z)));
			L.radius = len(col0) * sp.w;
			lights[t] = L;
			primInst[t] = int32_t(i);
			primId[t] = int32_t(f);
			const F3 c = light_center(L) * f3(in.sceneScale[0], in.sceneScale[1], in.sceneScale[2]);
			const uint32_t ax = to_u32(c.x), ay = to_u32(c.y), az = to_u32(c.z);
			keyHi[t] = hilbert3(ax >> 16, ay >> 16, az >> 16);
			keyLo[t] = hilbert3(ax & 0xffff, ay & 0xffff, az & 0xffff);
			order[t] = int32_t(t);
			return;
		}
		const bool tri = f < lod.numTriangles;
		const int corners = tri ? 3 : 4;
		const uint32_t base = tri ? 3u * f : 3u * lod.numTriangles + 4u * (f - lod.numTriangles);
		F3 pts[4]; float uv[4][2];
		for(int k = 0; k < corners; ++k) {
			const uint32_t vi = lod.indices[base + k];
			pts[k] = xform_point(m, ld(lod.vertices + 3 * size_t(vi)));
			uv[k][0] = lod.uvs ? lod.uvs[2 * size_t(vi)] : 0.0f;
			uv[k][1] = lod.uvs ? lod.uvs[2 * size_t(vi) + 1] : 0.0f;
		}
		L.material = in.faceMaterial[entry];
		if(tri) {
			// world_container.cpp:929-948 (mirroring swaps the last two corners)
			if(in.mirroring[i]) {
				const F3 tp = pts[1]; pts[1] = pts[2]; pts[2] = tp;
				for(int c = 0; c < 2; ++c) { const float tu = uv[1][c]; uv[1][c] = uv[2][c]; uv[2][c] = tu; }
			}
			L.type = LT_TRI;
			st(L.posV[0], pts[0]);
			st(L.posV[1], pts[1] - pts[0]);
			st(L.posV[2], pts[2] - pts[0]);
			for(int c = 0; c < 2; ++c) {
				L.uvV[0][c] = uv[0][c];
				L.uvV[1][c] = uv[1][c] - uv[0][c];
				L.uvV[2][c] = uv[2][c] - uv[0][c];
			}
		} else {
			if(in.mirroring[i]) {
				const F3 tp = pts[1]; pts[1] = pts[3]; pts[3] = tp;
				for(int c = 0; c < 2; ++c) { const float tu = uv[1][c]; uv[1][c] = uv[3][c]; uv[3][c] = tu; }
			}
			L.type = LT_QUAD;
			const F3 e2 = pts[1] - pts[0];
			st(L.posV[0], pts[0]);
			st(L.posV[1], pts[3] - pts[0]);
			st(L.posV[2], e2);
			st(L.posV[3], (pts[2] - pts[3]) - e2);
			for(int c = 0; c < 2; ++c) {
				const float u2 = uv[1][c] - uv[0][c];
				L.uvV[0][c] = uv[0][c];
				L.uvV[1][c] = uv[3][c] - uv[0][c];
				L.uvV[2][c] = u2;
				L.uvV[3][c] = (uv[2][c] - uv[3][c]) - u2;
			}
		}
		inst = int32_t(i);
		prim = int32_t(f);
	} else {
		const float* p = in.pointLights + 6 * size_t(t - in.numArea);
		L.type = LT_POINT;
		L.position[0] = p[0]; L.position[1] = p[1]; L.position[2] = p[2];
		L.intensity[0] = p[3]; L.intensity[1] = p[4]; L.intensity[2] = p[5];
	}
	lights[t] = L;
	primInst[t] = inst;
	primId[t] = prim;
	const F3 c = light_center(L) * f3(in.sceneScale[0], in.sceneScale[1], in.sceneScale[2]);
	const uint32_t ax = to_u32(c.x), ay = to_u32(c.y), az = to_u32(c.z);
	keyHi[t] = hilbert3(ax >> 16, ay >> 16, az >> 16);
	keyLo[t] = hilbert3(ax & 0xffff, ay & 0xffff, az & 0xffff);
	order[t] = int32_t(t);
}

__global__ void k_permute_keys(uint32_t n, const uint64_t* src, const int32_t* order, uint64_t* dst) {
	const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
	if(t < n) dst[t] = src[order[t]];
}

__global__ void k_gather_lights(uint32_t n, const int32_t* order, const DLight* unsorted, const int32_t* primInst,
                                const int32_t* primId, const DMaterial* mats, DLight* lights, int32_t* sInst,
                                int32_t* sPrim, float* flux) {
	const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
	if(t >= n) return;
	const int32_t o = order[t];
	const DLight L = unsorted[o];
	lights[t] = L;
	sInst[t] = primInst[o];
	sPrim[t] = primId[o];
	flux[t] = light_flux(L, primInst[o], primId[o], mats);
}

// One level of the tree: node firstNode + i gets the pair of children
// (childStart + 2i, childStart + 2i + 1), lights or nodes.
__global__ void k_tree_pairs(uint32_t count, DLightNode* nodes, uint32_t firstNode, uint32_t childStart,
                             int childrenAreNodes, const float* flux, const DLight* lights) {
	const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
	if(i >= count) return;
	DLightNode nd;
	const uint32_t l = childStart + 2 * i, r = l + 1;
	if(childrenAreNodes) {
		const DLightNode a = nodes[l], b = nodes[r];
		nd.leftFlux = a.leftFlux + a.rightFlux; nd.leftIndex = int32_t(l); nd.leftType = LT_INTERNAL;
		nd.rightFlux = b.leftFlux + b.rightFlux; nd.rightIndex = int32_t(r); nd.rightType = LT_INTERNAL;
	} else {
		nd.leftFlux = flux[l]; nd.leftIndex = int32_t(l); nd.leftType = lights[l].type;
		nd.rightFlux = flux[r]; nd.rightIndex = int32_t(r); nd.rightType = lights[r].type;
	}
	nodes[firstNode + i] = nd;
}

// The odd extra node: the last bottom node paired with light 0.
__global__ void k_tree_odd(DLightNode* nodes, uint32_t at, uint32_t node, const float* flux, const DLight* lights) {
	const DLightNode a = nodes[node];
	DLightNode nd;
	nd.leftFlux = a.leftFlux + a.rightFlux; nd.leftIndex = int32_t(node); nd.leftType = LT_INTERNAL;
	nd.rightFlux = flux[0]; nd.rightIndex = 0; nd.rightType = lights[0].type;
	nodes[at] = nd;
}

// light_tree.cpp fill_map: the node path of every area light as a code whose
// leading bits are the left/right decisions from the root.
__global__ void k_codes(uint32_t n, const int32_t* sInst, const int32_t* sPrim, uint32_t height, uint32_t extra,
                        uint64_t* keys, uint32_t* codes) {
	const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
	if(i >= n) return;
	const bool area = sInst[i] != -1;
	keys[i] = area ? ((uint64_t(uint32_t(sInst[i])) << 32) | uint32_t(sPrim[i])) : ~0ull;
	uint32_t code = 0;
	if(n > 1) {
		const uint32_t h = height;
		const uint32_t lowerLightCount = (1u << h) - extra;
		if(extra > 0 && i < lowerLightCount) code = (((1u << h) - 1u) - (lowerLightCount - i - 1u)) << (32u - h);
		else {
			const uint32_t hh = extra > 0 ? h + 1u : h;
			code = (i - lowerLightCount) << (32u - hh);
		}
	}
	codes[i] = code;
}

unsigned blocks(uint32_t n) { return (n + LB_THREADS - 1) / LB_THREADS; }

template < class T >
cudaError_t grow(T*& p, size_t n) {
	if(p) cudaFree(p);
	p = nullptr;
	return cudaMalloc(reinterpret_cast<void**>(&p), sizeof(T) * std::max<size_t>(n, 1));
}

} // namespace

void LightBuildScratch::release() {
	cudaFree(unsorted); cudaFree(primInst); cudaFree(primId); cudaFree(keyHi); cudaFree(keyLo); cudaFree(order);
	cudaFree(flux); cudaFree(sortedInst); cudaFree(sortedPrim);
	unsorted = nullptr; primInst = primId = nullptr; keyHi = keyLo = nullptr; order = nullptr; flux = nullptr;
	sortedInst = sortedPrim = nullptr;
	capacity = 0;
}

cudaError_t build_lights_gpu(const LightBuildInput& in, LightBuildScratch& S, LbvhBuilder& sorter,
                             const LightBuildOutput& out, LightTreeInfo& info, cudaStream_t stream) {
	info = LightTreeInfo{};
	const uint32_t n = in.numArea + in.numPoint;
	if(n == 0) return cudaSuccess;
	cudaError_t e = cudaSuccess;
	if(n > S.capacity) {
		S.release();
		if((e = grow(S.unsorted, n)) != cudaSuccess || (e = grow(S.primInst, n)) != cudaSuccess ||
		   (e = grow(S.primId, n)) != cudaSuccess || (e = grow(S.keyHi, n)) != cudaSuccess ||
		   (e = grow(S.keyLo, n)) != cudaSuccess || (e = grow(S.order, n)) != cudaSuccess ||
		   (e = grow(S.flux, n)) != cudaSuccess || (e = grow(S.sortedInst, n)) != cudaSuccess ||
		   (e = grow(S.sortedPrim, n)) != cudaSuccess) { S.release(); return e; }
		S.capacity = n;
	}
	k_make_lights<<<blocks(n), LB_THREADS, 0, stream>>>(in, n, S.unsorted, S.primInst, S.primId, S.keyHi, S.keyLo, S.order);
	if(n > 1) {
		// stable sort by (high key, low key): by the low key, then stably by the high key
		if((e = sorter.sort_pairs(S.keyLo, S.order, n, stream)) != cudaSuccess) return e;
		k_permute_keys<<<blocks(n), LB_THREADS, 0, stream>>>(n, S.keyHi, S.order, S.keyLo);
		if((e = sorter.sort_pairs(S.keyLo, S.order, n, stream)) != cudaSuccess) return e;
	}
	k_gather_lights<<<blocks(n), LB_THREADS, 0, stream>>>(n, S.order, S.unsorted, S.primInst, S.primId, in.materials,
	                                                       out.lights, S.sortedInst, S.sortedPrim, S.flux);
	uint32_t height = 0;
	while((uint64_t(1) << (height + 1)) <= n) ++height;
	const uint32_t full = 1u << height;
	const uint32_t extra = n - full;
	if(n > 1) {
		// light_tree.cpp:120-259: a balanced tree over the first 2^height
		// slots, with `extra` bottom nodes pairing the last 2 * extra lights
		if(extra > 0) {
			const uint32_t startNode = full - 1;
			k_tree_pairs<<<blocks(extra), LB_THREADS, 0, stream>>>(extra, out.nodes, startNode, n - 2 * extra, 0, S.flux, out.lights);
			const uint32_t startInner = (full >> 1) - 1;
			if(extra / 2 > 0)
				k_tree_pairs<<<blocks(extra / 2), LB_THREADS, 0, stream>>>(extra / 2, out.nodes, startInner, startNode, 1, S.flux, out.lights);
			if(extra % 2 != 0)
				k_tree_odd<<<1, 1, 0, stream>>>(out.nodes, startInner + extra / 2, startNode + extra - 1, S.flux, out.lights);
		}
		const uint32_t startLight = (extra % 2 == 0) ? 0u : 1u;
		const uint32_t nodeCount = (n - 2 * extra - startLight) / 2;
		if(nodeCount > 0)
			k_tree_pairs<<<blocks(nodeCount), LB_THREADS, 0, stream>>>(nodeCount, out.nodes, full - nodeCount - 1, startLight, 0,
			                                                           S.flux, out.lights);
		for(uint32_t level = height - 1; level >= 1 && height > 1; --level) {
			const uint32_t nodes = 1u << level;
			k_tree_pairs<<<blocks(nodes / 2), LB_THREADS, 0, stream>>>(nodes / 2, out.nodes, nodes / 2 - 1, nodes - 1, 1,
			                                                           S.flux, out.lights);
		}
	}
	k_codes<<<blocks(n), LB_THREADS, 0, stream>>>(n, S.sortedInst, S.sortedPrim, height, extra, out.primKeys, out.primCodes);
	if(n > 1 && (e = sorter.sort_pairs(out.primKeys, reinterpret_cast<int32_t*>(out.primCodes), n, stream)) != cudaSuccess)
		return e;
	if((e = cudaGetLastError()) != cudaSuccess) return e;
	if(n == 1) {
		float f = 0.0f;
		if((e = cudaMemcpyAsync(&f, S.flux, sizeof(float), cudaMemcpyDeviceToHost, stream)) != cudaSuccess) return e;
		if((e = cudaStreamSynchronize(stream)) != cudaSuccess) return e;
		info.rootFlux = f;
		info.rootType = in.numArea == 1 ? LT_QUAD : LT_POINT;
		info.rootIndex = 0;
		info.numNodes = 0;
	} else {
		float lr[2] = { 0.0f, 0.0f };
		if((e = cudaMemcpyAsync(lr, out.nodes, 2 * sizeof(float), cudaMemcpyDeviceToHost, stream)) != cudaSuccess) return e;
		if((e = cudaStreamSynchronize(stream)) != cudaSuccess) return e;
		info.rootFlux = lr[0] + lr[1];
		info.rootType = LT_INTERNAL;
		info.rootIndex = 0;
		info.numNodes = (full - 1) + extra;
	}
	return cudaSuccess;
}

} // namespace mb
