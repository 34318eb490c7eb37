// Flattening of the host world into the device scene: LoD geometry upload,
// GPU LBVH builds (one per used LoD, then the instance BVH), materials, the
// light tree and the camera.
//
// Host-side arithmetic here (instance inverses, instance boxes, the camera
// frame, light-tree fluxes) follows the reference step by step:
//   descriptors.hpp:108-129 (instance-to-world inverse), scene.cpp:111-419
//   (instance boxes, scene box, instance BVH), camera.hpp:81-96 and
//   pinhole.hpp:22 (camera frame), world_container.cpp:869-990 (emissive
//   quads become area lights), light_tree.cpp:120-447 and lights.cpp:10-62
//   (tree layout, fluxes, node-path codes), background.cpp:125-135
//   (environment flux).
// It is compiled without FP contraction so that it rounds exactly like the
// CPU oracle's copy of the same steps.
#include "world.hpp"

#include <algorithm>
#include <chrono>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <map>

namespace mb {
namespace {

struct V3 { float x, y, z; };
inline V3 operator+(V3 a, V3 b) { return { a.x + b.x, a.y + b.y, a.z + b.z }; }
inline V3 operator-(V3 a, V3 b) { return { a.x - b.x, a.y - b.y, a.z - b.z }; }
inline V3 operator*(V3 a, float s) { return { a.x * s, a.y * s, a.z * s }; }
inline V3 operator*(float s, V3 a) { return { s * a.x, s * a.y, s * a.z }; }
inline V3 operator*(V3 a, V3 b) { return { a.x * b.x, a.y * b.y, a.z * b.z }; }
inline V3 operator/(V3 a, float s) { return { a.x / s, a.y / s, a.z / s }; }
inline float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline V3 cross(V3 a, V3 b) { return { a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x }; }
inline float len(V3 a) { return std::sqrt(dot(a, a)); }
inline V3 normalize(V3 a) { return a / len(a); }
inline float bmin(float a, float b) { return b < a ? b : a; }
inline float bmax(float a, float b) { return a < b ? b : a; }
inline V3 vmin(V3 a, V3 b) { return { bmin(a.x, b.x), bmin(a.y, b.y), bmin(a.z, b.z) }; }
inline V3 vmax(V3 a, V3 b) { return { bmax(a.x, b.x), bmax(a.y, b.y), bmax(a.z, b.z) }; }
inline V3 ld3(const float* p) { return { p[0], p[1], p[2] }; }
inline void st3(float* p, V3 v) { p[0] = v.x; p[1] = v.y; p[2] = v.z; }

struct Box { V3 mn, mx; };
inline Box empty_box() { return { { FLT_MAX, FLT_MAX, FLT_MAX }, { -FLT_MAX, -FLT_MAX, -FLT_MAX } }; }

struct Mat34 { float m[12]; };
inline V3 xform_point(const Mat34& M, V3 p) {
	const float* m = M.m;
	return { m[0] * p.x + m[1] * p.y + m[2] * p.z + m[3],
	         m[4] * p.x + m[5] * p.y + m[6] * p.z + m[7],
	         m[8] * p.x + m[9] * p.y + m[10] * p.z + m[11] };
}
Mat34 instance_to_world(const float* r) {
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

constexpr float PI = 3.14159265358979f;

inline uint64_t scramble_seed(uint32_t x) {
	uint64_t z = uint64_t(x) + 0x9e3779b97f4a7c15ull;
	z = (z ^ (z >> 30u)) * 0xbf58476d1ce4e5b9ull;
	z = (z ^ (z >> 27u)) * 0x94d049bb133111ebull;
	return z ^ (z >> 31u);
}
inline float sample_uniform(uint32_t u) { return float(u) / 4294967810.0f; }

struct HostLight {
	uint16_t type;
	V3 position, intensity;
	V3 posV[4];
	float uvV[4][2];
	uint16_t material;
	int32_t primInst = -1, primId = -1;
};

inline V3 light_center(const HostLight& l) {
	if(l.type == LT_QUAD) return (l.posV[0] + (l.posV[1] + l.posV[2]) * 0.5f) + l.posV[3] * 0.25f;
	return l.position;
}

// lights.cpp:16-62 (the quad variant samples a low-discrepancy 2D sequence;
// its seed is derived from the primitive instead of the light's address)
float light_flux(const HostLight& l, const std::vector<DMaterial>& mats) {
	if(l.type == LT_POINT) {
		const V3 f = l.intensity * 4.0f * PI;
		return (f.x + f.y) + f.z;
	}
	const DMaterial& m = mats[l.material];
	const V3 rad = ld3(m.radiance);
	uint64_t state = scramble_seed(uint32_t(l.primId) * 2654435761u + uint32_t(l.primInst));
	V3 sum = { 0, 0, 0 };
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
		const V3 tx = l.posV[1] + ux * l.posV[3];
		const V3 ty = l.posV[2] + uy * l.posV[3];
		const float area = len(cross(ty, tx));
		sum = sum + area * rad;
	}
	sum = sum / 128.0f;
	const V3 f = sum * 2.0f * PI;
	return (f.x + f.y) + f.z;
}

struct LightTreeOut {
	std::vector<DLightNode> nodes;
	std::vector<std::pair<uint64_t, uint32_t>> codes;
	float rootFlux = 0.0f;
	uint16_t rootType = LT_INTERNAL;
	int32_t rootIndex = 0;
};

// light_tree.cpp:120-259 (balanced tree with extra bottom nodes) and fill_map
LightTreeOut build_pos_tree(const std::vector<HostLight>& lights, const std::vector<DMaterial>& mats) {
	LightTreeOut T;
	const size_t n = lights.size();
	if(n == 0) return T;
	std::vector<float> flux(n);
	for(size_t i = 0; i < n; ++i) flux[i] = light_flux(lights[i], mats);
	auto key = [&](const HostLight& l) { return (uint64_t(uint32_t(l.primInst)) << 32) | uint32_t(l.primId); };
	if(n == 1) {
		T.rootType = lights[0].type;
		T.rootIndex = 0;
		T.rootFlux = flux[0];
		if(lights[0].primInst != -1) T.codes.push_back({ key(lights[0]), 0u });
		return T;
	}
	size_t height = 0;
	while((size_t(1) << (height + 1)) <= n) ++height;
	const size_t extra = n - (size_t(1) << height);
	const size_t internalCount = ((size_t(1) << height) - 1) + extra;
	T.nodes.assign(internalCount, DLightNode{});
	std::vector<V3> centers(internalCount, V3{ 0, 0, 0 });
	struct Ref { float flux; int32_t index; uint16_t type; };
	auto lightRef = [&](size_t i) { return Ref{ flux[i], int32_t(i), lights[i].type }; };
	auto nodeRef = [&](size_t i) { return Ref{ T.nodes[i].leftFlux + T.nodes[i].rightFlux, int32_t(i), uint16_t(LT_INTERNAL) }; };
	auto refCenter = [&](const Ref& r) { return r.type == LT_INTERNAL ? centers[r.index] : light_center(lights[r.index]); };
	auto makeNode = [&](size_t at, Ref l, Ref r) {
		DLightNode nd;
		nd.leftFlux = l.flux; nd.leftIndex = l.index; nd.leftType = l.type;
		nd.rightFlux = r.flux; nd.rightIndex = r.index; nd.rightType = r.type;
		T.nodes[at] = nd;
		centers[at] = (refCenter(l) + refCenter(r)) / 2.0f;
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
	T.rootType = LT_INTERNAL;
	T.rootIndex = 0;
	T.rootFlux = T.nodes[0].leftFlux + T.nodes[0].rightFlux;
	int h = int(height);
	const uint32_t lowerLightCount = uint32_t(1u << h) - uint32_t(extra);
	uint32_t i = 0;
	if(extra > 0) {
		for(; i < lowerLightCount; ++i) {
			if(lights[i].primInst != -1) {
				uint32_t code = ((1u << h) - 1) - (lowerLightCount - i - 1);
				code <<= (32 - h);
				T.codes.push_back({ key(lights[i]), code });
			}
		}
		h += 1;
	}
	for(; i < n; ++i) {
		if(lights[i].primInst != -1) T.codes.push_back({ key(lights[i]), (i - lowerLightCount) << (32 - h) });
	}
	std::sort(T.codes.begin(), T.codes.end());
	return T;
}

// Copies count elements (in up to two parts) into a grow-only device buffer.
template < class T >
bool upload(T*& dst, size_t& cap, const T* src, size_t count, cudaStream_t s, std::string& err,
            const T* src2 = nullptr, size_t count2 = 0, uint64_t* bytes = nullptr) {
	const size_t total = count + count2;
	if(total == 0) return true;
	cudaError_t e = cudaSuccess;
	if(total > cap) {
		if(dst) cudaFree(dst);
		dst = nullptr;
		cap = 0;
		e = cudaMalloc(reinterpret_cast<void**>(&dst), sizeof(T) * total);
		if(e == cudaSuccess) cap = total;
	}
	if(e == cudaSuccess && count) e = cudaMemcpyAsync(dst, src, sizeof(T) * count, cudaMemcpyHostToDevice, s);
	if(e == cudaSuccess && count2) e = cudaMemcpyAsync(dst + count, src2, sizeof(T) * count2, cudaMemcpyHostToDevice, s);
	if(e != cudaSuccess) { err = std::string("device upload failed: ") + cudaGetErrorString(e); return false; }
	if(bytes) *bytes += sizeof(T) * total;
	return true;
}

inline V3 tex_value(const HostTexture* t, V3 fallback) {
	if(!t || t->texels.empty()) return fallback;
	return { t->texels[0], t->texels[1], t->texels[2] };
}

} // namespace

bool HostLod::bounds(float mn[3], float mx[3]) const {
	Box b = empty_box();
	for(size_t v = 0; v + 2 < vertices.size(); v += 3) {
		const V3 p = { vertices[v], vertices[v + 1], vertices[v + 2] };
		b.mn = vmin(b.mn, p); b.mx = vmax(b.mx, p);
	}
	for(size_t k = 0; k + 3 < spheres.size(); k += 4) {
		const V3 c = { spheres[k], spheres[k + 1], spheres[k + 2] };
		const float r = spheres[k + 3];
		b.mn = vmin(b.mn, c - V3{ r, r, r }); b.mx = vmax(b.mx, c + V3{ r, r, r });
	}
	st3(mn, b.mn); st3(mx, b.mx);
	return true;
}

void DeviceLod::release() {
	cudaFree(vertices); cudaFree(normals); cudaFree(uvs); cudaFree(indices);
	cudaFree(faceMat); cudaFree(spheres); cudaFree(sphereMat);
	vertices = normals = uvs = nullptr; indices = nullptr; faceMat = sphereMat = nullptr; spheres = nullptr;
	for(size_t& c : cap) c = 0;
	bvh.release();
}

void DeviceScene::release() {
	for(auto& l : lods) l.release();
	lods.clear();
	lodSources.clear();
	cudaFree(dLods); cudaFree(dW2I); cudaFree(dInstLod); cudaFree(dInstBoxes); cudaFree(dInstCentroids);
	tlas.release();
	cudaFree(dMaterials);
	for(auto* t : textureBuffers) cudaFree(t);
	textureBuffers.clear();
	cudaFree(dTextures); cudaFree(dLights); cudaFree(dLightNodes); cudaFree(dLightKeys); cudaFree(dLightCodes);
	dLods = nullptr; dW2I = nullptr; dInstLod = nullptr; dInstBoxes = nullptr; dInstCentroids = nullptr;
	dMaterials = nullptr; dTextures = nullptr; dLights = nullptr; dLightNodes = nullptr;
	dLightKeys = nullptr; dLightCodes = nullptr;
	for(size_t& c : cap) c = 0;
	desc = DScene{};
	valid = false;
}

// scenario.cpp:131-154, with the level clamped to the object's LoD slots in every case
uint32_t HostScenario::effective_lod(const HostInstance& inst) const {
	uint32_t level = globalLod;
	auto ii = instanceLods.find(inst.index);
	if(ii != instanceLods.end()) level = ii->second;
	else if(inst.object) {
		auto oi = objectLods.find(inst.object);
		if(oi != objectLods.end()) level = oi->second;
	}
	const uint32_t slots = inst.object ? inst.object->lod_slot_count() : 1u;
	return std::min(level, slots - 1u);
}

bool build_device_scene(MufflonInstance& inst, std::string& err) {
	HostScenario* sc = inst.current;
	if(!sc) { err = "no scenario loaded"; return false; }
	if(!sc->camera) { err = "scenario has no camera"; return false; }
	cudaStream_t s = inst.stream;
	DeviceScene& D = inst.scene;
	using clk = std::chrono::steady_clock;
	const auto t0 = clk::now();
	auto msSince = [](clk::time_point a) { return std::chrono::duration<float, std::milli>(clk::now() - a).count(); };
	float uploadMs = 0.0f, bvhMs = 0.0f;
	uint64_t h2d = 0;
	// keep the device buffers of the previous load (grow-only); textures are re-made
	D.valid = false;
	D.desc = DScene{};
	D.lodSources.clear();
	for(auto* t : D.textureBuffers) cudaFree(t);
	D.textureBuffers.clear();
	D.textureSources.clear();

	// --- materials per slot (scene.cpp load_materials)
	std::vector<DMaterial> mats(std::max<size_t>(sc->slotMaterials.size(), 1));
	std::vector<const HostTexture*> texList;
	for(size_t i = 0; i < sc->slotMaterials.size(); ++i) {
		const HostMaterial* m = sc->slotMaterials[i];
		DMaterial& d = mats[i];
		d = DMaterial{};
		d.albedoTex = -1;
		if(!m) { d.type = MAT_LAMBERT; continue; }
		d.type = m->type;
		const V3 alb = tex_value(m->albedo, V3{ 0.5f, 0.5f, 0.5f });
		st3(d.albedo, alb);
		if(m->albedo && (m->albedo->width > 1 || m->albedo->height > 1)) {
			d.albedoTex = int32_t(texList.size());
			texList.push_back(m->albedo);
		}
		if(m->roughness && !m->roughness->texels.empty()) {
			d.roughness[0] = m->roughness->texels[0];
			d.roughness[1] = m->roughness->channels > 1 ? m->roughness->texels[1] : m->roughness->texels[0];
		} else { d.roughness[0] = d.roughness[1] = 0.5f; }
		if(m->type == MAT_EMISSIVE) {
			const V3 rad = tex_value(m->radiance, V3{ 0, 0, 0 });
			st3(d.radiance, rad * ld3(m->scale));
		}
	}

	// --- instances and used LoDs (scene.cpp:153-303)
	const uint32_t numInst = uint32_t(inst.instances.size());
	std::vector<uint32_t> instLod(numInst, 0xFFFFFFFFu);
	std::map<const HostLod*, uint32_t> lodIndex;
	std::vector<uint8_t> masked(numInst, 0);
	for(uint32_t m : sc->maskedInstances) if(m < numInst) masked[m] = 1;
	const uint32_t numSlots = uint32_t(std::max<size_t>(sc->slotMaterials.size(), 1));
	for(uint32_t i = 0; i < numInst; ++i) {
		if(masked[i]) continue;
		const HostInstance& hi = *inst.instances[i];
		if(hi.frame != NO_FRAME && hi.frame != 0) continue;
		HostObject* obj = hi.object;
		if(!obj || obj->lods.empty()) continue;
		if(std::find(sc->maskedObjects.begin(), sc->maskedObjects.end(), obj) != sc->maskedObjects.end()) continue;
		const uint32_t level = sc->effective_lod(hi);
		auto lit = obj->lods.find(level);
		if(lit == obj->lods.end()) {
			err = "object '" + obj->name + "' has no LoD " + std::to_string(level);
			return false;
		}
		const HostLod* lod = lit->second.get();
		auto it = lodIndex.find(lod);
		if(it == lodIndex.end()) {
			// every material index must name a slot of the scenario: the device reads materials[index]
			uint32_t maxMat = 0;
			for(uint16_t m : lod->triMat) maxMat = std::max<uint32_t>(maxMat, m);
			for(uint16_t m : lod->quadMat) maxMat = std::max<uint32_t>(maxMat, m);
			for(uint16_t m : lod->sphereMat) maxMat = std::max<uint32_t>(maxMat, m);
			if(lod->num_prims() > 0 && maxMat >= numSlots) {
				err = "object '" + obj->name + "' uses material index " + std::to_string(maxMat) + " but the scenario declares "
				      + std::to_string(sc->slotMaterials.size()) + " material slots";
				return false;
			}
			const uint32_t idx = uint32_t(D.lodSources.size());
			lodIndex[lod] = idx;
			D.lodSources.push_back(lod);
			instLod[i] = idx;
		} else instLod[i] = it->second;
	}
	// --- upload LoDs and build their BVHs
	for(size_t li = D.lodSources.size(); li < D.lods.size(); ++li) D.lods[li].release();
	D.lods.resize(D.lodSources.size());
	std::vector<DLod> dl(std::max<size_t>(D.lods.size(), 1));
	for(size_t li = 0; li < D.lods.size(); ++li) {
		const HostLod& h = *D.lodSources[li];
		DeviceLod& g = D.lods[li];
		auto tu = clk::now();
		if(!upload(g.vertices, g.cap[0], h.vertices.data(), h.vertices.size(), s, err, (const float*)nullptr, 0, &h2d)) return false;
		if(!upload(g.normals, g.cap[1], h.normals.data(), h.normals.size(), s, err, (const float*)nullptr, 0, &h2d)) return false;
		if(!upload(g.uvs, g.cap[2], h.uvs.data(), h.uvs.size(), s, err, (const float*)nullptr, 0, &h2d)) return false;
		if(!upload(g.indices, g.cap[3], h.triIdx.data(), h.triIdx.size(), s, err, h.quadIdx.data(), h.quadIdx.size(), &h2d)) return false;
		if(!upload(g.faceMat, g.cap[4], h.triMat.data(), h.triMat.size(), s, err, h.quadMat.data(), h.quadMat.size(), &h2d)) return false;
		if(!upload(g.spheres, g.cap[5], reinterpret_cast<const float4*>(h.spheres.data()), h.spheres.size() / 4, s, err,
		           (const float4*)nullptr, 0, &h2d)) return false;
		if(!upload(g.sphereMat, g.cap[6], h.sphereMat.data(), h.sphereMat.size(), s, err, (const uint16_t*)nullptr, 0, &h2d)) return false;
		LodBuildInput in{};
		in.numTriangles = h.num_triangles(); in.numQuads = h.num_quads(); in.numSpheres = h.num_spheres();
		in.vertices = g.vertices; in.indices = g.indices; in.spheres = g.spheres;
		h.bounds(in.aabbMin, in.aabbMax);
		cudaStreamSynchronize(s);
		uploadMs += msSince(tu);
		auto tb = clk::now();
		cudaError_t e = inst.builder.build_lod(in, g.bvh, s);
		if(e != cudaSuccess) { err = std::string("LBVH build failed: ") + cudaGetErrorString(e); return false; }
		bvhMs += msSince(tb);
		DLod d{};
		d.numTriangles = in.numTriangles; d.numQuads = in.numQuads; d.numSpheres = in.numSpheres;
		d.numPrims = int32_t(h.num_prims());
		d.numInternal = g.bvh.numInternal;
		d.nodes = g.bvh.nodes; d.primIds = g.bvh.primIds; d.triSoup = g.bvh.triSoup;
		d.wnodes = g.bvh.wnodes; d.wprims = g.bvh.wprims; d.wsoup = g.bvh.wsoup; d.numWide = g.bvh.numWide;
		d.vertices = g.vertices; d.normals = g.normals; d.uvs = g.uvs; d.indices = g.indices;
		d.faceMaterials = g.faceMat; d.spheres = g.spheres; d.sphereMaterials = g.sphereMat;
		std::memcpy(d.aabbMin, in.aabbMin, sizeof(d.aabbMin));
		std::memcpy(d.aabbMax, in.aabbMax, sizeof(d.aabbMax));
		g.desc = d;
		dl[li] = d;
	}
	const auto tInst = clk::now();
	if(!upload(D.dLods, D.cap[0], dl.data(), D.lods.size(), s, err)) return false;

	// --- instance transforms, boxes, scene box (scene.cpp:203-303)
	std::vector<float4> w2i(size_t(std::max<uint32_t>(numInst, 1)) * 3);
	std::vector<float> boxes(size_t(std::max<uint32_t>(numInst, 1)) * 6, 0.0f), cents(size_t(std::max<uint32_t>(numInst, 1)) * 3, 0.0f);
	Box sceneBox = empty_box();
	int32_t active = 0;
	uint32_t valid = 0xFFFFFFFFu;
	for(uint32_t i = 0; i < numInst; ++i) {
		const float* m = inst.instances[i]->worldToInstance;
		w2i[3 * i] = make_float4(m[0], m[1], m[2], m[3]);
		w2i[3 * i + 1] = make_float4(m[4], m[5], m[6], m[7]);
		w2i[3 * i + 2] = make_float4(m[8], m[9], m[10], m[11]);
		if(instLod[i] == 0xFFFFFFFFu) { st3(&boxes[6 * i], empty_box().mn); st3(&boxes[6 * i + 3], empty_box().mx); continue; }
		++active;
		if(valid == 0xFFFFFFFFu) valid = i;
		const Mat34 i2w = instance_to_world(m);
		const DLod& d = dl[instLod[i]];
		const Box lb = { ld3(d.aabbMin), ld3(d.aabbMax) };
		const Box ib = xform_box(i2w, lb);
		const V3 c = xform_point(i2w, (lb.mn + lb.mx) * 0.5f);
		st3(&boxes[6 * i], ib.mn); st3(&boxes[6 * i + 3], ib.mx);
		st3(&cents[3 * i], c);
		sceneBox = { vmin(sceneBox.mn, ib.mn), vmax(sceneBox.mx, ib.mx) };
	}
	if(!upload(D.dW2I, D.cap[1], w2i.data(), size_t(numInst) * 3, s, err)) return false;
	if(!upload(D.dInstLod, D.cap[2], instLod.data(), numInst, s, err)) return false;
	if(!upload(D.dInstBoxes, D.cap[3], boxes.data(), size_t(numInst) * 6, s, err)) return false;
	if(!upload(D.dInstCentroids, D.cap[4], cents.data(), size_t(numInst) * 3, s, err)) return false;
	if(active > 1) {
		SceneBuildInput sin{};
		sin.numInstances = numInst; sin.activeInstances = uint32_t(active);
		sin.instBoxes = D.dInstBoxes; sin.instCentroids = D.dInstCentroids; sin.instanceLod = D.dInstLod;
		st3(sin.aabbMin, sceneBox.mn); st3(sin.aabbMax, sceneBox.mx);
		cudaError_t e = inst.builder.build_scene(sin, D.tlas, s);
		if(e != cudaSuccess) { err = std::string("instance BVH build failed: ") + cudaGetErrorString(e); return false; }
	}
	st3(D.aabb, sceneBox.mn); st3(D.aabb + 3, sceneBox.mx);
	const float instMs = msSince(tInst);
	const auto tLights = clk::now();

	// --- lights (world_container.cpp:869-990)
	std::vector<HostLight> lights;
	for(uint32_t i = 0; i < numInst; ++i) {
		if(instLod[i] == 0xFFFFFFFFu) continue;
		const HostLod& h = *D.lodSources[instLod[i]];
		const Mat34 i2w = instance_to_world(inst.instances[i]->worldToInstance);
		const float* m = i2w.m;
		const float det3 = m[0] * (m[5] * m[10] - m[9] * m[6]) - m[1] * (m[4] * m[10] - m[8] * m[6]) + m[2] * (m[4] * m[9] - m[8] * m[5]);
		const bool mirroring = det3 < 0.0f;
		const uint32_t nT = h.num_triangles();
		for(uint32_t q = 0; q < h.num_quads(); ++q) {
			const uint16_t slot = h.quadMat[q];
			if(slot >= mats.size() || mats[slot].type != MAT_EMISSIVE) continue;
			V3 pts[4]; float uv[4][2];
			for(int k = 0; k < 4; ++k) {
				const uint32_t vi = h.quadIdx[4 * q + k];
				pts[k] = xform_point(i2w, ld3(&h.vertices[3 * vi]));
				uv[k][0] = h.uvs.empty() ? 0.0f : h.uvs[2 * vi];
				uv[k][1] = h.uvs.empty() ? 0.0f : h.uvs[2 * vi + 1];
			}
			if(mirroring) { std::swap(pts[1], pts[3]); std::swap(uv[1], uv[3]); }
			HostLight L{};
			L.type = LT_QUAD;
			L.posV[0] = pts[0];
			L.posV[1] = pts[3] - pts[0];
			L.posV[2] = pts[1] - pts[0];
			L.posV[3] = (pts[2] - pts[3]) - L.posV[2];
			for(int c = 0; c < 2; ++c) {
				L.uvV[0][c] = uv[0][c];
				L.uvV[1][c] = uv[3][c] - uv[0][c];
				L.uvV[2][c] = uv[1][c] - uv[0][c];
				L.uvV[3][c] = (uv[2][c] - uv[3][c]) - L.uvV[2][c];
			}
			L.material = slot;
			L.primInst = int32_t(i);
			L.primId = int32_t(nT + q);
			lights.push_back(L);
		}
	}
	for(uint32_t li : sc->pointLights) {
		if(li >= inst.pointLights.size()) continue;
		HostLight L{};
		L.type = LT_POINT;
		L.position = ld3(inst.pointLights[li].position);
		L.intensity = ld3(inst.pointLights[li].intensity);
		lights.push_back(L);
	}
	if(lights.size() > 1) {
		const V3 scale = sceneBox.mx - sceneBox.mn;
		auto conv = [](float v) { return v <= 0.0f ? 0u : (v >= 4294967040.0f ? 0xFFFFFF00u : uint32_t(v)); };
		auto p16 = [](uint32_t x) {
			uint64_t r = x & 0xFFFF;
			r = (r | (r << 16)) & 0x0000ff0000ffull;
			r = (r | (r << 8)) & 0x00f00f00f00full;
			r = (r | (r << 4)) & 0x0c30c30c30c3ull;
			r = (r | (r << 2)) & 0x249249249249ull;
			return r;
		};
		auto hilbert = [&](uint32_t a, uint32_t b, uint32_t c) {
			uint64_t num = p16(a) | (p16(b) << 1u) | (p16(c) << 2u);
			num = num ^ (num >> 32); num = num ^ (num >> 16); num = num ^ (num >> 8);
			num = num ^ (num >> 4); num = num ^ (num >> 2); num = num ^ (num >> 1);
			return num;
		};
		std::stable_sort(lights.begin(), lights.end(), [&](const HostLight& a, const HostLight& b) {
			const V3 ca = light_center(a) * scale, cb = light_center(b) * scale;
			const uint32_t ax = conv(ca.x), ay = conv(ca.y), az = conv(ca.z);
			const uint32_t bx = conv(cb.x), by = conv(cb.y), bz = conv(cb.z);
			uint64_t A = hilbert(ax >> 16, ay >> 16, az >> 16), B = hilbert(bx >> 16, by >> 16, bz >> 16);
			if(A == B) { A = hilbert(ax & 0xffff, ay & 0xffff, az & 0xffff); B = hilbert(bx & 0xffff, by & 0xffff, bz & 0xffff); }
			return A < B;
		});
	}
	LightTreeOut T = build_pos_tree(lights, mats);
	std::vector<DLight> dlights(std::max<size_t>(lights.size(), 1));
	for(size_t i = 0; i < lights.size(); ++i) {
		DLight& d = dlights[i];
		d = DLight{};
		d.type = lights[i].type;
		d.material = lights[i].material;
		st3(d.position, lights[i].position);
		st3(d.intensity, lights[i].intensity);
		for(int k = 0; k < 4; ++k) { st3(d.posV[k], lights[i].posV[k]); d.uvV[k][0] = lights[i].uvV[k][0]; d.uvV[k][1] = lights[i].uvV[k][1]; }
	}
	std::vector<uint64_t> keys;
	std::vector<uint32_t> codes;
	for(auto& kc : T.codes) { keys.push_back(kc.first); codes.push_back(kc.second); }
	if(!upload(D.dLights, D.cap[5], dlights.data(), lights.size(), s, err)) return false;
	if(!upload(D.dLightNodes, D.cap[6], T.nodes.data(), T.nodes.size(), s, err)) return false;
	if(!upload(D.dLightKeys, D.cap[7], keys.data(), keys.size(), s, err)) return false;
	if(!upload(D.dLightCodes, D.cap[8], codes.data(), codes.size(), s, err)) return false;
	if(!upload(D.dMaterials, D.cap[9], mats.data(), mats.size(), s, err)) return false;
	// textures
	std::vector<DTexture> dtex(std::max<size_t>(texList.size(), 1));
	for(size_t t = 0; t < texList.size(); ++t) {
		float4* buf = nullptr;
		size_t bufCap = 0;
		if(!upload(buf, bufCap, reinterpret_cast<const float4*>(texList[t]->texels.data()), size_t(texList[t]->width) * texList[t]->height, s, err)) return false;
		D.textureBuffers.push_back(buf);
		D.textureSources.push_back(texList[t]);
		dtex[t] = DTexture{ texList[t]->width, texList[t]->height, buf };
	}
	if(!upload(D.dTextures, D.cap[10], dtex.data(), texList.size(), s, err)) return false;

	// --- scene descriptor
	DScene& S = D.desc;
	S = DScene{};
	S.lods = D.dLods; S.numLods = uint32_t(D.lods.size());
	S.worldToInstance = D.dW2I; S.instanceLod = D.dInstLod; S.numInstances = numInst;
	S.activeInstances = active; S.validInstance = valid;
	S.tlasNodes = D.tlas.nodes; S.tlasPrimIds = D.tlas.primIds; S.tlasNumInternal = D.tlas.numInternal;
	S.tlasWide = D.tlas.wnodes; S.tlasWidePrims = D.tlas.wprims; S.tlasNumWide = D.tlas.numWide;
	S.materials = D.dMaterials; S.textures = D.dTextures;
	S.lights = D.dLights; S.lightNodes = D.dLightNodes; S.lightPrimKeys = D.dLightKeys; S.lightPrimCodes = D.dLightCodes;
	S.numLightPrims = uint32_t(keys.size());
	S.rootFlux = T.rootFlux; S.rootType = T.rootType; S.rootIndex = T.rootIndex;
	S.dirFlux = 0.0f;
	S.hasBackground = 0;
	if(sc->background >= 0 && size_t(sc->background) < inst.backgrounds.size()) {
		const HostBackground& bg = inst.backgrounds[sc->background];
		S.hasBackground = 1;
		std::memcpy(S.bgColor, bg.color, sizeof(S.bgColor));
		std::memcpy(S.bgScale, bg.scale, sizeof(S.bgScale));
		// background.cpp:125-135
		const V3 diag = sceneBox.mx - sceneBox.mn;
		const float solidAngle = 4.0f * PI;
		const float area = 2.0f * PI * ((diag.x * diag.y + diag.x * diag.z) + diag.y * diag.z);
		const float f = solidAngle * area;
		st3(S.bgFlux, ld3(bg.color) * f);
	}
	st3(S.aabbMin, sceneBox.mn); st3(S.aabbMax, sceneBox.mx);
	// camera (camera.hpp:81-96, pinhole.hpp:22)
	{
		const HostCamera& c = *sc->camera;
		V3 dir = normalize(ld3(c.dir));
		V3 up = normalize(ld3(c.up));
		const float zDotY = dot(dir, up);
		up = normalize(up - zDotY * dir);
		st3(S.camera.position, ld3(c.position));
		st3(S.camera.viewDir, dir);
		st3(S.camera.up, up);
		S.camera.tanVFov = std::tan(c.vFov / 2.0f);
		S.camera.resX = uint16_t(sc->width);
		S.camera.resY = uint16_t(sc->height);
	}
	cudaError_t e = cudaStreamSynchronize(s);
	if(e != cudaSuccess) { err = std::string("scene upload failed: ") + cudaGetErrorString(e); return false; }
	cudaStreamSynchronize(s);
	D.loadMs[0] = msSince(t0);
	D.loadMs[1] = uploadMs;
	D.loadMs[2] = bvhMs;
	D.loadMs[3] = instMs;
	D.loadMs[4] = msSince(tLights);
	D.loadH2dBytes = h2d;
	D.valid = true;
	return true;
}

} // namespace mb
