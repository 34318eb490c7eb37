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
#include "light_build.hpp"
#include "instance_boxes.hpp"

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

// Grows a device buffer to hold at least count elements (contents are not kept).
template < class T >
bool reserve_device(T*& p, size_t& cap, size_t count, std::string& err) {
	if(count <= cap && p) return true;
	if(p) cudaFree(p);
	p = nullptr;
	cap = 0;
	const cudaError_t e = cudaMalloc(reinterpret_cast<void**>(&p), sizeof(T) * std::max<size_t>(count, 1));
	if(e != cudaSuccess) { err = std::string("device allocation failed: ") + cudaGetErrorString(e); return false; }
	cap = std::max<size_t>(count, 1);
	return true;
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
	cudaFree(dInstI2W); cudaFree(dWideInstBoxes); cudaFree(dLightMirror); cudaFree(dLightFirst); cudaFree(dLightLods);
	cudaFree(dEmissiveQuads); cudaFree(dQuadMaterial); cudaFree(dPointLights);
	dInstI2W = nullptr; dWideInstBoxes = nullptr; wideBoxCap = 0; dLightMirror = nullptr; dLightFirst = nullptr; dLightLods = nullptr;
	dEmissiveQuads = nullptr; dQuadMaterial = nullptr; dPointLights = nullptr;
	for(size_t& c : lightCap) c = 0;
	lightScratch.release();
	numLights = numLightNodes = 0;
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
	bool hasAlpha = false;
	for(size_t i = 0; i < sc->slotMaterials.size(); ++i) {
		const HostMaterial* m = sc->slotMaterials[i];
		DMaterial& d = mats[i];
		d = DMaterial{};
		d.albedoTex = -1;
		d.alphaTex = -1;
		if(!m) { d.type = MAT_LAMBERT; continue; }
		if(m->alpha) {
			d.alphaTex = int32_t(texList.size());
			texList.push_back(m->alpha);
			hasAlpha = true;
		}
		d.type = m->type;
		d.shadowing = m->shadowing;
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
			if(m->emissionOverride) st3(d.radiance, ld3(m->emission));
			else st3(d.radiance, tex_value(m->radiance, V3{ 0, 0, 0 }) * ld3(m->scale));
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
	std::vector<float> i2wAll(size_t(std::max<uint32_t>(numInst, 1)) * 12, 0.0f);
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
		std::memcpy(&i2wAll[12 * size_t(i)], i2w.m, sizeof(i2w.m));
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
	if(!upload(D.dInstI2W, D.lightCap[0], i2wAll.data(), size_t(numInst) * 12, s, err)) return false;
	if(active > 1) {
		SceneBuildInput sin{};
		sin.numInstances = numInst; sin.activeInstances = uint32_t(active);
		sin.instBoxes = D.dInstBoxes; sin.instCentroids = D.dInstCentroids; sin.instanceLod = D.dInstLod;
		st3(sin.aabbMin, sceneBox.mn); st3(sin.aabbMax, sceneBox.mx);
		// the 8-wide instance level is refitted to tight boxes (instance_boxes.cu)
		if(!reserve_device(D.dWideInstBoxes, D.wideBoxCap, size_t(numInst) * 6, err)) return false;
		cudaError_t e = tight_instance_boxes(D.dLods, D.dInstLod, D.dInstI2W, numInst, D.dInstBoxes, D.dWideInstBoxes, s);
		if(e != cudaSuccess) { err = std::string("instance boxes failed: ") + cudaGetErrorString(e); return false; }
		sin.wideBoxes = D.dWideInstBoxes;
		e = inst.builder.build_scene(sin, D.tlas, s);
		if(e != cudaSuccess) { err = std::string("instance BVH build failed: ") + cudaGetErrorString(e); return false; }
	}
	st3(D.aabb, sceneBox.mn); st3(D.aabb + 3, sceneBox.mx);
	const float instMs = msSince(tInst);
	const auto tLights = clk::now();

	// --- lights (world_container.cpp:869-990), list and tree built on the GPU (light_build.cu)
	if(!upload(D.dMaterials, D.cap[9], mats.data(), mats.size(), s, err)) return false;
	// world_container.cpp:929-990: emissive triangles, quads and spheres
	// become area lights (in that order, per instance). Emissive primitives
	// are listed once per LoD.
	std::vector<uint32_t> lodQuadStart(D.lodSources.size(), 0), lodQuadCount(D.lodSources.size(), 0);
	std::vector<uint32_t> lodSphereCount(D.lodSources.size(), 0);
	std::vector<uint32_t> emissiveQuads;
	std::vector<uint16_t> quadMaterial;
	// Scenes without emissive materials (only point lights or the background)
	// skip the per-face scan: for the 1.31 M-triangle mesh it took 1.3 ms of
	// every scene load.
	bool anyEmissive = false;
	for(const DMaterial& m : mats) anyEmissive = anyEmissive || m.type == MAT_EMISSIVE;
	for(size_t li = 0; li < D.lodSources.size() && anyEmissive; ++li) {
		const HostLod& h = *D.lodSources[li];
		auto emissive = [&](uint16_t m) { return m < mats.size() && mats[m].type == MAT_EMISSIVE; };
		lodQuadStart[li] = uint32_t(emissiveQuads.size());
		for(uint32_t t = 0; t < h.num_triangles(); ++t)
			if(emissive(h.triMat[t])) { emissiveQuads.push_back(t); quadMaterial.push_back(h.triMat[t]); }
		for(uint32_t q = 0; q < h.num_quads(); ++q)
			if(emissive(h.quadMat[q])) { emissiveQuads.push_back(h.num_triangles() + q); quadMaterial.push_back(h.quadMat[q]); }
		const uint32_t faces = h.num_triangles() + h.num_quads();
		for(uint32_t k = 0; k < h.num_spheres(); ++k)
			if(emissive(h.sphereMat[k])) { emissiveQuads.push_back(faces + k); quadMaterial.push_back(h.sphereMat[k]); ++lodSphereCount[li]; }
		lodQuadCount[li] = uint32_t(emissiveQuads.size()) - lodQuadStart[li];
	}
	// per instance: instance-to-world, mirroring, first light index (area lights in instance order)
	std::vector<uint8_t> lightMirror(std::max<uint32_t>(numInst, 1), 0);
	std::vector<uint32_t> firstLight(size_t(numInst) + 1, 0);
	uint64_t numArea64 = 0, numSphere64 = 0;
	for(uint32_t i = 0; i < numInst; ++i) {
		firstLight[i] = uint32_t(numArea64);
		if(instLod[i] == 0xFFFFFFFFu || lodQuadCount[instLod[i]] == 0) continue;
		numSphere64 += lodSphereCount[instLod[i]];
		const float* m = &i2wAll[12 * size_t(i)];
		const float det3 = m[0] * (m[5] * m[10] - m[9] * m[6]) - m[1] * (m[4] * m[10] - m[8] * m[6]) + m[2] * (m[4] * m[9] - m[8] * m[5]);
		lightMirror[i] = det3 < 0.0f ? 1 : 0;
		numArea64 += lodQuadCount[instLod[i]];
	}
	firstLight[numInst] = uint32_t(numArea64);
	std::vector<float> pointData;
	for(uint32_t li : sc->pointLights) {
		if(li >= inst.pointLights.size()) continue;
		const HostPointLight& P = inst.pointLights[li];
		pointData.insert(pointData.end(), { P.position[0], P.position[1], P.position[2], P.intensity[0], P.intensity[1], P.intensity[2] });
	}
	const uint64_t numLights64 = numArea64 + pointData.size() / 6;
	if(numLights64 >= (uint64_t(1) << 30)) { err = "too many lights for the light tree"; return false; }
	const uint32_t numArea = uint32_t(numArea64), numLights = uint32_t(numLights64);
	std::vector<LightLodInfo> lodInfo(std::max<size_t>(D.lodSources.size(), 1));
	for(size_t li = 0; li < D.lodSources.size(); ++li) {
		const HostLod& h = *D.lodSources[li];
		lodInfo[li] = LightLodInfo{ D.lods[li].vertices, h.uvs.empty() ? nullptr : D.lods[li].uvs, D.lods[li].indices,
		                            h.num_triangles(), lodQuadStart[li], h.num_quads(), D.lods[li].spheres };
	}
	if(!upload(D.dLightMirror, D.lightCap[1], lightMirror.data(), numArea ? lightMirror.size() : 0, s, err)) return false;
	if(!upload(D.dLightFirst, D.lightCap[2], firstLight.data(), numArea ? firstLight.size() : 0, s, err)) return false;
	if(!upload(D.dLightLods, D.lightCap[3], lodInfo.data(), numArea ? D.lodSources.size() : 0, s, err)) return false;
	if(!upload(D.dEmissiveQuads, D.lightCap[4], emissiveQuads.data(), emissiveQuads.size(), s, err)) return false;
	if(!upload(D.dQuadMaterial, D.lightCap[5], quadMaterial.data(), quadMaterial.size(), s, err)) return false;
	if(!upload(D.dPointLights, D.lightCap[6], pointData.data(), pointData.size(), s, err)) return false;
	if(!reserve_device(D.dLights, D.cap[5], numLights, err) || !reserve_device(D.dLightNodes, D.cap[6], numLights, err) ||
	   !reserve_device(D.dLightKeys, D.cap[7], numLights, err) || !reserve_device(D.dLightCodes, D.cap[8], numLights, err))
		return false;
	LightBuildInput lin{};
	lin.numInstances = numInst;
	lin.instLod = D.dInstLod;
	lin.instToWorld = D.dInstI2W;
	lin.mirroring = D.dLightMirror;
	lin.instFirstLight = D.dLightFirst;
	lin.lods = D.dLightLods;
	lin.emissiveFaces = D.dEmissiveQuads;
	lin.faceMaterial = D.dQuadMaterial;
	lin.numArea = numArea;
	lin.pointLights = D.dPointLights;
	lin.numPoint = numLights - numArea;
	lin.materials = D.dMaterials;
	st3(lin.sceneScale, sceneBox.mx - sceneBox.mn);
	LightTreeInfo tree;
	{
		const cudaError_t e = build_lights_gpu(lin, D.lightScratch, inst.builder,
		                                       LightBuildOutput{ D.dLights, D.dLightNodes, D.dLightKeys, D.dLightCodes }, tree, s);
		if(e != cudaSuccess) { err = std::string("light tree build failed: ") + cudaGetErrorString(e); return false; }
	}
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
	S.maxSteps = MAX_TRAVERSAL_STEPS;
	S.hasAlpha = hasAlpha ? 1 : 0;
	S.sphereLights = numSphere64 > 0 ? 1 : 0;
	S.tlasNodes = D.tlas.nodes; S.tlasPrimIds = D.tlas.primIds; S.tlasNumInternal = D.tlas.numInternal;
	S.tlasWide = D.tlas.wnodes; S.tlasWidePrims = D.tlas.wprims; S.tlasNumWide = D.tlas.numWide;
	S.materials = D.dMaterials; S.textures = D.dTextures;
	S.lights = D.dLights; S.lightNodes = D.dLightNodes; S.lightPrimKeys = D.dLightKeys; S.lightPrimCodes = D.dLightCodes;
	S.numLightPrims = numArea;
	S.rootFlux = tree.rootFlux; S.rootType = tree.rootType; S.rootIndex = tree.rootIndex;
	D.numLights = numLights; D.numLightNodes = tree.numNodes;
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
