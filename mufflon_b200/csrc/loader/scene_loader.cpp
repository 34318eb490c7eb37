// Scene-file import (src/mffloader/parsing/json_loader.cpp, binary.cpp).
//
// Order of work, as JsonLoader::load_file (json_loader.cpp:1036-1184) does it:
// JSON parse and version; binary header (materials, objects, instances);
// objects, instances and default instances; cameras; world_finalize;
// scenarios (camera, resolution, global LoD, lights, per-object and
// per-instance LoD and masks, material slots); world_load_scenario of the
// default scenario. Geometry is not read here: the core asks for each LoD
// the loaded scenario needs through the LoD-loader callback
// (mufflon_set_lod_loader), which reads it from the still open binary file.
//
// Materials and lights are created when the first scenario uses them, so a
// file that also describes models the CUDA path tracer does not implement
// still loads as long as no scenario uses them; a scenario that does use one
// fails with the core's message.
#include "scene_loader.hpp"
#include "../common/pfm.hpp"

#include <cctype>
#include <cmath>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <limits>
#include <sstream>
#include <unordered_map>

namespace mffl {

namespace fs = std::filesystem;

namespace {

constexpr float PI_F = 3.14159265358979323846f;

[[noreturn]] void core_fail(const std::string& what) {
	const char* e = core_get_dll_error();
	throw LoaderError(what + ((e && *e) ? std::string(": ") + e : std::string()));
}

// Typed access to the JSON document; messages carry the member path.
class Reader {
public:
	std::vector<std::string> path;

	std::string where() const {
		std::string s;
		for(const auto& p : path) { if(!s.empty()) s += '/'; s += p; }
		return s;
	}
	[[noreturn]] void fail(const std::string& m) const {
		throw LoaderError(path.empty() ? m : where() + ": " + m);
	}
	const JsonValue& object(const JsonValue& v, const std::string& what) const {
		if(!v.is_object()) fail(what + ": expected an object, got " + type_name(v.type));
		return v;
	}
	const JsonValue& req(const JsonValue& o, const std::string& key) const {
		if(!o.is_object()) fail("expected an object, got " + std::string(type_name(o.type)));
		const JsonValue* v = o.find(key);
		if(!v) fail("missing '" + key + "'");
		return *v;
	}
	const JsonValue* opt(const JsonValue& o, const std::string& key) const { return o.is_object() ? o.find(key) : nullptr; }
	float num(const JsonValue& v, const std::string& what) const {
		if(!v.is_number()) fail(what + ": expected a number, got " + type_name(v.type));
		return float(v.number);
	}
	uint32_t uint(const JsonValue& v, const std::string& what) const {
		if(!v.is_number() || v.number < 0.0 || v.number > 4294967295.0 || std::floor(v.number) != v.number)
			fail(what + ": expected a non-negative integer");
		return uint32_t(v.number);
	}
	bool flag(const JsonValue& v, const std::string& what) const {
		if(!v.is_bool()) fail(what + ": expected true or false, got " + type_name(v.type));
		return v.boolean;
	}
	std::string text(const JsonValue& v, const std::string& what) const {
		if(!v.is_string()) fail(what + ": expected a string, got " + type_name(v.type));
		return v.string;
	}
	void numbers(const JsonValue& v, size_t n, float* out, const std::string& what) const {
		if(!v.is_array() || v.array.size() != n) fail(what + ": expected an array of " + std::to_string(n) + " numbers");
		for(size_t i = 0; i < n; ++i) out[i] = num(v.array[i], what);
	}
	Vec3 vec3(const JsonValue& v, const std::string& what) const { float f[3]; numbers(v, 3, f, what); return Vec3{ f[0], f[1], f[2] }; }
	Vec2 vec2(const JsonValue& v, const std::string& what) const { float f[2]; numbers(v, 2, f, what); return Vec2{ f[0], f[1] }; }
	// [[x,y,z], ...] or a single [x,y,z]
	std::vector<Vec3> vec3_list(const JsonValue& v, const std::string& what) const {
		std::vector<Vec3> out;
		if(v.is_array() && !v.array.empty() && v.array[0].is_array()) {
			for(const auto& e : v.array) out.push_back(vec3(e, what));
		} else out.push_back(vec3(v, what));
		return out;
	}
	// [a, b, ...] or a single number
	std::vector<float> float_list(const JsonValue& v, const std::string& what) const {
		std::vector<float> out;
		if(v.is_array()) for(const auto& e : v.array) out.push_back(num(e, what));
		else out.push_back(num(v, what));
		if(out.empty()) fail(what + ": empty list");
		return out;
	}
};

struct Scope {
	Reader& r;
	Scope(Reader& reader, std::string s) : r(reader) { r.path.push_back(std::move(s)); }
	~Scope() { r.path.pop_back(); }
};

// Replaces the whole member path for a nested definition (a material or a
// light referenced from a scenario) and puts the caller's path back on every
// exit, exceptions included, so that the enclosing Scopes pop what they pushed.
struct PathSwap {
	Reader& r;
	std::vector<std::string> saved;
	PathSwap(Reader& reader, std::vector<std::string> path) : r(reader), saved(std::move(reader.path)) { r.path = std::move(path); }
	~PathSwap() { r.path = std::move(saved); }
};

// Brings lists of per-frame values to one length: a list of length one is
// repeated (json_loader.cpp load_lights / load_cameras).
template < class T >
void broadcast(std::vector<T>& v, size_t n) { if(v.size() == 1 && n != 1) v.assign(n, v.front()); }

std::string read_text_file(const fs::path& p) {
	std::ifstream f(p, std::ios::binary);
	if(!f) throw LoaderError("cannot open scene file '" + p.string() + "'");
	std::ostringstream ss;
	ss << f.rdbuf();
	return ss.str();
}

FileVersion parse_version(const std::string& s, const Reader& r) {
	FileVersion v{ 0, 0 };
	const size_t dot = s.find('.');
	try {
		size_t used = 0;
		v.major = unsigned(std::stoul(s.substr(0, dot), &used));
		if(used != dot && dot != std::string::npos) r.fail("malformed version '" + s + "'");
		v.minor = dot == std::string::npos ? 0u : unsigned(std::stoul(s.substr(dot + 1)));
	} catch(const std::logic_error&) {
		r.fail("malformed version '" + s + "'");
	}
	return v;
}

// Portable float map ("PF": RGB, little-endian when the scale is negative),
// rows as stored, alpha 0 (src/pfmloader/interface.cpp:80-150).
std::vector<float> read_pfm_rgb(const fs::path& p, uint32_t& w, uint32_t& h) {
	const std::string data = read_text_file(p);
	if(data.size() >= 2 && data.compare(0, 2, "Pf") == 0)
		throw LoaderError("texture '" + p.string() + "': single-channel PFM textures are not supported for colours");
	if(data.size() >= 2 && data.compare(0, 2, "PF") != 0)
		throw LoaderError("texture '" + p.string() + "': only PFM (\"PF\") textures are read by this loader");
	try {
		mb::PfmImage img = mb::parse_pfm(data);
		w = img.width;
		h = img.height;
		return std::move(img.rgba);
	} catch(const std::runtime_error& e) {
		throw LoaderError("texture '" + p.string() + "': " + e.what());
	}
}

void transform_box(const float* m, const float* mn, const float* mx, float* outMin, float* outMax) {
	for(int k = 0; k < 3; ++k) { outMin[k] = std::numeric_limits<float>::max(); outMax[k] = -std::numeric_limits<float>::max(); }
	for(int c = 0; c < 8; ++c) {
		const float p[3] = { (c & 1) ? mx[0] : mn[0], (c & 2) ? mx[1] : mn[1], (c & 4) ? mx[2] : mn[2] };
		for(int r = 0; r < 3; ++r) {
			const float q = m[4 * r] * p[0] + m[4 * r + 1] * p[1] + m[4 * r + 2] * p[2] + m[4 * r + 3];
			outMin[r] = std::min(outMin[r], q);
			outMax[r] = std::max(outMax[r], q);
		}
	}
}

class SceneFileLoader {
public:
	SceneFileLoader(LoaderState& state, const fs::path& file) : m_st(state), m_core(state.core), m_file(file) {}

	void load() {
		m_st.set_status("Loading JSON");
		const std::string text = read_text_file(m_file);
		m_doc = parse_json(text);
		r.object(m_doc, "scene file");

		if(const JsonValue* v = r.opt(m_doc, "version")) {
			Scope s(r, "version");
			m_version = parse_version(r.text(*v, "version"), r);
			if(CURRENT_VERSION < m_version)
				m_st.warn("scene file version " + std::to_string(m_version.major) + "." + std::to_string(m_version.minor)
				          + " is newer than the supported 1.7");
		} else {
			m_st.warn("scene file has no version; 1.7 assumed");
			m_version = CURRENT_VERSION;
		}
		m_st.version = m_version;

		fs::path bin = r.text(r.req(m_doc, "binary"), "binary");
		if(bin.empty()) r.fail("empty binary file path");
		if(bin.is_relative()) bin = m_file.parent_path() / bin;
		if(!fs::exists(bin)) throw LoaderError("binary file '" + bin.string() + "' does not exist");

		m_lights = &r.object(r.req(m_doc, "lights"), "lights");
		m_scenarios = &r.object(r.req(m_doc, "scenarios"), "scenarios");
		m_cameras = &r.object(r.req(m_doc, "cameras"), "cameras");
		m_materials = &r.object(r.req(m_doc, "materials"), "materials");
		if(m_scenarios->members.empty()) r.fail("the file has no scenario");
		m_default = m_scenarios->members.front().first;
		if(const JsonValue* v = r.opt(m_doc, "defaultScenario")) {
			const std::string name = r.text(*v, "defaultScenario");
			if(!name.empty()) m_default = name;
		}
		if(!m_scenarios->find(m_default)) r.fail("default scenario '" + m_default + "' does not exist");
		const bool deinstance = r.opt(m_doc, "deinstance") ? r.flag(*r.opt(m_doc, "deinstance"), "deinstance") : false;
		const bool noDefaultInstances = r.opt(m_doc, "noDefaultInstances")
			? r.flag(*r.opt(m_doc, "noDefaultInstances"), "noDefaultInstances") : false;
		if(deinstance)
			m_st.warn("'deinstance' is not applied: instances are traced through the two-level hierarchy (same geometry)");
		if(const JsonValue* v = r.opt(m_doc, "initTessellationLevel"); v && r.num(*v, "initTessellationLevel") > 0.0f)
			m_st.warn("'initTessellationLevel' is ignored: the path tracer does not tessellate");
		m_st.check_abort();

		m_st.set_status("Loading binary file");
		m_st.binary = std::make_unique<MffFile>();
		m_st.binary->open(bin.string());
		const MffFile& B = *m_st.binary;
		if(B.bone_count() > 0 && B.bone_frames() > 0)
			throw LoaderError("binary file '" + bin.string() + "' holds a skeletal animation ("
			                  + std::to_string(B.bone_count()) + " bones), which the path tracer does not support");
		load_objects_and_instances(noDefaultInstances);
		m_st.check_abort();

		m_st.set_status("Parsing cameras");
		load_cameras();
		m_st.check_abort();

		m_st.set_status("Checking world sanity");
		const char* msg = "";
		if(!world_finalize(m_core, Vec3{ m_aabbMin[0], m_aabbMin[1], m_aabbMin[2] },
		                   Vec3{ m_aabbMax[0], m_aabbMax[1], m_aabbMax[2] }, &msg))
			core_fail("world did not pass the sanity check");

		m_st.set_status("Parsing scenarios");
		load_scenarios();
		m_st.check_abort();

		m_st.set_status("Loading initial scenario");
		ScenarioHdl def = world_find_scenario(m_core, m_default.c_str());
		if(!def) core_fail("cannot find the default scenario '" + m_default + "'");
		m_st.lodError.clear();
		if(!world_load_scenario(m_core, def)) {
			const std::string why = m_st.lodError.empty() ? std::string() : " (" + m_st.lodError + ")";
			core_fail("cannot load the default scenario '" + m_default + "'" + why);
		}
		m_st.set_status("Done");
	}

private:
	LoaderState& m_st;
	MufflonInstanceHdl m_core;
	fs::path m_file;
	Reader r;
	JsonValue m_doc;
	FileVersion m_version{};
	const JsonValue* m_lights = nullptr;
	const JsonValue* m_scenarios = nullptr;
	const JsonValue* m_cameras = nullptr;
	const JsonValue* m_materials = nullptr;
	std::string m_default;
	float m_aabbMin[3] = { 1e30f, 1e30f, 1e30f }, m_aabbMax[3] = { -1e30f, -1e30f, -1e30f };
	std::vector<ObjectHdl> m_objects;
	std::unordered_map<std::string, InstanceHdl> m_instanceNames;
	std::map<std::string, CameraHdl> m_cameraHdl;
	std::map<std::string, MaterialHdl> m_materialHdl;
	std::map<std::string, LightHdl> m_lightHdl;
	std::map<std::string, bool> m_lightIgnored;
	std::map<std::string, TextureHdl> m_textures;

	void grow_box(const float* mn, const float* mx) {
		for(int k = 0; k < 3; ++k) { m_aabbMin[k] = std::min(m_aabbMin[k], mn[k]); m_aabbMax[k] = std::max(m_aabbMax[k], mx[k]); }
	}

	// binary.cpp read_object / read_instances: one core object per binary
	// object (with its LoD slot count), the instances of the file, then an
	// identity instance for every object that has none.
	void load_objects_and_instances(bool noDefaultInstances) {
		const MffFile& B = *m_st.binary;
		world_reserve_objects_instances(m_core, uint32_t(B.objects().size()),
		                                uint32_t(B.instances().size() + B.objects().size()));
		m_objects.resize(B.objects().size());
		for(size_t i = 0; i < B.objects().size(); ++i) {
			if((i & 255u) == 0) m_st.check_abort();
			const MffObject& o = B.objects()[i];
			ObjectHdl h = world_create_object(m_core, o.name.c_str(), ObjectFlags(o.flags));
			if(!h) core_fail("failed to create object '" + o.name + "'");
			if(!object_allocate_lod_slots(h, uint32_t(o.lodOffsets.size()))) core_fail("failed to allocate LoD slots");
			m_objects[i] = h;
			m_st.objectIds[h] = uint32_t(i);
		}
		m_st.set_status("Loading instances");
		std::vector<uint8_t> hasInstance(B.objects().size(), 0);
		const bool worldToInstance = m_version >= WORLD_TO_INSTANCE_VERSION;
		for(size_t i = 0; i < B.instances().size(); ++i) {
			if((i & 1023u) == 0) m_st.check_abort();
			const MffInstance& in = B.instances()[i];
			InstanceHdl h = world_create_instance(m_core, m_objects[in.objectId], in.keyframe);
			if(!h) core_fail("failed to create instance '" + in.name + "'");
			Mat3x4 m;
			std::memcpy(m.v, in.transform, sizeof(m.v));
			if(!instance_set_transformation_matrix(m_core, h, &m, worldToInstance))
				core_fail("failed to set the transformation of instance '" + in.name + "'");
			Mat3x4 toWorld;
			if(!instance_get_transformation_matrix(m_core, h, &toWorld)) core_fail("failed to read an instance transformation");
			const MffObject& o = B.objects()[in.objectId];
			float mn[3], mx[3];
			transform_box(toWorld.v, o.aabbMin, o.aabbMax, mn, mx);
			grow_box(mn, mx);
			m_instanceNames[in.name] = h;
			hasInstance[in.objectId] = 1;
		}
		if(noDefaultInstances) return;
		m_st.set_status("Creating default instances");
		for(size_t i = 0; i < B.objects().size(); ++i) {
			if(hasInstance[i]) continue;
			if(!world_create_instance(m_core, m_objects[i], MFF_NO_FRAME))
				core_fail("failed to create the default instance of object '" + B.objects()[i].name + "'");
			grow_box(B.objects()[i].aabbMin, B.objects()[i].aabbMax);
		}
	}

	// json_loader.cpp load_cameras:462-535
	void load_cameras() {
		Scope s0(r, "cameras");
		float diag = 0.0f;
		if(m_aabbMax[0] >= m_aabbMin[0]) {
			const float d[3] = { m_aabbMax[0] - m_aabbMin[0], m_aabbMax[1] - m_aabbMin[1], m_aabbMax[2] - m_aabbMin[2] };
			diag = std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
		}
		const bool absolute = m_version >= ABSOLUTE_NEAR_FAR_VERSION;
		for(const auto& [name, cam] : m_cameras->members) {
			Scope s1(r, name);
			r.object(cam, "camera");
			const float nearP = r.opt(cam, "near") ? r.num(*r.opt(cam, "near"), "near") : (absolute ? 0.01f : 1e-4f * diag);
			const float farP = r.opt(cam, "far") ? r.num(*r.opt(cam, "far"), "far") : (absolute ? 500.0f : 2.0f * diag);
			const std::string type = r.text(r.req(cam, "type"), "type");
			std::vector<Vec3> pos = r.vec3_list(r.req(cam, "path"), "path");
			std::vector<Vec3> dir = r.vec3_list(r.req(cam, "viewDir"), "viewDir");
			std::vector<Vec3> up = r.opt(cam, "up") ? r.vec3_list(*r.opt(cam, "up"), "up") : std::vector<Vec3>{ Vec3{ 0, 1, 0 } };
			const size_t n = std::max(pos.size(), std::max(dir.size(), up.size()));
			broadcast(pos, n); broadcast(dir, n); broadcast(up, n);
			if(pos.size() != dir.size()) r.fail("mismatched camera path size (view direction)");
			if(pos.size() != up.size()) r.fail("mismatched camera path size (up direction)");
			if(type == "pinhole") {
				const float fov = r.opt(cam, "fov") ? r.num(*r.opt(cam, "fov"), "fov") : 25.0f;
				CameraHdl h = world_add_pinhole_camera(m_core, name.c_str(), pos.data(), dir.data(), up.data(), uint32_t(n),
				                                       nearP, farP, fov * (PI_F / 180.0f));
				if(!h) core_fail("failed to add pinhole camera '" + name + "'");
				m_cameraHdl[name] = h;
			} else if(type == "focus") {
				// created on use: the core has no thin-lens camera
			} else if(type == "ortho") {
				m_st.warn("camera '" + name + "': orthographic cameras are not supported");
			} else {
				m_st.warn("camera '" + name + "' has unknown type '" + type + "'");
			}
		}
	}

	CameraHdl camera(const std::string& name) {
		auto it = m_cameraHdl.find(name);
		if(it != m_cameraHdl.end()) return it->second;
		const JsonValue* cam = m_cameras->find(name);
		if(cam && cam->is_object() && cam->find("type") && cam->find("type")->is_string() && cam->find("type")->string == "focus")
			r.fail("camera '" + name + "' is a focus (thin-lens) camera, which the CUDA path tracer does not implement");
		r.fail("camera '" + name + "' does not exist");
	}

	TextureHdl texture_file(const std::string& rel) {
		fs::path p = rel;
		if(p.is_relative()) p = m_file.parent_path() / p;
		if(!fs::exists(p)) r.fail("cannot find texture file '" + p.string() + "'");
		const std::string key = fs::canonical(p).string();
		auto it = m_textures.find(key);
		if(it != m_textures.end()) return it->second;
		uint32_t w = 0, h = 0;
		const std::vector<float> rgba = read_pfm_rgb(p, w, h);
		TextureHdl t = world_add_texture_rgba32f(m_core, key.c_str(), w, h, rgba.data(), SAMPLING_LINEAR);
		if(!t) core_fail("failed to add texture '" + key + "'");
		m_textures[key] = t;
		return t;
	}

	TextureHdl texture_value(const float* v, int n) {
		TextureHdl t = world_add_texture_value(m_core, v, n, SAMPLING_NEAREST);
		if(!t) core_fail("failed to add a value texture");
		return t;
	}

	// An RGB value or a texture path.
	TextureHdl colour(const JsonValue& v, const std::string& what) {
		if(v.is_array()) { const Vec3 c = r.vec3(v, what); return texture_value(&c.x, 3); }
		if(v.is_string()) return texture_file(v.string);
		r.fail(what + ": expected [r,g,b] or a texture path");
	}

	// A roughness number, [alpha_x, alpha_y] or a texture path.
	TextureHdl roughness(const JsonValue& v) {
		if(v.is_number()) { const float a = float(v.number); return texture_value(&a, 1); }
		if(v.is_array()) { const Vec2 a = r.vec2(v, "roughness"); return texture_value(&a.x, 2); }
		if(v.is_string()) return texture_file(v.string);
		r.fail("roughness: expected a number, [x,y] or a texture path");
	}

	ShadowingModel shadowing(const JsonValue& m) {
		const std::string s = r.opt(m, "shadowingModel") ? r.text(*r.opt(m, "shadowingModel"), "shadowingModel") : "vcavity";
		if(s == "smith") return SHADOWING_SMITH;
		if(s == "vcavity") return SHADOWING_VCAVITY;
		r.fail("unknown shadowing model '" + s + "'");
	}
	NormalDistFunction ndf(const JsonValue& m) {
		const std::string s = r.text(r.req(m, "ndf"), "ndf");
		if(s == "BS") return NDF_BECKMANN;
		if(s == "GGX") return NDF_GGX;
		if(s == "Cos") return NDF_COSINE;
		r.fail("unknown normal distribution function '" + s + "'");
	}

	// json_loader.cpp load_material:202-397. Nested layers are kept in `keep`.
	void material_params(const JsonValue& m, MaterialParams& p, std::vector<std::unique_ptr<MaterialParams>>& keep) {
		r.object(m, "material");
		std::memset(&p, 0, sizeof(p));
		if(const JsonValue* outer = r.opt(m, "outerMedium")) {
			Scope s(r, "outerMedium");
			p.outerMedium.absorption = r.vec3(r.req(*outer, "absorption"), "absorption");
			const JsonValue& ior = r.req(*outer, "ior");
			p.outerMedium.refractionIndex = ior.is_array() ? r.vec2(ior, "ior") : Vec2{ r.num(ior, "ior"), 0.0f };
		} else {
			p.outerMedium.refractionIndex = Vec2{ 1.0f, 0.0f };
		}
		const std::string type = r.text(r.req(m, "type"), "type");
		if(r.opt(m, "displacement")) r.fail("displacement maps are not supported by the CUDA path tracer");
		if(type == "lambert") {
			p.innerType = MATERIAL_LAMBERT;
			p.inner.lambert.albedo = colour(r.req(m, "albedo"), "albedo");
		} else if(type == "torrance") {
			p.innerType = MATERIAL_TORRANCE;
			p.inner.torrance.shadowingModel = shadowing(m);
			p.inner.torrance.ndf = ndf(m);
			p.inner.torrance.roughness = roughness(r.req(m, "roughness"));
			p.inner.torrance.albedo = colour(r.req(m, "albedo"), "albedo");
		} else if(type == "walter" || type == "microfacet") {
			p.innerType = type == "walter" ? MATERIAL_WALTER : MATERIAL_MICROFACET;
			p.inner.walter.shadowingModel = shadowing(m);
			p.inner.walter.ndf = ndf(m);
			p.inner.walter.absorption = r.vec3(r.req(m, "absorption"), "absorption");
			p.inner.walter.roughness = roughness(r.req(m, "roughness"));
			p.inner.walter.refractionIndex = r.num(r.req(m, "ior"), "ior");
		} else if(type == "emissive") {
			if(r.opt(m, "alpha")) m_st.warn(r.where() + ": alpha texture of an emissive material ignored");
			p.innerType = MATERIAL_EMISSIVE;
			p.inner.emissive.scale = r.opt(m, "scale") ? r.vec3(*r.opt(m, "scale"), "scale") : Vec3{ 1.0f, 1.0f, 1.0f };
			if(const JsonValue* rad = r.opt(m, "radiance")) p.inner.emissive.radiance = colour(*rad, "radiance");
			else if(r.opt(m, "temperature")) r.fail("black-body 'temperature' emission is not supported; give 'radiance'");
			else r.fail("missing 'radiance'");
		} else if(type == "orennayar") {
			p.innerType = MATERIAL_ORENNAYAR;
			p.inner.orennayar.roughness = r.opt(m, "roughness") ? r.num(*r.opt(m, "roughness"), "roughness") : 1.0f;
			p.inner.orennayar.albedo = colour(r.req(m, "albedo"), "albedo");
		} else if(type == "blend") {
			p.innerType = MATERIAL_BLEND;
			p.inner.blend.a.factor = r.num(r.req(m, "factorA"), "factorA");
			p.inner.blend.b.factor = r.num(r.req(m, "factorB"), "factorB");
			keep.push_back(std::make_unique<MaterialParams>());
			{ Scope s(r, "layerA"); material_params(r.req(m, "layerA"), *keep.back(), keep); }
			p.inner.blend.a.mat = keep.back().get();
			keep.push_back(std::make_unique<MaterialParams>());
			{ Scope s(r, "layerB"); material_params(r.req(m, "layerB"), *keep.back(), keep); }
			p.inner.blend.b.mat = keep.back().get();
		} else if(type == "fresnel") {
			p.innerType = MATERIAL_FRESNEL;
			const JsonValue& ior = r.req(m, "ior");
			p.inner.fresnel.refractionIndex = ior.is_array() ? r.vec2(ior, "ior") : Vec2{ r.num(ior, "ior"), 0.0f };
			keep.push_back(std::make_unique<MaterialParams>());
			{ Scope s(r, "layerReflection"); material_params(r.req(m, "layerReflection"), *keep.back(), keep); }
			p.inner.fresnel.a = keep.back().get();
			keep.push_back(std::make_unique<MaterialParams>());
			{ Scope s(r, "layerRefraction"); material_params(r.req(m, "layerRefraction"), *keep.back(), keep); }
			p.inner.fresnel.b = keep.back().get();
		} else {
			r.fail("material type '" + type + "' is not supported");
		}
		// the alpha texture comes last so that emissive materials drop it
		// (json_loader.cpp:232-233, 326-329, 401-407)
		if(type != "emissive")
			if(const JsonValue* a = r.opt(m, "alpha")) {
				if(!a->is_string()) r.fail("alpha: expected a texture path");
				p.alpha = texture_file(a->string);
			}
	}

	MaterialHdl material(const std::string& name) {
		auto it = m_materialHdl.find(name);
		if(it != m_materialHdl.end()) return it->second;
		const JsonValue* m = m_materials->find(name);
		if(!m) r.fail("unknown material name '" + name + "' in association");
		PathSwap ps(r, { "materials", name });
		MaterialParams p;
		std::vector<std::unique_ptr<MaterialParams>> keep;
		material_params(*m, p, keep);
		MaterialHdl h = world_add_material(m_core, name.c_str(), &p);
		if(!h) core_fail("materials/" + name + ": failed to add the material");
		m_materialHdl[name] = h;
		return h;
	}

	// json_loader.cpp load_lights:537-745. Returns false for a light that
	// is ignored (unknown type or a goniometric light, as the reference does).
	bool light(const std::string& name, LightHdl& out) {
		auto it = m_lightHdl.find(name);
		if(it != m_lightHdl.end()) { out = it->second; return true; }
		if(m_lightIgnored.count(name)) return false;
		const JsonValue* l = m_lights->find(name);
		if(!l) {
			m_st.warn("unknown light source '" + name + "' will be ignored");
			m_lightIgnored[name] = true;
			return false;
		}
		PathSwap ps(r, { "lights", name });
		r.object(*l, "light");
		const std::string type = r.text(r.req(*l, "type"), "type");
		LightHdl h{};
		bool ok = true;
		if(type == "point") {
			std::vector<Vec3> pos = r.vec3_list(r.req(*l, "position"), "position");
			std::vector<float> scale = r.opt(*l, "scale") ? r.float_list(*r.opt(*l, "scale"), "scale") : std::vector<float>{ 1.0f };
			std::vector<Vec3> intensity;
			if(const JsonValue* v = r.opt(*l, "intensity")) intensity = r.vec3_list(*v, "intensity");
			else if(const JsonValue* f = r.opt(*l, "flux")) {
				intensity = r.vec3_list(*f, "flux");
				const float fourPi = 4.0f * PI_F;
				for(Vec3& c : intensity) { c.x /= fourPi; c.y /= fourPi; c.z /= fourPi; }
			} else if(r.opt(*l, "temperature")) r.fail("black-body 'temperature' is not supported; give 'intensity' or 'flux'");
			else r.fail("missing 'intensity'");
			const size_t n = std::max(pos.size(), std::max(intensity.size(), scale.size()));
			broadcast(pos, n); broadcast(intensity, n); broadcast(scale, n);
			if(pos.size() != intensity.size()) r.fail("mismatched light path size (intensities)");
			if(pos.size() != scale.size()) r.fail("mismatched light path size (scales)");
			h = world_add_light(m_core, name.c_str(), LIGHT_POINT, uint32_t(n));
			if(h.type != LIGHT_POINT) core_fail("lights/" + name + ": failed to add point light");
			for(uint32_t i = 0; i < uint32_t(n); ++i) {
				const Vec3 I{ intensity[i].x * scale[i], intensity[i].y * scale[i], intensity[i].z * scale[i] };
				if(!world_set_point_light_position(m_core, h, pos[i], i) || !world_set_point_light_intensity(m_core, h, I, i))
					core_fail("lights/" + name + ": failed to set the point light");
			}
		} else if(type == "envmap") {
			Vec3 colourScale{ 1.0f, 1.0f, 1.0f };
			if(const JsonValue* s = r.opt(*l, "scale")) {
				if(s->is_array()) colourScale = r.vec3(*s, "scale");
				else { const float f = r.num(*s, "scale"); colourScale = Vec3{ f, f, f }; }
			}
			if(r.opt(*l, "map")) {
				h = world_add_background_light(m_core, name.c_str(), BACKGROUND_ENVMAP);
				if(h.type != LIGHT_ENVMAP) core_fail("lights/" + name + ": failed to add the environment map");
			} else {
				h = world_add_background_light(m_core, name.c_str(), BACKGROUND_MONOCHROME);
				if(h.type != LIGHT_ENVMAP || !world_set_env_light_color(m_core, h, colourScale))
					core_fail("lights/" + name + ": failed to add the monochrome background");
			}
		} else if(type == "spot") {
			h = world_add_light(m_core, name.c_str(), LIGHT_SPOT, 1);
			if(h.type != LIGHT_SPOT) core_fail("lights/" + name + ": failed to add spot light");
		} else if(type == "directional") {
			h = world_add_light(m_core, name.c_str(), LIGHT_DIRECTIONAL, 1);
			if(h.type != LIGHT_DIRECTIONAL) core_fail("lights/" + name + ": failed to add directional light");
		} else if(type == "sky") {
			h = world_add_background_light(m_core, name.c_str(), BACKGROUND_SKY_HOSEK);
			if(h.type != LIGHT_ENVMAP) core_fail("lights/" + name + ": failed to add sky light");
		} else if(type == "goniometric") {
			m_st.warn("light '" + name + "': goniometric lights are not supported and will be ignored");
			ok = false;
		} else {
			m_st.warn("light '" + name + "' has unknown type '" + type + "' and will be ignored");
			ok = false;
		}
		if(!ok) { m_lightIgnored[name] = true; return false; }
		m_lightHdl[name] = h;
		out = h;
		return true;
	}

	// Child keys override the parent's; nested objects merge (json_loader.cpp:1011-1030).
	static void merge_into(const JsonValue& src, JsonValue& dst) {
		for(const auto& [k, v] : src.members) {
			JsonValue* d = dst.find(k);
			if(d && v.is_object() && d->is_object()) merge_into(v, *d);
			else dst.set(k, v);
		}
	}
	JsonValue resolve_scenario(const std::string& name, size_t depth) {
		if(depth == 0) r.fail("loop in scenario inheritance");
		const JsonValue* sc = m_scenarios->find(name);
		if(!sc) r.fail("failed to find parent scenario '" + name + "'");
		r.object(*sc, "scenario");
		if(const JsonValue* parent = r.opt(*sc, "parentScenario")) {
			JsonValue merged = resolve_scenario(r.text(*parent, "parentScenario"), depth - 1);
			merge_into(*sc, merged);
			return merged;
		}
		return *sc;
	}

	// json_loader.cpp load_scenarios:783-980
	void load_scenarios() {
		const std::vector<std::string>& binMats = m_st.binary->material_names();
		world_reserve_scenarios(m_core, uint32_t(m_scenarios->members.size()));
		for(const auto& entry : m_scenarios->members) {
			m_st.check_abort();
			const std::string& name = entry.first;
			Scope s0(r, "scenarios");
			Scope s1(r, name);
			const JsonValue sc = resolve_scenario(name, m_scenarios->members.size());
			const std::string camName = r.text(r.req(sc, "camera"), "camera");
			float res[2];
			r.numbers(r.req(sc, "resolution"), 2, res, "resolution");
			if(res[0] < 1.0f || res[1] < 1.0f || std::floor(res[0]) != res[0] || std::floor(res[1]) != res[1])
				r.fail("resolution: expected two positive integers");
			const uint32_t lod = r.opt(sc, "lod") ? r.uint(*r.opt(sc, "lod"), "lod") : 0u;
			CameraHdl cam = camera(camName);
			ScenarioHdl h = world_create_scenario(m_core, name.c_str());
			if(!h) core_fail("failed to create scenario '" + name + "'");
			if(!scenario_set_camera(m_core, h, cam)) core_fail("failed to set camera '" + camName + "'");
			if(!scenario_set_resolution(h, uint32_t(res[0]), uint32_t(res[1]))) core_fail("failed to set the resolution");
			if(!scenario_set_global_lod_level(h, lod)) core_fail("failed to set LoD " + std::to_string(lod));

			if(const JsonValue* lights = r.opt(sc, "lights")) {
				Scope s(r, "lights");
				if(!lights->is_array()) r.fail("expected an array of light names");
				for(const JsonValue& ln : lights->array) {
					const std::string lname = r.text(ln, "light name");
					LightHdl lh;
					if(light(lname, lh) && !scenario_add_light(m_core, h, lh)) core_fail("failed to add light '" + lname + "'");
				}
			}
			if(const JsonValue* objs = r.opt(sc, "objectProperties")) {
				Scope s(r, "objectProperties");
				r.object(*objs, "objectProperties");
				scenario_reserve_custom_object_properties(h, objs->members.size());
				for(const auto& [oname, props] : objs->members) {
					Scope so(r, oname);
					r.object(props, "object properties");
					ObjectHdl oh = world_get_object(m_core, oname.c_str());
					if(!oh) r.fail("failed to find object '" + oname + "'");
					if(const JsonValue* l = r.opt(props, "lod"))
						if(!scenario_set_object_lod(h, oh, r.uint(*l, "lod"))) core_fail("failed to set the LoD of object '" + oname + "'");
					if(const JsonValue* m = r.opt(props, "mask"); m && r.flag(*m, "mask"))
						if(!scenario_mask_object(h, oh)) core_fail("failed to mask object '" + oname + "'");
					if(r.opt(props, "tessellation"))
						m_st.warn(r.where() + ": tessellation settings are ignored");
				}
			}
			if(const JsonValue* insts = r.opt(sc, "instanceProperties")) {
				Scope s(r, "instanceProperties");
				r.object(*insts, "instanceProperties");
				scenario_reserve_custom_instance_properties(h, insts->members.size());
				for(const auto& [iname, props] : insts->members) {
					Scope si(r, iname);
					r.object(props, "instance properties");
					auto it = m_instanceNames.find(iname);
					if(it == m_instanceNames.end()) continue; // as the reference: names not in the binary are skipped
					if(const JsonValue* l = r.opt(props, "lod"))
						if(!scenario_set_instance_lod(h, it->second, r.uint(*l, "lod")))
							core_fail("failed to set the LoD of instance '" + iname + "'");
					if(const JsonValue* m = r.opt(props, "mask"); m && r.flag(*m, "mask"))
						if(!scenario_mask_instance(h, it->second)) core_fail("failed to mask instance '" + iname + "'");
				}
			}
			{
				Scope s(r, "materialAssignments");
				const JsonValue& assign = r.object(r.req(sc, "materialAssignments"), "materialAssignments");
				scenario_reserve_material_slots(h, binMats.size());
				for(size_t i = 0; i < binMats.size(); ++i) {
					const std::string mname = r.text(r.req(assign, binMats[i]), binMats[i]);
					const MatIdx slot = scenario_declare_material_slot(h, binMats[i].c_str(), binMats[i].size());
					if(slot != MatIdx(i)) core_fail("failed to declare material slot '" + binMats[i] + "'");
					if(!scenario_assign_material(h, slot, material(mname)))
						core_fail("failed to assign material '" + mname + "'");
				}
			}
			const char* msg = "";
			if(!world_finalize_scenario(m_core, h, &msg)) core_fail("scenario '" + name + "' did not pass the sanity check");
		}
	}
};

} // namespace

void load_scene_file(LoaderState& state, const std::string& jsonPath) {
	SceneFileLoader(state, fs::path(jsonPath)).load();
}

void load_object_lod(LoaderState& state, ObjectHdl obj, uint32_t level) {
	if(!state.binary || !state.binary->is_open()) throw LoaderError("no binary file is open");
	auto it = state.objectIds.find(obj);
	if(it == state.objectIds.end()) throw LoaderError("the object was not loaded from the open scene file");
	const MffObject& o = state.binary->objects()[it->second];
	if(level >= o.lodOffsets.size())
		throw LoaderError("object '" + o.name + "' has " + std::to_string(o.lodOffsets.size()) + " LoDs, not " + std::to_string(level + 1));
	MffLod L = state.binary->read_lod(it->second, level);
	const MffLodHeader& hd = L.header;
	LodHdl lod = object_add_lod(obj, level, false);
	if(!lod) core_fail("failed to add LoD " + std::to_string(level) + " of object '" + o.name + "'");
	if(!polygon_reserve(lod, hd.vertices, hd.triangles, hd.quads) || !spheres_reserve(lod, hd.spheres))
		core_fail("failed to reserve LoD memory of object '" + o.name + "'");
	auto bulk = [](const void* p) { BulkLoader b; b.type = BULK_ARRAY; b.descriptor.bytes = static_cast<const char*>(p); return b; };
	if(hd.vertices > 0) {
		const BulkLoader bp = bulk(L.positions.data()), bn = bulk(L.normals.data()), bu = bulk(L.uvs.data());
		size_t rp = 0, rn = 0, ru = 0;
		if(polygon_add_vertex_bulk(lod, hd.vertices, &bp, &bn, &bu, nullptr, &rp, &rn, &ru) == INVALID_INDEX
		   || rp != hd.vertices || rn != hd.vertices || ru != hd.vertices)
			core_fail("failed to add the vertices of object '" + o.name + "'");
	}
	if(hd.triangles > 0 && polygon_add_triangle_bulk(lod, hd.triangles, reinterpret_cast<const UVec3*>(L.triangles.data()),
	                                                 L.faceMaterials.data()) == INVALID_INDEX)
		core_fail("failed to add the triangles of object '" + o.name + "'");
	if(hd.quads > 0 && polygon_add_quad_bulk(lod, hd.quads, reinterpret_cast<const UVec4*>(L.quads.data()),
	                                         L.faceMaterials.data() + hd.triangles) == INVALID_INDEX)
		core_fail("failed to add the quads of object '" + o.name + "'");
	if(hd.spheres > 0) {
		const BulkLoader bs = bulk(L.spheres.data()), bm = bulk(L.sphereMaterials.data());
		size_t rs = 0;
		if(spheres_add_sphere_bulk(lod, hd.spheres, &bs, nullptr, &rs) == INVALID_INDEX || rs != hd.spheres
		   || spheres_set_material_idx_bulk(lod, 0, hd.spheres, &bm) != hd.spheres)
			core_fail("failed to add the spheres of object '" + o.name + "'");
	}
}

} // namespace mffl
