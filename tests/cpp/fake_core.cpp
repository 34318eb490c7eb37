// A host-only stand-in for libmufflon_core.so's world-building C API, so the
// scene-file loader's control flow (including its error paths) can run on a
// CPU with sanitizers. It records what the loader builds, accepts the same
// models the CUDA path tracer does (Lambert, Torrance GGX/Smith, emissive;
// point lights and monochrome backgrounds; pinhole cameras) and rejects the
// others with an error, and world_load_scenario requests missing LoDs through
// the registered LoD loader with the core's LoD rule (instance over object
// over global level, clamped to the object's LoD slots).
//
// dump_world() prints the recorded world as JSON for the test to compare.
#include "../../include/mufflon_core.h"

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

namespace {

thread_local std::string s_err;

struct Lod {
	std::vector<float> v, n, uv, sph;
	std::vector<uint32_t> tri, quad;
	std::vector<uint16_t> triMat, quadMat, sphMat;
};
struct Object { std::string name; uint32_t id = 0, slots = 0; std::map<uint32_t, std::unique_ptr<Lod>> lods; };
struct Instance { Object* obj; uint32_t index, frame; float w2i[12] = { 1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0 }; };
struct Texture { uint32_t w = 1, h = 1, ch = 4; std::vector<float> t; };
struct Material { std::string name; int type; };
struct Camera { std::string name; float pos[3], dir[3], up[3], nearP, farP, fov; };
struct Light { std::string name; int kind; float a[3] = {}, b[3] = {}; };
struct Scenario {
	std::string name;
	uint32_t w = 0, h = 0, globalLod = 0;
	Camera* cam = nullptr;
	std::vector<int> lights;
	std::vector<std::string> slots;
	std::vector<Material*> mats;
	std::vector<uint32_t> maskedInst;
	std::vector<Object*> maskedObj;
	std::map<Object*, uint32_t> objLod;
	std::map<uint32_t, uint32_t> instLod;
};
struct World {
	std::vector<std::unique_ptr<Object>> objects;
	std::vector<std::unique_ptr<Instance>> instances;
	std::vector<std::unique_ptr<Texture>> textures;
	std::vector<std::unique_ptr<Material>> materials;
	std::vector<std::unique_ptr<Camera>> cameras;
	std::vector<Light> lights;
	std::vector<std::unique_ptr<Scenario>> scenarios;
	Scenario* current = nullptr;
	Boolean (*loadLod)(void*, ObjectHdl, uint32_t, Boolean) = nullptr;
	void* user = nullptr;
	std::vector<std::string> loadedScenarios;
};

struct Err : std::runtime_error { using std::runtime_error::runtime_error; };
#define TRY try {
#define CATCH(ret) } catch(const std::exception& e) { s_err = std::string(__func__) + ": " + e.what(); return ret; }
#define CHECK(c, m) do { if(!(c)) throw Err(m); } while(0)

World& W(void* h) { CHECK(h, "invalid instance"); return *static_cast<World*>(h); }
Lod& L(void* h) { CHECK(h, "invalid LoD"); return *static_cast<Lod*>(h); }

size_t bulk(const BulkLoader* b, void* dst, size_t bytes) {
	CHECK(b && b->type == BULK_ARRAY, "only array bulk streams");
	std::memcpy(dst, b->descriptor.bytes, bytes);
	return bytes;
}

uint32_t effective(const Scenario& s, const Instance& i) {
	uint32_t lvl = s.globalLod;
	if(auto it = s.instLod.find(i.index); it != s.instLod.end()) lvl = it->second;
	else if(auto jt = s.objLod.find(i.obj); jt != s.objLod.end()) lvl = jt->second;
	const uint32_t slots = i.obj->slots ? i.obj->slots : 1u;
	return std::min(lvl, slots - 1u);
}

} // namespace

extern "C" {

const char* core_get_dll_error(void) { return s_err.c_str(); }
MufflonInstanceHdl mufflon_initialize(void) { return new World(); }
void mufflon_destroy(MufflonInstanceHdl h) { delete static_cast<World*>(h); }

Boolean mufflon_set_lod_loader(MufflonInstanceHdl h, Boolean (*f)(void*, ObjectHdl, uint32_t, Boolean),
                               Boolean (*)(void*, uint32_t, uint16_t*, uint32_t*), Boolean (*)(void*, LodMetadata*, size_t*),
                               void* user) {
	TRY W(h).loadLod = f; W(h).user = user; return true; CATCH(false)
}

void world_clear_all(MufflonInstanceHdl h) {
	TRY World& w = W(h);
	auto f = w.loadLod; auto u = w.user;
	w = World();
	w.loadLod = f; w.user = u;
	CATCH()
}
Boolean world_finalize(MufflonInstanceHdl h, const Vec3, const Vec3, const char** msg) {
	TRY if(msg) *msg = ""; CHECK(!W(h).cameras.empty(), "world has no camera"); return true; CATCH(false)
}
void world_reserve_objects_instances(MufflonInstanceHdl, const uint32_t, const uint32_t) {}
ObjectHdl world_create_object(MufflonInstanceHdl h, const char* name, ObjectFlags) {
	TRY World& w = W(h);
	w.objects.push_back(std::make_unique<Object>());
	w.objects.back()->name = name; w.objects.back()->id = uint32_t(w.objects.size() - 1);
	return w.objects.back().get();
	CATCH(nullptr)
}
ObjectHdl world_get_object(MufflonInstanceHdl h, const char* name) {
	TRY for(auto& o : W(h).objects) if(o->name == name) return o.get(); throw Err("object not found"); CATCH(nullptr)
}
Boolean object_allocate_lod_slots(ObjectHdl o, LodLevel n) { TRY CHECK(o && n, "bad"); static_cast<Object*>(o)->slots = n; return true; CATCH(false) }
LodHdl object_add_lod(ObjectHdl o, LodLevel level, Boolean) {
	TRY Object& ob = *static_cast<Object*>(o);
	CHECK(!ob.slots || level < ob.slots, "LoD level beyond the object's LoD slots");
	auto& s = ob.lods[level]; if(!s) s = std::make_unique<Lod>(); return s.get();
	CATCH(nullptr)
}
InstanceHdl world_create_instance(MufflonInstanceHdl h, ObjectHdl o, const uint32_t frame) {
	TRY World& w = W(h); CHECK(o, "invalid object");
	w.instances.push_back(std::make_unique<Instance>(Instance{ static_cast<Object*>(o), uint32_t(w.instances.size()), frame }));
	return w.instances.back().get();
	CATCH(nullptr)
}
Boolean instance_set_transformation_matrix(MufflonInstanceHdl, InstanceHdl i, const Mat3x4* m, const Boolean w2i) {
	TRY CHECK(i && m, "bad"); CHECK(w2i, "the fake core takes world-to-instance matrices");
	std::memcpy(static_cast<Instance*>(i)->w2i, m->v, 48); return true; CATCH(false)
}
Boolean instance_get_transformation_matrix(MufflonInstanceHdl, InstanceHdl i, Mat3x4* m) {
	TRY CHECK(i && m, "bad"); std::memcpy(m->v, static_cast<Instance*>(i)->w2i, 48); return true; CATCH(false)
}

Boolean polygon_reserve(LodHdl l, size_t, size_t, size_t) { TRY (void)L(l); return true; CATCH(false) }
Boolean spheres_reserve(LodHdl l, size_t) { TRY (void)L(l); return true; CATCH(false) }
VertexHdl polygon_add_vertex_bulk(LodHdl l, size_t n, const BulkLoader* p, const BulkLoader* nn, const BulkLoader* uv,
                                  const AABB*, size_t* pr, size_t* nr, size_t* ur) {
	TRY Lod& d = L(l);
	d.v.resize(3 * n); d.n.resize(3 * n); d.uv.resize(2 * n);
	*pr = bulk(p, d.v.data(), 12 * n) / 12; *nr = bulk(nn, d.n.data(), 12 * n) / 12; *ur = bulk(uv, d.uv.data(), 8 * n) / 8;
	return 0;
	CATCH(INVALID_INDEX)
}
FaceHdl polygon_add_triangle_bulk(LodHdl l, size_t n, const UVec3* v, const MatIdx* m) {
	TRY Lod& d = L(l); const size_t nv = d.v.size() / 3;
	for(size_t i = 0; i < n; ++i) {
		CHECK(v[i].x < nv && v[i].y < nv && v[i].z < nv, "triangle index out of range");
		d.tri.insert(d.tri.end(), { v[i].x, v[i].y, v[i].z }); d.triMat.push_back(m[i]);
	}
	return 0;
	CATCH(INVALID_INDEX)
}
FaceHdl polygon_add_quad_bulk(LodHdl l, size_t n, const UVec4* v, const MatIdx* m) {
	TRY Lod& d = L(l); const size_t nv = d.v.size() / 3;
	for(size_t i = 0; i < n; ++i) {
		CHECK(v[i].x < nv && v[i].y < nv && v[i].z < nv && v[i].w < nv, "quad index out of range");
		d.quad.insert(d.quad.end(), { v[i].x, v[i].y, v[i].z, v[i].w }); d.quadMat.push_back(m[i]);
	}
	return 0;
	CATCH(INVALID_INDEX)
}
SphereHdl spheres_add_sphere_bulk(LodHdl l, size_t n, const BulkLoader* s, const AABB*, size_t* r) {
	TRY Lod& d = L(l); d.sph.resize(4 * n); *r = bulk(s, d.sph.data(), 16 * n) / 16; return 0; CATCH(INVALID_INDEX)
}
size_t spheres_set_material_idx_bulk(LodHdl l, SphereHdl, size_t n, const BulkLoader* s) {
	TRY Lod& d = L(l); d.sphMat.resize(n); return bulk(s, d.sphMat.data(), 2 * n) / 2; CATCH(size_t(-1))
}

TextureHdl world_add_texture_value(MufflonInstanceHdl h, const float* v, int n, TextureSampling) {
	TRY World& w = W(h); CHECK(v && n >= 1 && n <= 4, "texture value needs 1 to 4 channels");
	w.textures.push_back(std::make_unique<Texture>()); w.textures.back()->ch = uint32_t(n);
	w.textures.back()->t.assign(v, v + n); return w.textures.back().get();
	CATCH(nullptr)
}
TextureHdl world_add_texture_rgba32f(MufflonInstanceHdl h, const char*, uint32_t wd, uint32_t ht, const float* t, TextureSampling) {
	TRY World& w = W(h); CHECK(t && wd && ht, "invalid texture");
	w.textures.push_back(std::make_unique<Texture>()); Texture& x = *w.textures.back();
	x.w = wd; x.h = ht; x.t.assign(t, t + size_t(wd) * ht * 4); return &x;
	CATCH(nullptr)
}
MaterialHdl world_add_material(MufflonInstanceHdl h, const char* name, const MaterialParams* p) {
	TRY World& w = W(h); CHECK(p, "null");
	switch(p->innerType) {
		case MATERIAL_LAMBERT: CHECK(p->inner.lambert.albedo, "no albedo"); break;
		case MATERIAL_TORRANCE:
			CHECK(p->inner.torrance.ndf == NDF_GGX && p->inner.torrance.shadowingModel == SHADOWING_SMITH,
			      "the CUDA path tracer implements Torrance with GGX and Smith shadowing");
			CHECK(static_cast<Texture*>(p->inner.torrance.roughness)->w == 1, "constant roughness only");
			break;
		case MATERIAL_EMISSIVE: CHECK(static_cast<Texture*>(p->inner.emissive.radiance)->w == 1, "constant radiance only"); break;
		default: throw Err("material type not implemented by the CUDA path tracer");
	}
	w.materials.push_back(std::make_unique<Material>(Material{ name, int(p->innerType) }));
	return w.materials.back().get();
	CATCH(nullptr)
}
CameraHdl world_add_pinhole_camera(MufflonInstanceHdl h, const char* name, const Vec3* p, const Vec3* d, const Vec3* u,
                                   const uint32_t n, float nearP, float farP, float fov) {
	TRY World& w = W(h); CHECK(p && d && u && n >= 1, "invalid camera");
	w.cameras.push_back(std::make_unique<Camera>(Camera{ name, { p->x, p->y, p->z }, { d->x, d->y, d->z },
	                                                     { u->x, u->y, u->z }, nearP, farP, fov }));
	return w.cameras.back().get();
	CATCH(nullptr)
}
LightHdl world_add_light(MufflonInstanceHdl h, const char* name, LightType t, const uint32_t) {
	LightHdl bad; bad.type = 7; bad.index = 0;
	TRY World& w = W(h); CHECK(t == LIGHT_POINT, "the CUDA path tracer implements point, area and environment lights");
	w.lights.push_back(Light{ name, 0 }); LightHdl r; r.type = LIGHT_POINT; r.index = uint32_t(w.lights.size() - 1); return r;
	CATCH(bad)
}
LightHdl world_add_background_light(MufflonInstanceHdl h, const char* name, BackgroundType t) {
	LightHdl bad; bad.type = 7; bad.index = 0;
	TRY World& w = W(h); CHECK(t == BACKGROUND_MONOCHROME, "the CUDA path tracer implements monochrome backgrounds");
	w.lights.push_back(Light{ name, 1 }); LightHdl r; r.type = LIGHT_ENVMAP; r.index = uint32_t(w.lights.size() - 1); return r;
	CATCH(bad)
}
Boolean world_set_point_light_position(MufflonInstanceHdl h, LightHdl l, Vec3 p, const uint32_t f) {
	TRY if(f == 0) { Light& x = W(h).lights.at(l.index); x.a[0] = p.x; x.a[1] = p.y; x.a[2] = p.z; } return true; CATCH(false)
}
Boolean world_set_point_light_intensity(MufflonInstanceHdl h, LightHdl l, Vec3 p, const uint32_t f) {
	TRY if(f == 0) { Light& x = W(h).lights.at(l.index); x.b[0] = p.x; x.b[1] = p.y; x.b[2] = p.z; } return true; CATCH(false)
}
Boolean world_set_env_light_color(MufflonInstanceHdl h, LightHdl l, Vec3 c) {
	TRY Light& x = W(h).lights.at(l.index); x.a[0] = c.x; x.a[1] = c.y; x.a[2] = c.z; return true; CATCH(false)
}

void world_reserve_scenarios(MufflonInstanceHdl, const uint32_t) {}
ScenarioHdl world_create_scenario(MufflonInstanceHdl h, const char* name) {
	TRY World& w = W(h); w.scenarios.push_back(std::make_unique<Scenario>()); w.scenarios.back()->name = name;
	return w.scenarios.back().get(); CATCH(nullptr)
}
ScenarioHdl world_find_scenario(MufflonInstanceHdl h, const char* name) {
	TRY for(auto& s : W(h).scenarios) if(s->name == name) return s.get(); throw Err("scenario not found"); CATCH(nullptr)
}
Boolean scenario_set_camera(MufflonInstanceHdl, ScenarioHdl s, CameraHdl c) {
	TRY CHECK(s && c, "bad"); static_cast<Scenario*>(s)->cam = static_cast<Camera*>(c); return true; CATCH(false)
}
Boolean scenario_set_resolution(ScenarioHdl s, uint32_t w, uint32_t h) {
	TRY CHECK(w && h, "resolution out of range"); static_cast<Scenario*>(s)->w = w; static_cast<Scenario*>(s)->h = h; return true; CATCH(false)
}
Boolean scenario_set_global_lod_level(ScenarioHdl s, LodLevel l) { TRY static_cast<Scenario*>(s)->globalLod = l; return true; CATCH(false) }
Boolean scenario_add_light(MufflonInstanceHdl, ScenarioHdl s, LightHdl l) {
	TRY CHECK(l.type == LIGHT_POINT || l.type == LIGHT_ENVMAP, "bad light"); static_cast<Scenario*>(s)->lights.push_back(int(l.index));
	return true; CATCH(false)
}
void scenario_reserve_custom_object_properties(ScenarioHdl, size_t) {}
void scenario_reserve_custom_instance_properties(ScenarioHdl, size_t) {}
void scenario_reserve_material_slots(ScenarioHdl, size_t) {}
Boolean scenario_set_object_lod(ScenarioHdl s, ObjectHdl o, LodLevel l) {
	TRY static_cast<Scenario*>(s)->objLod[static_cast<Object*>(o)] = l; return true; CATCH(false)
}
Boolean scenario_set_instance_lod(ScenarioHdl s, InstanceHdl i, LodLevel l) {
	TRY static_cast<Scenario*>(s)->instLod[static_cast<Instance*>(i)->index] = l; return true; CATCH(false)
}
Boolean scenario_mask_object(ScenarioHdl s, ObjectHdl o) { TRY static_cast<Scenario*>(s)->maskedObj.push_back(static_cast<Object*>(o)); return true; CATCH(false) }
Boolean scenario_mask_instance(ScenarioHdl s, InstanceHdl i) {
	TRY static_cast<Scenario*>(s)->maskedInst.push_back(static_cast<Instance*>(i)->index); return true; CATCH(false)
}
MatIdx scenario_declare_material_slot(ScenarioHdl s, const char* name, size_t len) {
	TRY Scenario& sc = *static_cast<Scenario*>(s); sc.slots.emplace_back(name, len); sc.mats.push_back(nullptr);
	return MatIdx(sc.slots.size() - 1); CATCH(MatIdx(0xFFFF))
}
Boolean scenario_assign_material(ScenarioHdl s, MatIdx i, MaterialHdl m) {
	TRY Scenario& sc = *static_cast<Scenario*>(s); CHECK(m && i < sc.mats.size(), "bad slot");
	sc.mats[i] = static_cast<Material*>(m); return true; CATCH(false)
}
Boolean world_finalize_scenario(MufflonInstanceHdl, ScenarioHdl s, const char** msg) {
	TRY if(msg) *msg = ""; CHECK(static_cast<Scenario*>(s)->cam, "scenario has no camera"); return true; CATCH(false)
}
SceneHdl world_load_scenario(MufflonInstanceHdl h, ScenarioHdl s) {
	TRY World& w = W(h); CHECK(s, "invalid scenario");
	Scenario& sc = *static_cast<Scenario*>(s);
	w.current = &sc;
	for(auto& i : w.instances) {
		if(i->frame != 0xFFFFFFFFu && i->frame != 0) continue;
		if(std::count(sc.maskedInst.begin(), sc.maskedInst.end(), i->index)) continue;
		if(std::count(sc.maskedObj.begin(), sc.maskedObj.end(), i->obj)) continue;
		const uint32_t lvl = effective(sc, *i);
		if(i->obj->lods.count(lvl)) continue;
		CHECK(w.loadLod, "no LoD loader");
		CHECK(w.loadLod(w.user, i->obj, lvl, false), "the LoD loader failed");
		CHECK(i->obj->lods.count(lvl), "the LoD loader did not add the LoD");
	}
	w.loadedScenarios.push_back(sc.name);
	return &sc;
	CATCH(nullptr)
}

// JSON summary of the recorded world (floats as IEEE bit patterns).
const char* fake_core_dump(MufflonInstanceHdl h) {
	static std::string out;
	World& w = W(h);
	std::ostringstream os;
	auto bits = [](float f) { uint32_t u; std::memcpy(&u, &f, 4); return u; };
	auto fl = [&](const float* p, size_t n) { os << '['; for(size_t i = 0; i < n; ++i) os << (i ? "," : "") << bits(p[i]); os << ']'; };
	os << "{\"objects\":[";
	for(size_t o = 0; o < w.objects.size(); ++o) {
		const Object& ob = *w.objects[o];
		os << (o ? "," : "") << "{\"name\":\"" << ob.name << "\",\"slots\":" << ob.slots << ",\"lods\":{";
		bool first = true;
		for(const auto& [lvl, l] : ob.lods) {
			os << (first ? "" : ",") << '"' << lvl << "\":{\"v\":";
			first = false;
			fl(l->v.data(), l->v.size());
			os << ",\"n\":"; fl(l->n.data(), l->n.size());
			os << ",\"tri\":" << l->tri.size() / 3 << ",\"quad\":" << l->quad.size() / 4 << ",\"sph\":" << l->sph.size() / 4 << '}';
		}
		os << "}}";
	}
	os << "],\"instances\":[";
	for(size_t i = 0; i < w.instances.size(); ++i) {
		os << (i ? "," : "") << "{\"object\":" << w.instances[i]->obj->id << ",\"frame\":" << w.instances[i]->frame << ",\"w2i\":";
		fl(w.instances[i]->w2i, 12);
		os << '}';
	}
	os << "],\"materials\":[";
	for(size_t i = 0; i < w.materials.size(); ++i) os << (i ? "," : "") << "[\"" << w.materials[i]->name << "\"," << w.materials[i]->type << ']';
	os << "],\"lights\":[";
	for(size_t i = 0; i < w.lights.size(); ++i) {
		os << (i ? "," : "") << "{\"name\":\"" << w.lights[i].name << "\",\"kind\":" << w.lights[i].kind << ",\"a\":";
		fl(w.lights[i].a, 3); os << ",\"b\":"; fl(w.lights[i].b, 3); os << '}';
	}
	os << "],\"cameras\":[";
	for(size_t i = 0; i < w.cameras.size(); ++i) {
		const Camera& c = *w.cameras[i];
		os << (i ? "," : "") << "{\"name\":\"" << c.name << "\",\"fov\":" << bits(c.fov) << ",\"near\":" << bits(c.nearP)
		   << ",\"far\":" << bits(c.farP) << ",\"pos\":";
		fl(c.pos, 3); os << '}';
	}
	os << "],\"scenarios\":[";
	for(size_t i = 0; i < w.scenarios.size(); ++i) {
		const Scenario& s = *w.scenarios[i];
		os << (i ? "," : "") << "{\"name\":\"" << s.name << "\",\"res\":[" << s.w << ',' << s.h << "],\"lod\":" << s.globalLod
		   << ",\"camera\":\"" << (s.cam ? s.cam->name : "") << "\",\"lights\":[";
		for(size_t k = 0; k < s.lights.size(); ++k) os << (k ? "," : "") << s.lights[k];
		os << "],\"slots\":[";
		for(size_t k = 0; k < s.slots.size(); ++k) os << (k ? "," : "") << "[\"" << s.slots[k] << "\",\"" << (s.mats[k] ? s.mats[k]->name : "") << "\"]";
		os << "],\"maskedInstances\":[";
		for(size_t k = 0; k < s.maskedInst.size(); ++k) os << (k ? "," : "") << s.maskedInst[k];
		os << "],\"maskedObjects\":[";
		for(size_t k = 0; k < s.maskedObj.size(); ++k) os << (k ? "," : "") << s.maskedObj[k]->id;
		os << "],\"objectLods\":{";
		bool first = true;
		for(const auto& [o, l] : s.objLod) { os << (first ? "" : ",") << '"' << o->id << "\":" << l; first = false; }
		os << "},\"instanceLods\":{";
		first = true;
		for(const auto& [i2, l] : s.instLod) { os << (first ? "" : ",") << '"' << i2 << "\":" << l; first = false; }
		os << "}}";
	}
	os << "],\"loaded\":[";
	for(size_t i = 0; i < w.loadedScenarios.size(); ++i) os << (i ? "," : "") << '"' << w.loadedScenarios[i] << '"';
	os << "]}";
	out = os.str();
	return out.c_str();
}

} // extern "C"
