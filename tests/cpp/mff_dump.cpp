// Test driver for the scene-file readers of libmufflon_loader.so, built from
// the same sources without the CUDA core so that CPU tests can check them:
//
//   mff_dump json <file>      the parsed JSON document, re-serialised
//   mff_dump mff <file>       everything the binary reader returns, floats as
//                             their IEEE bit patterns (exact comparison)
//   mff_dump unpack <u32>...  decoded packed normals as bit patterns
//
// Errors print "ERROR: <message>" and exit with status 2.
#include "../../mufflon_b200/csrc/loader/json.hpp"
#include "../../mufflon_b200/csrc/loader/mff_binary.hpp"

#include <cstdio>
#include <cstring>
#include <fstream>
#include <iostream>
#include <sstream>
#include <string>

using namespace mffl;

namespace {

std::string quote(const std::string& s) {
	std::string o = "\"";
	for(unsigned char c : s) {
		if(c == '"' || c == '\\') { o += '\\'; o += char(c); }
		else if(c < 0x20) { char b[8]; std::snprintf(b, sizeof(b), "\\u%04x", c); o += b; }
		else o += char(c);
	}
	return o + "\"";
}

void emit(const JsonValue& v, std::ostream& os) {
	switch(v.type) {
		case JsonValue::NUL: os << "null"; break;
		case JsonValue::BOOL: os << (v.boolean ? "true" : "false"); break;
		case JsonValue::NUMBER: { char b[40]; std::snprintf(b, sizeof(b), "%.17g", v.number); os << b; break; }
		case JsonValue::STRING: os << quote(v.string); break;
		case JsonValue::ARRAY:
			os << '[';
			for(size_t i = 0; i < v.array.size(); ++i) { if(i) os << ','; emit(v.array[i], os); }
			os << ']';
			break;
		case JsonValue::OBJECT:
			os << '{';
			for(size_t i = 0; i < v.members.size(); ++i) {
				if(i) os << ',';
				os << quote(v.members[i].first) << ':';
				emit(v.members[i].second, os);
			}
			os << '}';
			break;
	}
}

uint32_t bits(float f) { uint32_t u; std::memcpy(&u, &f, 4); return u; }

template < class T > void list(std::ostream& os, const std::vector<T>& v) {
	os << '[';
	for(size_t i = 0; i < v.size(); ++i) { if(i) os << ','; os << uint64_t(v[i]); }
	os << ']';
}
void flist(std::ostream& os, const float* p, size_t n) {
	os << '[';
	for(size_t i = 0; i < n; ++i) { if(i) os << ','; os << bits(p[i]); }
	os << ']';
}

void dump_mff(const std::string& path) {
	MffFile f;
	f.open(path);
	std::ostringstream os;
	os << "{\"materials\":[";
	for(size_t i = 0; i < f.material_names().size(); ++i) { if(i) os << ','; os << quote(f.material_names()[i]); }
	os << "],\"flags\":" << f.global_flags() << ",\"bones\":[" << f.bone_count() << ',' << f.bone_frames() << "],\"objects\":[";
	for(uint32_t o = 0; o < f.objects().size(); ++o) {
		const MffObject& obj = f.objects()[o];
		if(o) os << ',';
		os << "{\"name\":" << quote(obj.name) << ",\"flags\":" << obj.flags << ",\"keyframe\":" << obj.keyframe
		   << ",\"aabb\":";
		float box[6] = { obj.aabbMin[0], obj.aabbMin[1], obj.aabbMin[2], obj.aabbMax[0], obj.aabbMax[1], obj.aabbMax[2] };
		flist(os, box, 6);
		os << ",\"unique\":";
		list(os, f.read_unique_materials(o));
		os << ",\"lods\":[";
		for(uint32_t l = 0; l < obj.lodOffsets.size(); ++l) {
			const MffLod L = f.read_lod(o, l);
			if(l) os << ',';
			const MffLodHeader& h = L.header;
			os << "{\"header\":[" << h.triangles << ',' << h.quads << ',' << h.spheres << ',' << h.vertices << ','
			   << h.edges << ',' << h.vertexAttributes << ',' << h.faceAttributes << ',' << h.sphereAttributes << ']';
			os << ",\"positions\":"; flist(os, L.positions.data(), L.positions.size());
			os << ",\"normals\":"; flist(os, L.normals.data(), L.normals.size());
			os << ",\"uvs\":"; flist(os, L.uvs.data(), L.uvs.size());
			os << ",\"triangles\":"; list(os, L.triangles);
			os << ",\"quads\":"; list(os, L.quads);
			os << ",\"faceMaterials\":"; list(os, L.faceMaterials);
			os << ",\"spheres\":"; flist(os, L.spheres.data(), L.spheres.size());
			os << ",\"sphereMaterials\":"; list(os, L.sphereMaterials);
			os << '}';
		}
		os << "]}";
	}
	os << "],\"instances\":[";
	for(size_t i = 0; i < f.instances().size(); ++i) {
		const MffInstance& in = f.instances()[i];
		if(i) os << ',';
		os << "{\"name\":" << quote(in.name) << ",\"object\":" << in.objectId << ",\"keyframe\":" << in.keyframe
		   << ",\"transform\":";
		flist(os, in.transform, 12);
		os << '}';
	}
	os << "]}";
	std::cout << os.str() << std::endl;
}

} // namespace

int main(int argc, char** argv) {
	if(argc < 3) { std::fprintf(stderr, "usage: mff_dump json|mff|unpack ...\n"); return 1; }
	try {
		const std::string mode = argv[1];
		if(mode == "json") {
			std::ifstream in(argv[2], std::ios::binary);
			std::stringstream ss;
			ss << in.rdbuf();
			emit(parse_json(ss.str()), std::cout);
			std::cout << std::endl;
		} else if(mode == "mff") {
			dump_mff(argv[2]);
		} else if(mode == "unpack") {
			std::cout << '[';
			for(int i = 2; i < argc; ++i) {
				float n[3];
				unpack_normal32(uint32_t(std::stoul(argv[i])), n);
				if(i > 2) std::cout << ',';
				std::cout << '[' << bits(n[0]) << ',' << bits(n[1]) << ',' << bits(n[2]) << ']';
			}
			std::cout << ']' << std::endl;
		} else {
			std::fprintf(stderr, "unknown mode '%s'\n", mode.c_str());
			return 1;
		}
	} catch(const std::exception& e) {
		std::cout << "ERROR: " << e.what() << std::endl;
		return 2;
	}
	return 0;
}
