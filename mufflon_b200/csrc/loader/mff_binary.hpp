// Reader of Mufflon's binary geometry file (*.mff): material names, objects
// with their LoD jump tables, instances, and the geometry of one LoD on
// request. The layout is the one of doc/FileFormat.md ("The binary file")
// as src/mffloader/parsing/binary.cpp reads it:
//
//   'Mats' u64:next u32:M M*<string>
//   ['Bone' u64:next u32:B u32:K K*B*8*f32]
//   'Objs' u64:instances u32:flags u32:N N*u64  (flags: 1 deflate, 2 packed normals)
//     N * ('Obj_' <string> u32:flags u32:keyframe u32:prevObj 6*f32:aabb
//          u32:D D*u64 [u32:U U*u16 (file version >= 1.7)] D*<LoD>)
//   'Inst' u32:I I*(<string> u32:obj u32:keyframe u32:prevInst 12*f32)
//
// Every read is bounds-checked against the file size, so a truncated or
// corrupt file ends in an MffError instead of a huge allocation or a read
// past the end. Counts are little-endian as on x86_64.
#pragma once

#include <cstdint>
#include <cstdio>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

namespace mffl {

struct MffError : std::runtime_error { using std::runtime_error::runtime_error; };

constexpr uint32_t fourcc(char a, char b, char c, char d) {
	return uint32_t(uint8_t(a)) | (uint32_t(uint8_t(b)) << 8) | (uint32_t(uint8_t(c)) << 16) | (uint32_t(uint8_t(d)) << 24);
}
constexpr uint32_t MAGIC_MATERIALS = fourcc('M', 'a', 't', 's');
constexpr uint32_t MAGIC_BONES = fourcc('B', 'o', 'n', 'e');
constexpr uint32_t MAGIC_OBJECTS = fourcc('O', 'b', 'j', 's');
constexpr uint32_t MAGIC_OBJECT = fourcc('O', 'b', 'j', '_');
constexpr uint32_t MAGIC_LOD = fourcc('L', 'O', 'D', '_');
constexpr uint32_t MAGIC_ATTRIBUTE = fourcc('A', 't', 't', 'r');
constexpr uint32_t MAGIC_INSTANCES = fourcc('I', 'n', 's', 't');

constexpr uint32_t MFF_DEFLATE = 1u;
constexpr uint32_t MFF_COMPRESSED_NORMALS = 2u;
constexpr uint32_t MFF_NO_FRAME = 0xFFFFFFFFu;

struct MffObject {
	std::string name;
	uint32_t flags = 0, keyframe = MFF_NO_FRAME, prevAnimObject = MFF_NO_FRAME;
	float aabbMin[3] = {}, aabbMax[3] = {};
	uint64_t offset = 0;                 // of the 'Obj_' tag
	uint64_t afterJumpTable = 0;         // where the unique material list of version 1.7 starts
	std::vector<uint64_t> lodOffsets;    // absolute offsets of the 'LOD_' tags
};

struct MffInstance {
	std::string name;
	uint32_t objectId = 0, keyframe = MFF_NO_FRAME, prevAnimInstance = MFF_NO_FRAME;
	float transform[12] = {};
};

struct MffLodHeader {
	uint32_t triangles = 0, quads = 0, spheres = 0, vertices = 0, edges = 0;
	uint32_t vertexAttributes = 0, faceAttributes = 0, sphereAttributes = 0;
};

struct MffLod {
	MffLodHeader header;
	std::vector<float> positions, normals, uvs; // 3, 3, 2 per vertex
	std::vector<uint32_t> triangles, quads;     // 3, 4 per face
	std::vector<uint16_t> faceMaterials;        // triangles first, then quads
	std::vector<float> spheres;                 // centre xyz, radius
	std::vector<uint16_t> sphereMaterials;
};

// Octahedral decoding of a packed normal (doc/FileFormat.md, "Normal
// Compression", unpackNormal32), normalised.
void unpack_normal32(uint32_t packed, float out[3]);

class MffFile {
public:
	MffFile() = default;
	~MffFile();
	MffFile(const MffFile&) = delete;
	MffFile& operator=(const MffFile&) = delete;

	// Opens the file and reads everything but the LoD contents.
	void open(const std::string& path);
	void close();
	bool is_open() const { return m_file != nullptr; }
	const std::string& path() const { return m_path; }

	const std::vector<std::string>& material_names() const { return m_materials; }
	const std::vector<MffObject>& objects() const { return m_objects; }
	const std::vector<MffInstance>& instances() const { return m_instances; }
	uint32_t global_flags() const { return m_flags; }
	uint32_t bone_count() const { return m_bones; }
	uint32_t bone_frames() const { return m_boneFrames; }

	MffLodHeader read_lod_header(uint32_t objectId, uint32_t level) const;
	// Geometry of LoD `level` (must be < the object's LoD count).
	MffLod read_lod(uint32_t objectId, uint32_t level) const;
	// Sorted unique material indices of an object (file version >= 1.7).
	std::vector<uint16_t> read_unique_materials(uint32_t objectId) const;

private:
	std::FILE* m_file = nullptr;
	std::string m_path;
	uint64_t m_size = 0;
	uint32_t m_flags = 0;
	uint32_t m_bones = 0, m_boneFrames = 0;
	std::vector<std::string> m_materials;
	std::vector<MffObject> m_objects;
	std::vector<MffInstance> m_instances;

	friend class MffCursor;
};

} // namespace mffl
