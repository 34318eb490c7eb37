#include "mff_binary.hpp"

#include <cmath>
#include <cstring>
#include <sys/stat.h>
#include <unistd.h>
#include <zlib.h>

namespace mffl {

void unpack_normal32(uint32_t packed, float out[3]) {
	const float u = float(int16_t(uint16_t(packed & 0xFFFFu))) / 32767.0f;
	const float v = float(int16_t(uint16_t(packed >> 16))) / 32767.0f;
	const float z = 1.0f - std::fabs(u) - std::fabs(v);
	float x = u, y = v;
	if(z < 0.0f) {
		x = (1.0f - std::fabs(v)) * (u >= 0.0f ? 1.0f : -1.0f);
		y = (1.0f - std::fabs(u)) * (v >= 0.0f ? 1.0f : -1.0f);
	}
	const float len = std::sqrt(x * x + y * y + z * z);
	out[0] = x / len;
	out[1] = y / len;
	out[2] = z / len;
}

// Sequential, bounds-checked reads at an absolute file position.
class MffCursor {
public:
	MffCursor(const MffFile& f, uint64_t pos) : m_f(f), m_pos(pos) {}

	uint64_t pos() const { return m_pos; }
	void seek(uint64_t pos) {
		if(pos > m_f.m_size) fail("offset " + std::to_string(pos) + " beyond the end of the file");
		m_pos = pos;
	}
	void skip(uint64_t bytes) {
		if(bytes > m_f.m_size - m_pos) fail("section runs past the end of the file");
		m_pos += bytes;
	}
	uint64_t remaining() const { return m_f.m_size - m_pos; }

	void bytes(void* dst, uint64_t n) {
		if(n > remaining()) fail("section runs past the end of the file");
		if(n == 0) return;
		unsigned char* d = static_cast<unsigned char*>(dst);
		uint64_t done = 0;
		while(done < n) {
			const ssize_t r = pread(fileno(m_f.m_file), d + done, size_t(n - done), off_t(m_pos + done));
			if(r <= 0) fail("read error");
			done += uint64_t(r);
		}
		m_pos += n;
	}
	template < class T > T get() { T v; bytes(&v, sizeof(T)); return v; }
	uint32_t u32() { return get<uint32_t>(); }
	uint64_t u64() { return get<uint64_t>(); }
	std::string str() {
		const uint32_t n = u32();
		if(n > remaining()) fail("string runs past the end of the file");
		std::string s(n, '\0');
		bytes(s.data(), n);
		return s;
	}
	void expect(uint32_t magic, const std::string& what) {
		const uint64_t at = m_pos;
		if(u32() != magic) {
			m_pos = at;
			fail("invalid " + what + " magic constant");
		}
	}
	// Reads `count` elements of `elemBytes` into `out`, checking the size first.
	template < class T > void array(std::vector<T>& out, uint64_t count, uint64_t perElem = 1) {
		const uint64_t n = count * perElem;
		if(count != 0 && (n / count != perElem || n > remaining() / sizeof(T))) fail("array runs past the end of the file");
		out.resize(size_t(n));
		bytes(out.data(), n * sizeof(T));
	}
	// One DEFLATE block (u32 compressed size, u32 decompressed size, zlib
	// stream) whose decompressed size must be exactly `expected` bytes.
	std::vector<unsigned char> inflate(uint64_t expected, const std::string& what) {
		const uint32_t packed = u32();
		const uint32_t unpacked = u32();
		if(unpacked != expected)
			fail(what + ": the compressed block holds " + std::to_string(unpacked) + " bytes, expected " + std::to_string(expected));
		// DEFLATE expands at most ~1032:1; a larger claim is a corrupt header
		if(uint64_t(unpacked) > uint64_t(packed) * 1100u + 1024u) fail(what + ": implausible compression ratio");
		std::vector<unsigned char> in(packed);
		bytes(in.data(), packed);
		std::vector<unsigned char> out(unpacked);
		uLongf outLen = uLongf(unpacked);
		const int rc = uncompress(out.data(), &outLen, in.data(), uLong(packed));
		if(rc != Z_OK) fail(what + ": failed to inflate (zlib error " + std::to_string(rc) + ")");
		if(outLen != uLongf(unpacked)) fail(what + ": decompressed size mismatch");
		return out;
	}
	void skip_block() {
		const uint32_t packed = u32();
		(void)u32();
		skip(packed);
	}
	// Uncompressed attribute list: 'Attr' then per attribute name, meta,
	// flags, type, u64 byte count and the bytes (binary.cpp:245-335).
	void skip_attributes(uint32_t count) {
		expect(MAGIC_ATTRIBUTE, "attribute");
		for(uint32_t i = 0; i < count; ++i) {
			(void)str();
			(void)str();
			(void)u32();
			(void)u32();
			skip(u64());
		}
	}

	[[noreturn]] void fail(const std::string& what) const {
		throw MffError("binary file '" + m_f.m_path + "': " + what + " (at byte " + std::to_string(m_pos) + ")");
	}

private:
	const MffFile& m_f;
	uint64_t m_pos;
};

MffFile::~MffFile() { close(); }

void MffFile::close() {
	if(m_file) std::fclose(m_file);
	m_file = nullptr;
}

void MffFile::open(const std::string& path) {
	close();
	m_path = path;
	m_materials.clear();
	m_objects.clear();
	m_instances.clear();
	m_file = std::fopen(path.c_str(), "rb");
	if(!m_file) throw MffError("cannot open binary file '" + path + "'");
	struct stat st;
	if(fstat(fileno(m_file), &st) != 0) throw MffError("cannot stat binary file '" + path + "'");
	m_size = uint64_t(st.st_size);

	MffCursor c(*this, 0);
	c.expect(MAGIC_MATERIALS, "materials header");
	const uint64_t next = c.u64();
	const uint32_t numMaterials = c.u32();
	if(numMaterials > 0xFFFFu) c.fail("more materials than 16-bit indices address");
	for(uint32_t i = 0; i < numMaterials; ++i) m_materials.push_back(c.str());
	c.seek(next);

	uint32_t magic = c.u32();
	if(magic == MAGIC_BONES) {
		const uint64_t objStart = c.u64();
		m_bones = c.u32();
		m_boneFrames = c.u32();
		c.seek(objStart);
		magic = c.u32();
	}
	if(magic != MAGIC_OBJECTS) c.fail("invalid objects header magic constant");
	const uint64_t instStart = c.u64();
	m_flags = c.u32();
	const uint32_t numObjects = c.u32();
	if(uint64_t(numObjects) * 8u > c.remaining()) c.fail("object jump table runs past the end of the file");
	std::vector<uint64_t> jump(numObjects);
	c.bytes(jump.data(), uint64_t(numObjects) * 8u);
	m_objects.resize(numObjects);
	for(uint32_t i = 0; i < numObjects; ++i) {
		MffObject& o = m_objects[i];
		MffCursor oc(*this, 0);
		oc.seek(jump[i]);
		o.offset = jump[i];
		oc.expect(MAGIC_OBJECT, "object");
		o.name = oc.str();
		o.flags = oc.u32();
		o.keyframe = oc.u32();
		o.prevAnimObject = oc.u32();
		oc.bytes(o.aabbMin, sizeof(o.aabbMin));
		oc.bytes(o.aabbMax, sizeof(o.aabbMax));
		const uint32_t numLods = oc.u32();
		if(numLods == 0) oc.fail("object '" + o.name + "' has no LoD");
		if(uint64_t(numLods) * 8u > oc.remaining()) oc.fail("LoD jump table runs past the end of the file");
		o.lodOffsets.resize(numLods);
		oc.bytes(o.lodOffsets.data(), uint64_t(numLods) * 8u);
		o.afterJumpTable = oc.pos();
	}

	c.seek(instStart);
	c.expect(MAGIC_INSTANCES, "instance");
	const uint32_t numInstances = c.u32();
	// each instance takes at least 64 bytes: a guard before reserving
	if(uint64_t(numInstances) * 64u > c.remaining()) c.fail("instance list runs past the end of the file");
	m_instances.resize(numInstances);
	for(uint32_t i = 0; i < numInstances; ++i) {
		MffInstance& in = m_instances[i];
		in.name = c.str();
		in.objectId = c.u32();
		in.keyframe = c.u32();
		in.prevAnimInstance = c.u32();
		c.bytes(in.transform, sizeof(in.transform));
		if(in.objectId >= numObjects)
			c.fail("instance '" + in.name + "' names object " + std::to_string(in.objectId) + " of " + std::to_string(numObjects));
	}
}

MffLodHeader MffFile::read_lod_header(uint32_t objectId, uint32_t level) const {
	if(!m_file) throw MffError("binary file is not open");
	if(objectId >= m_objects.size()) throw MffError("object index out of range");
	const MffObject& o = m_objects[objectId];
	if(level >= o.lodOffsets.size()) throw MffError("LoD index out of range for object '" + o.name + "'");
	MffCursor c(*this, 0);
	c.seek(o.lodOffsets[level]);
	c.expect(MAGIC_LOD, "LoD");
	MffLodHeader h;
	h.triangles = c.u32(); h.quads = c.u32(); h.spheres = c.u32(); h.vertices = c.u32(); h.edges = c.u32();
	h.vertexAttributes = c.u32(); h.faceAttributes = c.u32(); h.sphereAttributes = c.u32();
	return h;
}

namespace {
template < class T >
void take(std::vector<T>& dst, const unsigned char* src, size_t count) {
	dst.resize(count);
	if(count) std::memcpy(dst.data(), src, count * sizeof(T));
}
} // namespace

// Section order of a LoD (binary.cpp read_lod:672-743): vertex data, vertex
// attributes, triangles, quads, face materials, face attributes, spheres
// with their materials and attributes. A section of zero elements is absent.
MffLod MffFile::read_lod(uint32_t objectId, uint32_t level) const {
	MffLod L;
	L.header = read_lod_header(objectId, level);
	const MffLodHeader& h = L.header;
	MffCursor c(*this, m_objects[objectId].lodOffsets[level] + 36u);
	const bool packedNormals = (m_flags & MFF_COMPRESSED_NORMALS) != 0;
	const uint64_t V = h.vertices, T = h.triangles, Q = h.quads, S = h.spheres, F = T + Q;
	std::vector<uint32_t> packed;
	if(m_flags & MFF_DEFLATE) {
		if(V > 0) {
			const uint64_t nb = packedNormals ? 4u : 12u;
			const auto blk = c.inflate(V * (12u + nb + 8u), "vertex data");
			take(L.positions, blk.data(), size_t(V * 3));
			if(packedNormals) take(packed, blk.data() + V * 12u, size_t(V));
			else take(L.normals, blk.data() + V * 12u, size_t(V * 3));
			take(L.uvs, blk.data() + V * (12u + nb), size_t(V * 2));
			if(h.vertexAttributes > 0) { c.expect(MAGIC_ATTRIBUTE, "attribute"); c.skip_block(); }
		}
		if(T > 0) { const auto b = c.inflate(T * 12u, "triangles"); take(L.triangles, b.data(), size_t(T * 3)); }
		if(Q > 0) { const auto b = c.inflate(Q * 16u, "quads"); take(L.quads, b.data(), size_t(Q * 4)); }
		if(F > 0) {
			const auto b = c.inflate(F * 2u, "face materials");
			take(L.faceMaterials, b.data(), size_t(F));
			if(h.faceAttributes > 0) { c.expect(MAGIC_ATTRIBUTE, "attribute"); c.skip_block(); }
		}
		if(S > 0) {
			const auto b = c.inflate(S * 18u, "spheres");
			take(L.spheres, b.data(), size_t(S * 4));
			take(L.sphereMaterials, b.data() + S * 16u, size_t(S));
			if(h.sphereAttributes > 0) { c.expect(MAGIC_ATTRIBUTE, "attribute"); c.skip_block(); }
		}
	} else {
		if(V > 0) {
			c.array(L.positions, V, 3);
			if(packedNormals) c.array(packed, V);
			else c.array(L.normals, V, 3);
			c.array(L.uvs, V, 2);
			if(h.vertexAttributes > 0) c.skip_attributes(h.vertexAttributes);
		}
		c.array(L.triangles, T, 3);
		c.array(L.quads, Q, 4);
		if(F > 0) {
			c.array(L.faceMaterials, F);
			if(h.faceAttributes > 0) c.skip_attributes(h.faceAttributes);
		}
		if(S > 0) {
			c.array(L.spheres, S, 4);
			c.array(L.sphereMaterials, S);
			if(h.sphereAttributes > 0) c.skip_attributes(h.sphereAttributes);
		}
	}
	if(packedNormals) {
		L.normals.resize(size_t(V * 3));
		for(size_t i = 0; i < packed.size(); ++i) unpack_normal32(packed[i], &L.normals[3 * i]);
	}
	const size_t numMats = m_materials.size();
	for(uint16_t m : L.faceMaterials)
		if(m >= numMats) c.fail("face material index " + std::to_string(m) + " of object '" + m_objects[objectId].name
		                        + "' exceeds the " + std::to_string(numMats) + " materials of the file");
	for(uint16_t m : L.sphereMaterials)
		if(m >= numMats) c.fail("sphere material index " + std::to_string(m) + " of object '" + m_objects[objectId].name
		                        + "' exceeds the " + std::to_string(numMats) + " materials of the file");
	return L;
}

std::vector<uint16_t> MffFile::read_unique_materials(uint32_t objectId) const {
	if(!m_file) throw MffError("binary file is not open");
	if(objectId >= m_objects.size()) throw MffError("object index out of range");
	MffCursor c(*this, m_objects[objectId].afterJumpTable);
	const uint32_t n = c.u32();
	std::vector<uint16_t> out;
	c.array(out, n);
	return out;
}

} // namespace mffl
