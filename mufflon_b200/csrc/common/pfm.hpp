// Portable float map (PFM) texture reading, shared by the core's
// world_add_texture and the scene-file loader. Follows the reference's PFM
// texture plugin (src/pfmloader/interface.cpp:74-160): "PF" is RGB, stored as
// RGBA with alpha 0 (FORMAT_RGBA32F); "Pf" is one channel (FORMAT_R32F), kept
// here in the first of four channels; rows as stored; a positive scale means
// big-endian data.
#pragma once

#include <cctype>
#include <cstdint>
#include <cstring>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

namespace mb {

struct PfmImage {
	uint32_t width = 0, height = 0, channels = 0; // channels: 1 ("Pf") or 3 ("PF")
	std::vector<float> rgba;                      // width * height * 4
};

// Parses the bytes of a PFM file; throws std::runtime_error with a message.
inline PfmImage parse_pfm(const std::string& data) {
	size_t pos = 0;
	auto fail = [](const std::string& m) { throw std::runtime_error(m); };
	auto skip_ws = [&]() { while(pos < data.size() && std::isspace(static_cast<unsigned char>(data[pos]))) ++pos; };
	auto token = [&]() {
		skip_ws();
		const size_t s = pos;
		while(pos < data.size() && !std::isspace(static_cast<unsigned char>(data[pos]))) ++pos;
		return data.substr(s, pos - s);
	};
	if(data.size() < 2) fail("not a PFM file");
	const std::string bands = data.substr(0, 2);
	if(bands != "PF" && bands != "Pf") fail("unknown PFM bands '" + bands + "' (expected \"PF\" or \"Pf\")");
	pos = 2;
	long long wi = 0, hi = 0;
	double scale = 0.0;
	try {
		wi = std::stoll(token());
		hi = std::stoll(token());
		scale = std::stod(token());
	} catch(const std::logic_error&) { fail("malformed PFM header"); }
	if(wi <= 0 || hi <= 0 || wi > 65536 || hi > 65536) fail("invalid PFM size");
	if(pos < data.size() && data[pos] == '\r') ++pos;
	if(pos >= data.size() || data[pos] != '\n') fail("expected a newline after the PFM header");
	++pos;
	PfmImage img;
	img.channels = bands == "PF" ? 3u : 1u;
	const size_t texels = size_t(wi) * size_t(hi);
	if(data.size() - pos < texels * img.channels * 4u) fail("PFM data shorter than its header says");
	const bool swap = scale > 0.0; // big-endian data on a little-endian host
	img.rgba.assign(texels * 4u, 0.0f);
	for(size_t i = 0; i < texels; ++i) {
		for(uint32_t c = 0; c < img.channels; ++c) {
			unsigned char b[4];
			std::memcpy(b, data.data() + pos + (img.channels * i + c) * 4, 4);
			if(swap) { std::swap(b[0], b[3]); std::swap(b[1], b[2]); }
			std::memcpy(&img.rgba[4 * i + c], b, 4);
		}
	}
	img.width = uint32_t(wi);
	img.height = uint32_t(hi);
	return img;
}

} // namespace mb
