// Known answers from the reference's own integer code (test infrastructure).
//
// Compiled by `make -C oracle ref` against the reference's sources
// (src/core/math/rng.hpp, src/core/math/sfcurves.hpp, src/core/export/core_api.h)
// with the stand-in headers of oracle/refpin/stub, and run by
// tests/golden/make_ref_kat.py, which writes tests/golden/ref_rng_sfcurves_kat.json.
// The oracle's restatements are then checked against these values
// (tests/test_oracle_refpin.py), so the random streams, seeding and
// space-filling-curve codes are pinned to the reference itself:
//   * scramble_seed (SplitMix64, rng.hpp:12-17) and PCG64 seeding and output
//     (rng.hpp:70-93), including the per-pixel seeds pixel + seed * (W*H + 1)
//     of cpu_pt.cpp:40-45 at 1080p;
//   * GoldenRatio2D (rng.hpp:119-140), the light-flux sample sequence;
//   * part_by_two21 / part_by_two16 / part_by_two10, get_morton_code,
//     get_hilbert_code, gray_to_binary (sfcurves.hpp:12-77).
#include "core/math/rng.hpp"

#include <cstdio>
#include <vector>

using namespace mufflon;
using namespace mufflon::math;

static void list_u64(const char* name, const std::vector<u64>& v, bool last = false) {
	std::printf("  \"%s\": [", name);
	for(size_t i = 0; i < v.size(); ++i) std::printf("%s\"%llu\"", i ? ", " : "", (unsigned long long)v[i]);
	std::printf("]%s\n", last ? "" : ",");
}

int main() {
	const u32 seeds[] = { 0u, 1u, 2u, 7u, 42u, 123456u, 0x7fffffffu, 0x80000000u, 0xfffffffeu, 0xffffffffu,
	                      // cpu_pt.cpp:40-45 at 1920 x 1080: pixel + seed * (numPixels + 1), u32 arithmetic
	                      0u + 1u * (1920u * 1080u + 1u), 1919u + 3u * (1920u * 1080u + 1u),
	                      2073599u + 17u * (1920u * 1080u + 1u) };
	std::printf("{\n");
	std::vector<u64> v;
	for(u32 s : seeds) v.push_back(s);
	list_u64("seeds", v);
	v.clear();
	for(u32 s : seeds) v.push_back(scramble_seed(s));
	list_u64("scramble_seed", v);
	// first 8 outputs of PCG64(seed), seed-major
	v.clear();
	for(u32 s : seeds) { PCG64 r(s); for(int i = 0; i < 8; ++i) v.push_back(r.next()); }
	list_u64("pcg64_first8", v);
	// GoldenRatio2D(seed): first 8 outputs
	v.clear();
	for(u32 s : seeds) { GoldenRatio2D g(s); for(int i = 0; i < 8; ++i) v.push_back(g.next()); }
	list_u64("golden_ratio2d_first8", v);
	// Morton pieces
	const u32 xs21[] = { 0u, 1u, 2u, 3u, 5u, 0x155555u, 0xaaaaau, 0x100000u, 0x1fffffu, 1234567u, 0x0f0f0fu };
	v.clear();
	for(u32 x : xs21) v.push_back(x);
	list_u64("x21", v);
	v.clear();
	for(u32 x : xs21) v.push_back(part_by_two21(x));
	list_u64("part_by_two21", v);
	const u32 xs10[] = { 0u, 1u, 2u, 0x155u, 0x2aau, 0x200u, 0x3ffu, 777u };
	v.clear();
	for(u32 x : xs10) v.push_back(x);
	list_u64("x10", v);
	v.clear();
	for(u32 x : xs10) v.push_back(part_by_two10(x));
	list_u64("part_by_two10", v);
	const u16 tri[][3] = { { 0, 0, 0 }, { 1, 0, 0 }, { 0, 1, 0 }, { 0, 0, 1 }, { 0xffff, 0, 0 }, { 0x1234, 0xabcd, 0x0f0f },
	                       { 0xffff, 0xffff, 0xffff }, { 40000, 2, 65000 }, { 7, 300, 12345 } };
	v.clear();
	for(auto& t : tri) { v.push_back(t[0]); v.push_back(t[1]); v.push_back(t[2]); }
	list_u64("triples16", v);
	v.clear();
	for(auto& t : tri) v.push_back(part_by_two16(t[0]));
	list_u64("part_by_two16", v);
	v.clear();
	for(auto& t : tri) v.push_back(get_morton_code(t[0], t[1], t[2]));
	list_u64("morton_code", v);
	v.clear();
	for(auto& t : tri) v.push_back(get_hilbert_code(t[0], t[1], t[2]));
	list_u64("hilbert_code", v);
	v.clear();
	for(auto& t : tri) v.push_back(gray_to_binary(get_morton_code(t[0], t[1], t[2]) ^ 0x5a5a5a5a5a5aull));
	list_u64("gray_to_binary_of_morton_xor_5a", v, true);
	std::printf("}\n");
	return 0;
}
