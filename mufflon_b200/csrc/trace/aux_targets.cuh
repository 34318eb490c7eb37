// The path tracer's auxiliary targets (pt_params.hpp:16-26), as
// pt_common.hpp:75-156 contributes them: at every vertex with path length
// >= the minimum, the guide weight times the vertex's position, incident
// distance ("Depth"), shading normal, uv, albedo (Lambert and Torrance; 0 for
// emitters and misses) and the mean of its MIS-weighted emission
// ("Lightness"); at every unoccluded next-event sample the guide weight times
// its cosine term (also "Lightness"). The guide weight is 1 / (1 + solid
// angle) of the camera path's footprint (pt_common.hpp:49-61,
// footprint.hpp:137-165: FootprintV0 with pChoice 1, every sampled direction
// adding 1 / sqrt(its pdf) to m_a, solid angle m_a^2).
#pragma once

#include "dmath.cuh"
#include "scene_types.hpp"

namespace mb {

// Channels of a pixel's iteration values: position 3, depth 1, normal 3,
// uv 2, albedo 3, lightness 1.
// (AUX_CHANNELS = 13, scene_types.hpp)
enum { AUX_POS = 0, AUX_DEPTH = 3, AUX_NORMAL = 4, AUX_UV = 7, AUX_ALBEDO = 9, AUX_LIGHT = 12 };
static_assert(AUX_LIGHT + 1 == AUX_CHANNELS, "auxiliary channel layout");
constexpr int AUX_TARGETS = 6;
// first channel and channel count of target a, in the order Position, Depth,
// Normal, UV, Albedo, Lightness
MBD int aux_first(int a) { return a == 0 ? AUX_POS : a == 1 ? AUX_DEPTH : a == 2 ? AUX_NORMAL : a == 3 ? AUX_UV : a == 4 ? AUX_ALBEDO : AUX_LIGHT; }
MBD int aux_count(int a) { return a == 0 || a == 2 || a == 4 ? 3 : a == 3 ? 2 : 1; }

// m_a after one more segment sampled with pdf `pdf`, and the guide weight
// of the vertex it reaches.
MBD float guide_after_segment(float& ma, float pdf) {
	ma = __fadd_rn(ma, __fdiv_rn(1.0f, sqrt_(pdf)));
	return __fdiv_rn(1.0f, __fadd_rn(1.0f, __fmul_rn(ma, ma)));
}
// the mean of three channels
MBD float avg3(f3 v) { return __fdiv_rn(__fadd_rn(__fadd_rn(v.x, v.y), v.z), 3.0f); }

// The contributions of one vertex; add(channel, value) accumulates (a NaN
// value counts as 0, render_target.hpp:64-75).
template < class Add >
MBD void aux_vertex(Add&& add, float gw, f3 position, float depth, f3 normal, f2 uv, f3 albedo, f3 emission) {
	add(AUX_POS, __fmul_rn(gw, position.x)); add(AUX_POS + 1, __fmul_rn(gw, position.y)); add(AUX_POS + 2, __fmul_rn(gw, position.z));
	add(AUX_DEPTH, __fmul_rn(gw, depth));
	add(AUX_NORMAL, __fmul_rn(gw, normal.x)); add(AUX_NORMAL + 1, __fmul_rn(gw, normal.y)); add(AUX_NORMAL + 2, __fmul_rn(gw, normal.z));
	add(AUX_UV, __fmul_rn(gw, uv.x)); add(AUX_UV + 1, __fmul_rn(gw, uv.y));
	add(AUX_ALBEDO, __fmul_rn(gw, albedo.x)); add(AUX_ALBEDO + 1, __fmul_rn(gw, albedo.y)); add(AUX_ALBEDO + 2, __fmul_rn(gw, albedo.z));
	add(AUX_LIGHT, __fmul_rn(gw, avg3(emission)));
}

} // namespace mb
