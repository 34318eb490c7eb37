/* TextureCallback functions (core_interface.h:237-239) for the texture-file
 * tests: ctypes cannot define callbacks that return a struct by value, so the
 * tests load these from a small shared library. */
#include <stdint.h>
#include "mufflon_core.h"

static uint32_t g_calls = 0;
static uint32_t g_formats = 0;   /* bit per TextureFormat seen */
static uint32_t g_layers = 0;    /* bit per layer seen */
static uint64_t g_xy_sum = 0;    /* sum of x + 65536 * y over the calls */
static float g_last[64][4];      /* the first 64 values as seen, in call order */

/* Scales red by 0.5 and green by 0.25, keeps blue, sets alpha to 1. */
Vec4 halve_red_quarter_green(uint32_t x, uint32_t y, uint32_t layer, TextureFormat format, Vec4 value, void* user) {
	(void)user;
	if(g_calls < 64) { g_last[g_calls][0] = value.x; g_last[g_calls][1] = value.y; g_last[g_calls][2] = value.z; g_last[g_calls][3] = value.w; }
	++g_calls;
	g_formats |= 1u << (uint32_t)format;
	g_layers |= 1u << layer;
	g_xy_sum += (uint64_t)x + 65536ull * (uint64_t)y;
	Vec4 out = { value.x * 0.5f, value.y * 0.25f, value.z, 1.0f };
	return out;
}

/* Returns the value unchanged, recording the call. */
Vec4 record_only(uint32_t x, uint32_t y, uint32_t layer, TextureFormat format, Vec4 value, void* user) {
	(void)user;
	if(g_calls < 64) { g_last[g_calls][0] = value.x; g_last[g_calls][1] = value.y; g_last[g_calls][2] = value.z; g_last[g_calls][3] = value.w; }
	++g_calls;
	g_formats |= 1u << (uint32_t)format;
	g_layers |= 1u << layer;
	g_xy_sum += (uint64_t)x + 65536ull * (uint64_t)y;
	return value;
}

void callbacks_reset(void) { g_calls = 0; g_formats = 0; g_layers = 0; g_xy_sum = 0; }
uint32_t callbacks_calls(void) { return g_calls; }
uint32_t callbacks_formats(void) { return g_formats; }
uint32_t callbacks_layers(void) { return g_layers; }
uint64_t callbacks_xy_sum(void) { return g_xy_sum; }
const float* callbacks_values(void) { return &g_last[0][0]; }
