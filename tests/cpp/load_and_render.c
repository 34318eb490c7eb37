/* The flow of examples/example.c (load a scene file, enable a renderer by
 * name, iterate, save a screenshot) against the B200 libraries, with the
 * renderer's device set to DEVICE_CUDA: the CUDA path tracer is the only
 * variation this core registers.
 *
 *   load_and_render <renderer> <target> <scene.json> <iterations> <out.pfm>
 */
#include "core_interface.h"
#include "mff_interface.h"

#include <stdbool.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define CHECK_ERROR(expr)                                            \
	if(!(expr)) {                                                    \
		fprintf(stderr, "Expression failed: '%s' (%s)\n", #expr,     \
		        core_get_dll_error());                               \
		return EXIT_FAILURE;                                         \
	}

static bool enable_renderer(MufflonInstanceHdl inst, const char* name, RenderDevice device) {
	const uint32_t count = render_get_renderer_count(inst);
	for(uint32_t i = 0; i < count; ++i) {
		const char* full = render_get_renderer_name(inst, i);
		const char* shortName = render_get_renderer_short_name(inst, i);
		if(strcmp(name, full) == 0 || strcmp(name, shortName) == 0) {
			const uint32_t variations = render_get_renderer_variations(inst, i);
			for(uint32_t v = 0; v < variations; ++v)
				if(device == render_get_renderer_devices(inst, i, v))
					return render_enable_renderer(inst, i, v);
		}
	}
	return false;
}

int main(int argc, const char* argv[]) {
	if(argc < 6) {
		printf("Usage: %s renderer rendertarget scenefile iterations output.pfm\n", argv[0]);
		return EXIT_FAILURE;
	}
	const long iterations = strtol(argv[4], NULL, 10);
	MufflonInstanceHdl inst;
	CHECK_ERROR(inst = mufflon_initialize());
	MufflonLoaderInstanceHdl loader;
	CHECK_ERROR(loader = loader_initialize(inst));
	if(loader_load_json(loader, argv[3]) != LOADER_SUCCESS) {
		fprintf(stderr, "Failed to load scene file '%s': %s\n", argv[3], loader_get_dll_error());
		return EXIT_FAILURE;
	}
	if(!enable_renderer(inst, argv[1], DEVICE_CUDA)) {
		fprintf(stderr, "Could not find renderer with the name '%s'\n", argv[1]);
		return EXIT_FAILURE;
	}
	CHECK_ERROR(render_enable_render_target(inst, argv[2], false));
	for(long i = 0; i < iterations; ++i)
		CHECK_ERROR(render_iterate(inst, NULL, NULL, NULL));
	CHECK_ERROR(render_save_screenshot(inst, argv[5], argv[2], false));
	loader_destroy(loader);
	mufflon_destroy(inst);
	return EXIT_SUCCESS;
}
