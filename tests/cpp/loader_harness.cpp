// Runs the scene-file loader against the host-only fake core
// (tests/cpp/fake_core.cpp) and prints, as one JSON line, the load status,
// the loader's error and warnings, and the recorded world. With a second
// argument, that scenario is loaded afterwards (on-demand LoDs).
//
//   loader_harness <scene.json> [scenario]
#include "../../include/mff_interface.h"

#include <cstdio>
#include <string>

extern "C" const char* fake_core_dump(MufflonInstanceHdl h);

namespace {
std::string quote(const char* s) {
	std::string o = "\"";
	for(const char* p = s ? s : ""; *p; ++p) {
		const unsigned char c = static_cast<unsigned char>(*p);
		if(c == '"' || c == '\\') { o += '\\'; o += char(c); }
		else if(c < 0x20) { char b[8]; std::snprintf(b, sizeof(b), "\\u%04x", c); o += b; }
		else o += char(c);
	}
	return o + "\"";
}
} // namespace

int main(int argc, char** argv) {
	if(argc < 2) return 1;
	MufflonInstanceHdl core = mufflon_initialize();
	MufflonLoaderInstanceHdl loader = loader_initialize(core);
	const LoaderStatus st = loader_load_json(loader, argv[1]);
	std::string error = st == LOADER_SUCCESS ? "" : loader_get_dll_error();
	bool switched = false;
	if(st == LOADER_SUCCESS && argc > 2) {
		ScenarioHdl s = world_find_scenario(core, argv[2]);
		switched = s && world_load_scenario(core, s);
		if(!switched) error = core_get_dll_error();
	}
	std::printf("{\"status\":%d,\"error\":%s,\"warnings\":%s,\"switched\":%s,\"abortIdle\":%u,\"world\":%s}\n", int(st),
	            quote(error.c_str()).c_str(), quote(loader_get_warnings(loader)).c_str(), switched ? "true" : "false",
	            unsigned(loader_abort(loader)), fake_core_dump(core));
	loader_destroy(loader);
	mufflon_destroy(core);
	return 0;
}
