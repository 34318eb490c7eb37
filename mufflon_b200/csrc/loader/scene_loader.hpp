// Scene-file import: a JSON scene description (cameras, lights, materials,
// scenarios) plus its binary geometry file, fed into the core through the
// world-building C API, as src/mffloader/parsing/json_loader.cpp does.
#pragma once

#include "../../../include/mufflon_core.h"
#include "json.hpp"
#include "mff_binary.hpp"

#include <atomic>
#include <map>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

namespace mffl {

struct LoaderError : std::runtime_error { using std::runtime_error::runtime_error; };
struct LoaderAbort : std::runtime_error { LoaderAbort() : std::runtime_error("loading aborted") {} };

struct FileVersion {
	unsigned major = 1, minor = 7;
	bool operator<(const FileVersion& o) const { return major != o.major ? major < o.major : minor < o.minor; }
	bool operator>=(const FileVersion& o) const { return !(*this < o); }
};
constexpr FileVersion CURRENT_VERSION{ 1, 7 };
constexpr FileVersion WORLD_TO_INSTANCE_VERSION{ 1, 4 };   // instance matrices map world to instance
constexpr FileVersion ABSOLUTE_NEAR_FAR_VERSION{ 1, 5 };   // camera planes default to 0.01 / 500
constexpr FileVersion UNIQUE_MATERIALS_VERSION{ 1, 7 };    // objects list their material indices

// State shared between a load and the LoD requests the core makes later.
struct LoaderState {
	MufflonInstanceHdl core = nullptr;
	std::atomic<bool> abortRequested{ false };
	std::atomic<bool> loading{ false };
	std::mutex statusMutex;
	std::string status;
	std::string statusCopy;                 // what loader_get_loading_status hands out
	std::vector<std::string> warnings;
	std::string warningsCopy;
	FileVersion version{};
	std::unique_ptr<MffFile> binary;        // kept open for LoDs requested later
	std::map<const void*, uint32_t> objectIds; // core object handle -> binary object index
	std::string lodError;                   // why the last LoD request from the core failed

	void set_status(const std::string& s) { std::lock_guard<std::mutex> l(statusMutex); status = s; }
	void warn(const std::string& w) { std::lock_guard<std::mutex> l(statusMutex); warnings.push_back(w); }
	void check_abort() const { if(abortRequested.load()) throw LoaderAbort(); }
};

// Loads `jsonPath` into the (cleared) world of `state.core` and loads its
// default scenario. Throws LoaderError / JsonError / MffError / LoaderAbort.
void load_scene_file(LoaderState& state, const std::string& jsonPath);

// Adds LoD `level` of core object `obj` from the open binary file.
void load_object_lod(LoaderState& state, ObjectHdl obj, uint32_t level);

} // namespace mffl
