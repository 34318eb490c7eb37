// C API of the scene-file loader (src/mffloader/interface/interface.cpp).
// No exception crosses the ABI: failures store a message for
// loader_get_dll_error() and return LOADER_ERROR / false / nullptr.
#include "../../../include/mff_interface.h"
#include "scene_loader.hpp"

#include <filesystem>
#include <string>

using namespace mffl;

namespace {

thread_local std::string s_lastError;

struct MufflonLoaderInstance {
	LoaderState state;
};

MufflonLoaderInstance& linst(MufflonLoaderInstanceHdl h) {
	if(!h) throw LoaderError("invalid loader instance handle (null)");
	return *static_cast<MufflonLoaderInstance*>(h);
}

#define TRY try {
#define CATCH_ALL(ret) } catch(const std::exception& ex) { s_lastError = std::string(__func__) + ": " + ex.what(); return ret; } \
	catch(...) { s_lastError = std::string(__func__) + ": unknown error"; return ret; }

Boolean cb_load_lod(void* user, ObjectHdl obj, uint32_t lod, Boolean asReduced) {
	return loader_load_lod(user, obj, lod, asReduced);
}
Boolean cb_material_indices(void* user, uint32_t objId, uint16_t* buffer, uint32_t* read) {
	return loader_load_object_material_indices(user, objId, buffer, read);
}
Boolean cb_metadata(void* user, LodMetadata* data, size_t* read) {
	return loader_load_lod_metadatas(user, data, read);
}

} // namespace

extern "C" {

const char* loader_get_dll_error(void) { return s_lastError.c_str(); }

MufflonLoaderInstanceHdl loader_initialize(MufflonInstanceHdl instHdl) {
	TRY
	if(!instHdl) throw LoaderError("invalid mufflon instance handle (null)");
	auto* l = new MufflonLoaderInstance();
	l->state.core = instHdl;
	return l;
	CATCH_ALL(nullptr)
}

void loader_destroy(MufflonLoaderInstanceHdl hdl) {
	TRY
	if(!hdl) return;
	auto* l = static_cast<MufflonLoaderInstance*>(hdl);
	if(l->state.binary) mufflon_set_lod_loader(l->state.core, nullptr, nullptr, nullptr, nullptr);
	delete l;
	CATCH_ALL()
}

LoaderStatus loader_load_json(MufflonLoaderInstanceHdl hdl, const char* path) {
	TRY
	MufflonLoaderInstance& L = linst(hdl);
	if(!path) throw LoaderError("invalid path (null)");
	namespace fs = std::filesystem;
	const fs::path file = fs::u8path(path);
	if(!fs::exists(file)) throw LoaderError("file '" + file.string() + "' does not exist");
	if(fs::is_directory(file)) throw LoaderError("path '" + file.string() + "' is a directory, not a file");
	LoaderState& st = L.state;
	st.abortRequested = false;
	st.loading = true;
	{
		std::lock_guard<std::mutex> lock(st.statusMutex);
		st.warnings.clear();
		st.status = "Starting";
	}
	if(file.extension() != ".json") st.warn("scene file does not end with '.json'; parsing it anyway");
	st.binary.reset();
	st.objectIds.clear();
	LoaderStatus result = LOADER_SUCCESS;
	try {
		world_clear_all(st.core);
		if(!mufflon_set_lod_loader(st.core, cb_load_lod, cb_material_indices, cb_metadata, hdl))
			throw LoaderError(std::string("cannot register the LoD loader: ") + core_get_dll_error());
		load_scene_file(st, file.string());
	} catch(const LoaderAbort&) {
		result = LOADER_ABORT;
		s_lastError = "loader_load_json: loading aborted";
	} catch(const std::exception& ex) {
		result = LOADER_ERROR;
		s_lastError = std::string("loader_load_json: ") + ex.what();
	}
	st.loading = false;
	if(result != LOADER_SUCCESS) {
		// leave nothing behind that could call back into a half-loaded file
		mufflon_set_lod_loader(st.core, nullptr, nullptr, nullptr, nullptr);
		st.binary.reset();
		st.objectIds.clear();
	}
	return result;
	CATCH_ALL(LOADER_ERROR)
}

Boolean loader_load_lod(MufflonLoaderInstanceHdl hdl, ObjectHdl obj, uint32_t lod, Boolean) {
	TRY
	MufflonLoaderInstance& L = linst(hdl);
	if(!obj) throw LoaderError("invalid object handle (null)");
	try {
		load_object_lod(L.state, obj, lod);
	} catch(const std::exception& ex) {
		L.state.lodError = ex.what(); // for the message of the load that asked for it
		throw;
	}
	return true;
	CATCH_ALL(false)
}

Boolean loader_load_object_material_indices(MufflonLoaderInstanceHdl hdl, const uint32_t objId, uint16_t* indexBuffer,
                                            uint32_t* readIndices) {
	TRY
	MufflonLoaderInstance& L = linst(hdl);
	if(!indexBuffer) throw LoaderError("invalid material index buffer (null)");
	if(L.state.version < UNIQUE_MATERIALS_VERSION) {
		if(readIndices) *readIndices = 0;
		return true;
	}
	if(!L.state.binary) throw LoaderError("no scene file is loaded");
	const std::vector<uint16_t> idx = L.state.binary->read_unique_materials(objId);
	for(size_t i = 0; i < idx.size(); ++i) indexBuffer[i] = idx[i];
	if(readIndices) *readIndices = uint32_t(idx.size());
	return true;
	CATCH_ALL(false)
}

Boolean loader_load_lod_metadatas(MufflonLoaderInstanceHdl hdl, LodMetadata* data, size_t* read) {
	TRY
	MufflonLoaderInstance& L = linst(hdl);
	if(!data) throw LoaderError("invalid LoD metadata buffer (null)");
	if(!L.state.binary) throw LoaderError("no scene file is loaded");
	const MffFile& B = *L.state.binary;
	size_t k = 0;
	for(uint32_t o = 0; o < B.objects().size(); ++o)
		for(uint32_t lvl = 0; lvl < B.objects()[o].lodOffsets.size(); ++lvl) {
			const MffLodHeader h = B.read_lod_header(o, lvl);
			data[k++] = LodMetadata{ h.vertices, h.triangles, h.quads, h.edges, h.spheres };
		}
	if(read) *read = k;
	return true;
	CATCH_ALL(false)
}

Boolean loader_abort(MufflonLoaderInstanceHdl hdl) {
	TRY
	MufflonLoaderInstance& L = linst(hdl);
	if(!L.state.loading.load()) throw LoaderError("no load is running that could be aborted");
	L.state.abortRequested = true;
	return true;
	CATCH_ALL(false)
}

const char* loader_get_loading_status(MufflonLoaderInstanceHdl hdl) {
	TRY
	MufflonLoaderInstance& L = linst(hdl);
	std::lock_guard<std::mutex> lock(L.state.statusMutex);
	L.state.statusCopy = L.state.loading.load() ? L.state.status : std::string();
	return L.state.statusCopy.c_str();
	CATCH_ALL(nullptr)
}

const char* loader_get_warnings(MufflonLoaderInstanceHdl hdl) {
	TRY
	MufflonLoaderInstance& L = linst(hdl);
	std::lock_guard<std::mutex> lock(L.state.statusMutex);
	L.state.warningsCopy.clear();
	for(const auto& w : L.state.warnings) { L.state.warningsCopy += w; L.state.warningsCopy += '\n'; }
	return L.state.warningsCopy.c_str();
	CATCH_ALL(nullptr)
}

} // extern "C"
