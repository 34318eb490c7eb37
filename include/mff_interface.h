/*
 * C ABI of the scene-file loader (libmufflon_loader.so): imports Mufflon's
 * JSON scene description plus its binary geometry file (*.mff) into a core
 * instance through the world-building C API, and supplies object LoDs when
 * the core asks for them.
 *
 * Names, types and return conventions are those of
 * src/mffloader/interface/mff_interface.h:16-40, so examples/example.c and
 * the Python binding (bindings.py:313-317, 346-347) link unchanged. Failing
 * calls return LOADER_ERROR / false / NULL and leave a message for
 * loader_get_dll_error().
 *
 * Not provided: loader_save_scene (scene export) and the loader_profiling_*
 * family (the reference's CPU profiler).
 */
#ifndef MUFFLON_B200_MFF_INTERFACE_H
#define MUFFLON_B200_MFF_INTERFACE_H

#include "mufflon_core.h"

#ifdef __cplusplus
extern "C" {
#endif

#define LOADER_API __attribute__((visibility("default")))

typedef void* MufflonLoaderInstanceHdl;

/* mff_interface.h:14-18 */
typedef enum {
	LOADER_SUCCESS,
	LOADER_ERROR,
	LOADER_ABORT
} LoaderStatus;

/* mff_interface.h:20: message of the last failed call on this thread (the
 * returned string stays valid until the next failing call on the thread). */
LOADER_API const char* CDECL loader_get_dll_error(void);
/* mff_interface.h:21-22. Destroy a loader before the core instance it was
 * created for: destroying it unregisters its LoD loader from that instance. */
LOADER_API MufflonLoaderInstanceHdl CDECL loader_initialize(MufflonInstanceHdl instHdl);
LOADER_API void CDECL loader_destroy(MufflonLoaderInstanceHdl hdl);
/* mff_interface.h:23: clears the world, loads the file and its default
 * scenario (interface.cpp:137-171). LOADER_ABORT after loader_abort(). */
LOADER_API LoaderStatus CDECL loader_load_json(MufflonLoaderInstanceHdl hdl, const char* path);
/* mff_interface.h:25: adds LoD `lod` of `obj` from the loaded binary file;
 * registered with the core through mufflon_set_lod_loader. */
LOADER_API Boolean CDECL loader_load_lod(MufflonLoaderInstanceHdl hdl, ObjectHdl obj, uint32_t lod, Boolean asReduced);
/* mff_interface.h:26-27: the object's sorted unique material indices (file
 * version >= 1.7; *readIndices = 0 for older files). indexBuffer must hold
 * as many entries as the file lists. */
LOADER_API Boolean CDECL loader_load_object_material_indices(MufflonLoaderInstanceHdl hdl, const uint32_t objId,
                                                             uint16_t* indexBuffer, uint32_t* readIndices);
/* mff_interface.h:28: one LodMetadata per LoD of every object, objects in
 * file order; data must hold that many entries. */
LOADER_API Boolean CDECL loader_load_lod_metadatas(MufflonLoaderInstanceHdl hdl, LodMetadata* data, size_t* read);
/* mff_interface.h:29-30: request that a running loader_load_json stops;
 * its status text while it runs. */
LOADER_API Boolean CDECL loader_abort(MufflonLoaderInstanceHdl hdl);
LOADER_API const char* CDECL loader_get_loading_status(MufflonLoaderInstanceHdl hdl);

/* EXTENSION: warnings of the last load, one per line (parts of a file that
 * are ignored, such as goniometric lights or tessellation settings). */
LOADER_API const char* CDECL loader_get_warnings(MufflonLoaderInstanceHdl hdl);

#ifdef __cplusplus
}
#endif

#endif
