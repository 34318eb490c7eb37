"""Python binding of libmufflon_core.so (ctypes), mirroring Mufflon's
src/pythonbinding/bindings.py: ``DllInterface`` wraps the C API one call per
method (same method names), ``RenderActions`` is the convenience layer
(enable a renderer by name, iterate, read targets). ``load_scene_spec`` builds
a procedural :class:`mufflon_b200.scenes.SceneSpec` through the same C API
calls that Mufflon's scene loader issues.

There is no CPU fallback: constructing a ``DllInterface`` without the built
library or without a CUDA device raises.
"""
from __future__ import annotations

import ctypes
import os
from ctypes import (POINTER, Structure, Union, byref, c_bool, c_char_p, c_float, c_int, c_int32, c_size_t,
                    c_uint8, c_uint16, c_uint32, c_uint64, c_ulonglong, c_void_p)
from enum import IntEnum

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_LIB = os.path.join(_HERE, "lib", "libmufflon_core.so")
LOADER_LIB_NAME = "libmufflon_loader.so"


class ProcessTime(Structure):
    _fields_ = [("cycles", c_ulonglong), ("microseconds", c_ulonglong)]


class Vec2(Structure):
    _fields_ = [("u", c_float), ("v", c_float)]


class Vec3(Structure):
    _fields_ = [("x", c_float), ("y", c_float), ("z", c_float)]


class UVec3(Structure):
    _fields_ = [("x", c_uint32), ("y", c_uint32), ("z", c_uint32)]


class Vec4(Structure):
    _fields_ = [("x", c_float), ("y", c_float), ("z", c_float), ("w", c_float)]


class IVec2(Structure):
    _fields_ = [("x", c_int32), ("y", c_int32)]


# Vec4 (*TextureCallback)(x, y, layer, TextureFormat, Vec4 value, void* userParams), core_interface.h:237-239
TextureCallback = ctypes.CFUNCTYPE(Vec4, c_uint32, c_uint32, c_uint32, c_int, Vec4, c_void_p)


class UVec4(Structure):
    _fields_ = [("x", c_uint32), ("y", c_uint32), ("z", c_uint32), ("w", c_uint32)]


class Mat3x4(Structure):
    _fields_ = [("v", c_float * 12)]


class AABB(Structure):
    _fields_ = [("min", Vec3), ("max", Vec3)]


class NormalDistFunction(IntEnum):
    BECKMANN = 0
    GGX = 1
    COSINE = 2


class ShadowingModel(IntEnum):
    VCAVITY = 0
    SMITH = 1


class MaterialParamType(IntEnum):
    EMISSIVE = 0
    LAMBERT = 1
    ORENNAYAR = 2
    TORRANCE = 3
    WALTER = 4
    BLEND = 5
    FRESNEL = 6
    MICROFACET = 7


class LoaderStatus(IntEnum):
    SUCCESS = 0
    ERROR = 1
    ABORT = 2


class LodMetadata(Structure):
    _fields_ = [("vertices", c_uint32), ("triangles", c_uint32), ("quads", c_uint32), ("edges", c_uint32),
                ("spheres", c_uint32)]


class LightType(IntEnum):
    POINT = 0
    SPOT = 1
    DIRECTIONAL = 2
    ENVMAP = 3


class BackgroundType(IntEnum):
    MONOCHROME = 0
    ENVMAP = 1
    SKY_HOSEK = 2


class Device(IntEnum):
    CPU = 1
    CUDA = 2
    OPENGL = 4


class LogLevel(IntEnum):
    PEDANTIC = 0
    INFO = 1
    WARNING = 2
    ERROR = 3
    FATAL_ERROR = 4


class Medium(Structure):
    _fields_ = [("refractionIndex", Vec2), ("absorption", Vec3)]


class LambertParams(Structure):
    _fields_ = [("albedo", c_void_p)]


class TorranceParams(Structure):
    _fields_ = [("roughness", c_void_p), ("shadowingModel", c_int), ("ndf", c_int), ("albedo", c_void_p)]


class WalterParams(Structure):
    _fields_ = [("roughness", c_void_p), ("shadowingModel", c_int), ("ndf", c_int), ("absorption", Vec3),
                ("refractionIndex", c_float)]


class EmissiveParams(Structure):
    _fields_ = [("radiance", c_void_p), ("scale", Vec3)]


class OrennayarParams(Structure):
    _fields_ = [("albedo", c_void_p), ("roughness", c_float)]


class BlendLayer(Structure):
    _fields_ = [("factor", c_float), ("mat", c_void_p)]


class BlendParams(Structure):
    _fields_ = [("a", BlendLayer), ("b", BlendLayer)]


class FresnelParams(Structure):
    _fields_ = [("refractionIndex", Vec2), ("a", c_void_p), ("b", c_void_p)]


class MaterialParamsDisplacement(Structure):
    _fields_ = [("map", c_void_p), ("maxMips", c_void_p), ("bias", c_float), ("scale", c_float)]


class _MaterialInner(Union):
    _fields_ = [("lambert", LambertParams), ("torrance", TorranceParams), ("walter", WalterParams),
                ("emissive", EmissiveParams), ("orennayar", OrennayarParams), ("blend", BlendParams),
                ("fresnel", FresnelParams)]


class MaterialParams(Structure):
    _fields_ = [("outerMedium", Medium), ("innerType", c_int), ("alpha", c_void_p),
                ("displacement", MaterialParamsDisplacement), ("inner", _MaterialInner)]


class LightHdl(Structure):
    _fields_ = [("type", c_uint32, 3), ("index", c_uint32, 29)]


class _BulkDescriptor(Union):
    _fields_ = [("file", c_void_p), ("bytes", c_void_p)]


class BulkLoader(Structure):
    _fields_ = [("type", c_int), ("descriptor", _BulkDescriptor)]


class MufflonRenderStats(Structure):
    _fields_ = [("rays", c_uint64), ("shadowRays", c_uint64), ("nodeVisits", c_uint64), ("primTests", c_uint64),
                ("instanceVisits", c_uint64), ("errors", c_uint32), ("kernelMs", c_float)]


class MufflonStageStats(Structure):
    _fields_ = [("extensionRays", c_uint64), ("extendNodeVisits", c_uint64), ("extendPrimTests", c_uint64),
                ("extendInstanceVisits", c_uint64), ("shadowRays", c_uint64), ("shadowNodeVisits", c_uint64),
                ("shadowPrimTests", c_uint64), ("shadowInstanceVisits", c_uint64), ("cameraMs", c_float),
                ("extendMs", c_float), ("tailMs", c_float), ("shadeMs", c_float), ("finalizeMs", c_float),
                ("launches", c_uint32), ("wavefront", c_uint32), ("binMs", c_float)]


class MufflonLoadStats(Structure):
    _fields_ = [("totalMs", c_float), ("uploadMs", c_float), ("bvhMs", c_float), ("instanceBvhMs", c_float),
                ("otherMs", c_float), ("pad", c_uint32), ("h2dBytes", c_uint64)]


class MufflonBatchJob(Structure):
    _fields_ = [("instance", c_void_p), ("width", c_uint32), ("height", c_uint32), ("spp", c_uint32),
                ("seed", c_int32), ("minPathLength", c_int32), ("maxPathLength", c_int32),
                ("rrStartDepth", c_int32), ("neeCount", c_int32)]


class MufflonBatchStats(Structure):
    _fields_ = [("deviceMs", c_float), ("launches", c_uint32), ("usedGraph", c_uint32), ("pixels", c_uint32)]


def _bulk(a: np.ndarray) -> BulkLoader:
    b = BulkLoader()
    b.type = 1  # BULK_ARRAY
    b.descriptor.bytes = a.ctypes.data
    return b


def _ptr(a):
    return a.ctypes.data_as(c_void_p) if a is not None and a.size else None


class DllHolder:
    """Loads the library and declares the C signatures."""

    def __init__(self, binary_path=None, useLoader=False):
        path = binary_path or os.environ.get("MUFFLON_CORE_LIB", DEFAULT_LIB)
        if not os.path.exists(path):
            raise RuntimeError(f"libmufflon_core.so not built ({path}); run mufflon_b200.build.build()")
        self.path = path
        self.core = ctypes.CDLL(path, mode=ctypes.RTLD_GLOBAL)
        self.mffLoader = None
        if useLoader:
            lpath = os.path.join(os.path.dirname(path), LOADER_LIB_NAME)
            if not os.path.exists(lpath):
                raise RuntimeError(f"{LOADER_LIB_NAME} not built ({lpath}); run mufflon_b200.build.build()")
            self.mffLoader = ctypes.CDLL(lpath, mode=ctypes.RTLD_GLOBAL)
            for name, (res, args) in {
                "loader_get_dll_error": (c_char_p, []),
                "loader_initialize": (c_void_p, [c_void_p]),
                "loader_destroy": (None, [c_void_p]),
                "loader_load_json": (c_int, [c_void_p, c_char_p]),
                "loader_load_lod": (c_uint32, [c_void_p, c_void_p, c_uint32, c_uint32]),
                "loader_load_object_material_indices": (c_uint32, [c_void_p, c_uint32, c_void_p, POINTER(c_uint32)]),
                "loader_load_lod_metadatas": (c_uint32, [c_void_p, POINTER(LodMetadata), POINTER(c_size_t)]),
                "loader_abort": (c_uint32, [c_void_p]),
                "loader_get_loading_status": (c_char_p, [c_void_p]),
                "loader_get_warnings": (c_char_p, [c_void_p]),
            }.items():
                f = getattr(self.mffLoader, name)
                f.restype = res
                f.argtypes = args
        c = self.core
        sig = {
            "core_get_dll_error": (c_char_p, []),
            "core_set_log_level": (c_uint32, [c_int32]),
            "mufflon_initialize": (c_void_p, []),
            "mufflon_destroy": (None, [c_void_p]),
            "mufflon_is_cuda_available": (c_uint32, []),
            "mufflon_get_cuda_device_index": (c_int32, []),
            "mufflon_get_target_image": (c_uint32, [c_void_p, c_char_p, c_uint32, POINTER(POINTER(c_float))]),
            "mufflon_get_target_image_num_channels": (c_uint32, [c_void_p, POINTER(c_int)]),
            "world_clear_all": (None, [c_void_p]),
            "world_create_object": (c_void_p, [c_void_p, c_char_p, c_int]),
            "object_add_lod": (c_void_p, [c_void_p, c_uint32, c_uint32]),
            "polygon_add_vertex": (c_int32, [c_void_p, Vec3, Vec3, Vec2]),
            "polygon_add_triangle_material": (c_int32, [c_void_p, UVec3, c_uint16]),
            "polygon_add_quad_material": (c_int32, [c_void_p, UVec4, c_uint16]),
            "polygon_add_vertex_bulk": (c_int32, [c_void_p, c_size_t, POINTER(BulkLoader), POINTER(BulkLoader),
                                                  POINTER(BulkLoader), c_void_p, POINTER(c_size_t),
                                                  POINTER(c_size_t), POINTER(c_size_t)]),
            "polygon_add_triangle_bulk": (c_int32, [c_void_p, c_size_t, c_void_p, c_void_p]),
            "polygon_add_quad_bulk": (c_int32, [c_void_p, c_size_t, c_void_p, c_void_p]),
            "spheres_add_sphere_bulk": (c_int32, [c_void_p, c_size_t, POINTER(BulkLoader), c_void_p, POINTER(c_size_t)]),
            "spheres_set_material_idx_bulk": (c_size_t, [c_void_p, c_int32, c_size_t, POINTER(BulkLoader)]),
            "world_create_instance": (c_void_p, [c_void_p, c_void_p, c_uint32]),
            "world_get_instance_count": (c_uint32, [c_void_p, c_uint32]),
            "world_get_object": (c_void_p, [c_void_p, c_char_p]),
            "object_has_lod": (c_uint32, [c_void_p, c_uint32]),
            "object_get_id": (c_uint32, [c_void_p, POINTER(c_uint32)]),
            "instance_get_transformation_matrix": (c_uint32, [c_void_p, c_void_p, POINTER(Mat3x4)]),
            "scenario_get_global_lod_level": (c_uint32, [c_void_p]),
            "scenario_set_global_lod_level": (c_uint32, [c_void_p, c_uint32]),
            "scenario_set_object_lod": (c_uint32, [c_void_p, c_void_p, c_uint32]),
            "scenario_set_instance_lod": (c_uint32, [c_void_p, c_void_p, c_uint32]),
            "scenario_mask_object": (c_uint32, [c_void_p, c_void_p]),
            "scenario_get_resolution": (c_uint32, [c_void_p, POINTER(c_uint32), POINTER(c_uint32)]),
            "scenario_get_name": (c_char_p, [c_void_p]),
            "instance_set_transformation_matrix": (c_uint32, [c_void_p, c_void_p, POINTER(Mat3x4), c_uint32]),
            "world_add_material": (c_void_p, [c_void_p, c_char_p, POINTER(MaterialParams)]),
            "world_add_texture_value": (c_void_p, [c_void_p, POINTER(c_float), c_int, c_int]),
            "world_add_texture_rgba32f": (c_void_p, [c_void_p, c_char_p, c_uint32, c_uint32, c_void_p, c_int]),
            "mufflon_lbvh_build_ex": (c_uint32, [c_void_p, c_uint32, c_void_p, c_uint32, c_uint32, c_void_p, c_uint32,
                                                 c_int32, c_void_p, c_void_p, c_void_p, c_void_p, POINTER(c_int32),
                                                 c_void_p]),
            "world_add_texture": (c_void_p, [c_void_p, c_char_p, c_int, c_int, TextureCallback, c_void_p]),
            "world_get_texture": (c_void_p, [c_void_p, c_char_p]),
            "world_get_texture_name": (c_char_p, [c_void_p]),
            "world_get_texture_size": (c_uint32, [c_void_p, POINTER(IVec2)]),
            "world_add_pinhole_camera": (c_void_p, [c_void_p, c_char_p, POINTER(Vec3), POINTER(Vec3), POINTER(Vec3),
                                                    c_uint32, c_float, c_float, c_float]),
            "world_get_camera": (c_void_p, [c_void_p, c_char_p]),
            "world_create_scenario": (c_void_p, [c_void_p, c_char_p]),
            "world_find_scenario": (c_void_p, [c_void_p, c_char_p]),
            "world_get_current_scenario": (c_void_p, [c_void_p]),
            "world_finalize_scenario": (c_uint32, [c_void_p, c_void_p, POINTER(c_char_p)]),
            "world_load_scenario": (c_void_p, [c_void_p, c_void_p]),
            "scenario_set_resolution": (c_uint32, [c_void_p, c_uint32, c_uint32]),
            "scenario_set_camera": (c_uint32, [c_void_p, c_void_p, c_void_p]),
            "scenario_mask_instance": (c_uint32, [c_void_p, c_void_p]),
            "scenario_add_light": (c_uint32, [c_void_p, c_void_p, LightHdl]),
            "scenario_declare_material_slot": (c_uint16, [c_void_p, c_char_p, c_size_t]),
            "scenario_assign_material": (c_uint32, [c_void_p, c_uint16, c_void_p]),
            "world_add_light": (LightHdl, [c_void_p, c_char_p, c_int, c_uint32]),
            "world_add_background_light": (LightHdl, [c_void_p, c_char_p, c_int]),
            "world_set_point_light_position": (c_uint32, [c_void_p, LightHdl, Vec3, c_uint32]),
            "world_set_point_light_intensity": (c_uint32, [c_void_p, LightHdl, Vec3, c_uint32]),
            "world_set_env_light_color": (c_uint32, [c_void_p, LightHdl, Vec3]),
            "world_set_env_light_scale": (c_uint32, [c_void_p, LightHdl, Vec3]),
            "render_get_renderer_count": (c_uint32, [c_void_p]),
            "render_get_renderer_variations": (c_uint32, [c_void_p, c_uint32]),
            "render_get_renderer_name": (c_char_p, [c_void_p, c_uint32]),
            "render_get_renderer_short_name": (c_char_p, [c_void_p, c_uint32]),
            "render_get_renderer_devices": (c_uint32, [c_void_p, c_uint32, c_uint32]),
            "render_enable_renderer": (c_uint32, [c_void_p, c_uint32, c_uint32]),
            "render_iterate": (c_uint32, [c_void_p, POINTER(ProcessTime), POINTER(ProcessTime), POINTER(ProcessTime)]),
            "render_get_current_iteration": (c_uint32, [c_void_p]),
            "render_reset": (c_uint32, [c_void_p]),
            "render_save_screenshot": (c_uint32, [c_void_p, c_char_p, c_char_p, c_uint32]),
            "render_get_render_target_count": (c_uint32, [c_void_p]),
            "render_get_render_target_name": (c_char_p, [c_void_p, c_uint32]),
            "render_enable_render_target": (c_uint32, [c_void_p, c_char_p, c_uint32]),
            "render_disable_render_target": (c_uint32, [c_void_p, c_char_p, c_uint32]),
            "render_is_render_target_enabled": (c_uint32, [c_void_p, c_char_p, c_uint32]),
            "renderer_get_num_parameters": (c_uint32, [c_void_p]),
            "renderer_get_parameter_desc": (c_char_p, [c_void_p, c_uint32, POINTER(c_int)]),
            "renderer_set_parameter_int": (c_uint32, [c_void_p, c_char_p, c_int32]),
            "renderer_get_parameter_int": (c_uint32, [c_void_p, c_char_p, POINTER(c_int32)]),
            "renderer_set_parameter_float": (c_uint32, [c_void_p, c_char_p, c_float]),
            "renderer_get_parameter_float": (c_uint32, [c_void_p, c_char_p, POINTER(c_float)]),
            "renderer_set_parameter_bool": (c_uint32, [c_void_p, c_char_p, c_uint32]),
            "renderer_get_parameter_bool": (c_uint32, [c_void_p, c_char_p, POINTER(c_uint32)]),
            "renderer_set_parameter_enum": (c_uint32, [c_void_p, c_char_p, c_int32]),
            "mufflon_get_render_stats": (c_uint32, [c_void_p, POINTER(MufflonRenderStats)]),
            "mufflon_get_stage_stats": (c_uint32, [c_void_p, POINTER(MufflonStageStats)]),
            "mufflon_get_load_stats": (c_uint32, [c_void_p, POINTER(MufflonLoadStats)]),
            "mufflon_get_light_tree": (c_uint32, [c_void_p] + [c_void_p] * 8),
            "mufflon_get_lt_records": (c_uint32, [c_void_p, c_void_p, c_void_p, c_uint64]),
            "mufflon_texture_update": (c_uint32, [c_void_p, c_void_p, c_void_p]),
            "mufflon_albedo_gradient": (c_uint32, [c_void_p, c_void_p, c_uint32, c_void_p, c_void_p, POINTER(c_float)]),
            "mufflon_emission_gradient": (c_uint32, [c_void_p, c_void_p, c_uint32, c_void_p, c_void_p, POINTER(c_float)]),
            "mufflon_set_emitted_radiance": (c_uint32, [c_void_p, c_void_p, c_void_p]),
            "mufflon_render_batch": (c_uint32, [POINTER(MufflonBatchJob), c_uint32, c_int32, c_void_p, c_void_p,
                                                POINTER(c_float), POINTER(MufflonBatchStats)]),
            "mufflon_trace_rays": (c_uint32, [c_void_p, c_void_p, c_void_p, c_float, c_uint32, c_void_p, c_void_p,
                                              c_void_p, c_void_p]),
            "mufflon_trace_occlusion": (c_uint32, [c_void_p, c_void_p, c_void_p, c_uint32, c_void_p]),
            "mufflon_get_bvh": (c_uint32, [c_void_p, c_int32, POINTER(c_int32), POINTER(c_int32), c_void_p, c_void_p]),
            "mufflon_lbvh_build": (c_uint32, [c_void_p, c_uint32, c_void_p, c_uint32, c_uint32, c_void_p, c_uint32,
                                              c_void_p, c_void_p, c_void_p, c_void_p, POINTER(c_int32), c_void_p]),
            "mufflon_lbvh_build_device": (c_uint32, [c_void_p, c_void_p, c_uint32, c_uint32, c_void_p, c_uint32,
                                                     c_void_p, POINTER(c_int32), POINTER(c_float), c_void_p]),
            "mufflon_sort_pairs": (c_uint32, [c_void_p, c_void_p, c_uint32]),
            "mufflon_measure_l2_bandwidth": (c_uint32, [c_uint64, c_int32, POINTER(c_float)]),
        }
        for name, (res, args) in sig.items():
            f = getattr(c, name)
            f.restype = res
            f.argtypes = args


class MufflonError(RuntimeError):
    pass


class DllInterface:
    """One method per C function (names as in Mufflon's bindings.py)."""

    def __init__(self, binary_path=None, useLoader=False):
        self.dllHolder = DllHolder(binary_path, useLoader)
        self.core = self.dllHolder.core
        self.loader = self.dllHolder.mffLoader
        self.muffLoaderInst = None
        if not self.core.mufflon_is_cuda_available():
            raise MufflonError("no CUDA device available; the B200 core has no CPU fallback")
        self.muffInst = self.core.mufflon_initialize()
        if not self.muffInst:
            raise MufflonError("mufflon_initialize failed: " + self.core_get_dll_error())
        if self.loader is not None:
            self.muffLoaderInst = self.loader.loader_initialize(self.muffInst)
            if not self.muffLoaderInst:
                raise MufflonError("loader_initialize failed: " + self.loader_get_dll_error())

    def __del__(self):
        try:
            # the loader first: destroying it unregisters its LoD callback from the core instance
            if getattr(self, "muffLoaderInst", None):
                self.loader.loader_destroy(self.muffLoaderInst)
                self.muffLoaderInst = None
            if getattr(self, "muffInst", None):
                self.core.mufflon_destroy(self.muffInst)
                self.muffInst = None
        except Exception:
            pass

    # -- scene-file loader (libmufflon_loader.so, mff_interface.h)
    def loader_get_dll_error(self):
        e = self.loader.loader_get_dll_error()
        return e.decode() if e else ""

    def loader_load_json(self, sceneJson):
        return LoaderStatus(self.loader.loader_load_json(self.muffLoaderInst, str(sceneJson).encode("utf-8")))

    def loader_abort(self):
        return self.loader.loader_abort(self.muffLoaderInst) != 0

    def loader_get_loading_status(self):
        s = self.loader.loader_get_loading_status(self.muffLoaderInst)
        return s.decode() if s else ""

    def loader_get_warnings(self):
        s = self.loader.loader_get_warnings(self.muffLoaderInst)
        return [w for w in (s.decode() if s else "").split("\n") if w]

    def loader_load_lod_metadatas(self, count):
        buf = (LodMetadata * max(count, 1))()
        n = c_size_t(0)
        if not self.loader.loader_load_lod_metadatas(self.muffLoaderInst, buf, byref(n)):
            raise MufflonError("loader_load_lod_metadatas failed: " + self.loader_get_dll_error())
        return [(m.vertices, m.triangles, m.quads, m.edges, m.spheres) for m in buf[:n.value]]

    def loader_load_object_material_indices(self, objId, capacity=65536):
        buf = (c_uint16 * capacity)()
        n = c_uint32(0)
        if not self.loader.loader_load_object_material_indices(self.muffLoaderInst, objId, buf, byref(n)):
            raise MufflonError("loader_load_object_material_indices failed: " + self.loader_get_dll_error())
        return list(buf[:n.value])

    def close(self):
        self.__del__()

    def _check(self, ok, what):
        if not ok:
            raise MufflonError(f"{what} failed: {self.core_get_dll_error()}")
        return ok

    def core_get_dll_error(self):
        e = self.core.core_get_dll_error()
        return e.decode() if e else ""

    def core_set_log_level(self, logLevel):
        return self.core.core_set_log_level(int(logLevel)) != 0

    def world_clear_all(self):
        self.core.world_clear_all(self.muffInst)

    def renderer_set_parameter_bool(self, parameterName, value):
        return self.core.renderer_set_parameter_bool(self.muffInst, parameterName.encode(), 1 if value else 0) != 0

    def renderer_get_parameter_bool(self, parameterName):
        v = c_uint32(0)
        self._check(self.core.renderer_get_parameter_bool(self.muffInst, parameterName.encode(), byref(v)),
                    "renderer_get_parameter_bool")
        return v.value != 0

    def renderer_set_parameter_float(self, parameterName, value):
        return self.core.renderer_set_parameter_float(self.muffInst, parameterName.encode(), value) != 0

    def renderer_set_parameter_int(self, parameterName, value):
        return self.core.renderer_set_parameter_int(self.muffInst, parameterName.encode(), int(value)) != 0

    def renderer_get_parameter_float(self, parameterName):
        v = c_float(0.0)
        self._check(self.core.renderer_get_parameter_float(self.muffInst, parameterName.encode(), byref(v)),
                    "renderer_get_parameter_float")
        return v.value

    def renderer_get_parameter_int(self, parameterName):
        v = c_int32(0)
        self._check(self.core.renderer_get_parameter_int(self.muffInst, parameterName.encode(), byref(v)), "renderer_get_parameter_int")
        return v.value

    def renderer_set_parameter_enum(self, parameterName, value):
        return self.core.renderer_set_parameter_enum(self.muffInst, parameterName.encode(), int(value)) != 0

    def render_iterate(self):
        iterateTime, preTime, postTime = ProcessTime(0, 0), ProcessTime(0, 0), ProcessTime(0, 0)
        self._check(self.core.render_iterate(self.muffInst, byref(iterateTime), byref(preTime), byref(postTime)),
                    "render_iterate")
        return iterateTime, preTime, postTime

    def render_reset(self):
        return self.core.render_reset(self.muffInst) != 0

    def render_get_current_iteration(self):
        return self.core.render_get_current_iteration(self.muffInst)

    def render_save_screenshot(self, fileName, targetName, variance):
        return self.core.render_save_screenshot(self.muffInst, fileName.encode(), targetName.encode(), int(variance)) != 0

    def render_get_render_target_count(self):
        return self.core.render_get_render_target_count(self.muffInst)

    def render_get_render_target_name(self, index):
        return self.core.render_get_render_target_name(self.muffInst, index).decode()

    def render_is_render_target_enabled(self, targetName, variance):
        return self.core.render_is_render_target_enabled(self.muffInst, targetName.encode(), int(variance)) != 0

    def render_enable_render_target(self, targetName, variance):
        return self.core.render_enable_render_target(self.muffInst, targetName.encode(), int(variance)) != 0

    def render_disable_render_target(self, targetName, variance):
        return self.core.render_disable_render_target(self.muffInst, targetName.encode(), int(variance)) != 0

    def render_enable_renderer(self, rendererIndex, variation):
        return self.core.render_enable_renderer(self.muffInst, rendererIndex, variation) != 0

    def render_get_renderer_count(self):
        return self.core.render_get_renderer_count(self.muffInst)

    def render_get_renderer_variations(self, index):
        return self.core.render_get_renderer_variations(self.muffInst, index)

    def render_get_renderer_name(self, rendererIndex):
        return self.core.render_get_renderer_name(self.muffInst, rendererIndex).decode()

    def render_get_renderer_short_name(self, rendererIndex):
        return self.core.render_get_renderer_short_name(self.muffInst, rendererIndex).decode()

    def render_get_renderer_devices(self, rendererIndex, variation):
        return self.core.render_get_renderer_devices(self.muffInst, rendererIndex, variation)

    def world_find_scenario(self, name):
        return self.core.world_find_scenario(self.muffInst, name.encode())

    def world_load_scenario(self, hdl):
        return self.core.world_load_scenario(self.muffInst, hdl)

    def world_get_current_scenario(self):
        return self.core.world_get_current_scenario(self.muffInst)

    def world_get_camera(self, name):
        return self.core.world_get_camera(self.muffInst, name.encode())

    def scenario_set_camera(self, scenario, cam):
        return self.core.scenario_set_camera(self.muffInst, scenario, cam) != 0

    def instance_set_transformation_matrix(self, instHdl, mat, isWorldToInst):
        return self.core.instance_set_transformation_matrix(self.muffInst, instHdl, byref(mat), int(isWorldToInst)) != 0

    # -- image readback
    def get_target_image(self, targetName: str, copy: bool = True, variance: bool = False) -> np.ndarray:
        """Cumulative mean of a target (with variance=True: its recorded variance) as (height, width,
        channels) float32, y = 0 first. With copy=False the array is a view of the library's page-locked
        read-back buffer, valid until the next call of this function (the C API's ownership rule)."""
        p = POINTER(c_float)()
        self._check(self.core.mufflon_get_target_image(self.muffInst, targetName.encode(), 1 if variance else 0,
                                                       byref(p)), "mufflon_get_target_image")
        ch = c_int(0)
        self.core.mufflon_get_target_image_num_channels(self.muffInst, byref(ch))
        if not p:
            return None
        w, h = self.current_resolution()
        view = np.ctypeslib.as_array(p, shape=(h * w * ch.value,)).reshape(h, w, ch.value)
        return view.copy() if copy else view

    def current_resolution(self):
        """(width, height) of the loaded scenario."""
        sc = self.core.world_get_current_scenario(self.muffInst)
        if not sc:
            return self.resolution
        w, h = c_uint32(0), c_uint32(0)
        self._check(self.core.scenario_get_resolution(sc, byref(w), byref(h)), "scenario_get_resolution")
        return w.value, h.value

    # -- extensions
    def render_stats(self):
        s = MufflonRenderStats()
        self._check(self.core.mufflon_get_render_stats(self.muffInst, byref(s)), "mufflon_get_render_stats")
        return {k: getattr(s, k) for k, _ in MufflonRenderStats._fields_}

    def stage_stats(self):
        s = MufflonStageStats()
        self._check(self.core.mufflon_get_stage_stats(self.muffInst, byref(s)), "mufflon_get_stage_stats")
        return {k: getattr(s, k) for k, _ in MufflonStageStats._fields_}

    def lt_records(self, max_path_length: int):
        """The light tracer's camera connections of the last iteration (integer parameter "Record
        connections" set): pixel index per (photon, path length) slot, -1 for none, and the
        (radiance rgb, lightness, density) each added."""
        w, h = self.current_resolution()
        n = w * h * max(1, max_path_length)
        pix = np.zeros(n, np.int32)
        val = np.zeros((n, 5), np.float32)
        self._check(self.core.mufflon_get_lt_records(self.muffInst, _ptr(pix), _ptr(val), n), "mufflon_get_lt_records")
        return pix, val

    def bpt_records(self, max_path_length: int):
        """The bidirectional path tracer's contributions of the last iteration (integer parameter
        "Record connections" set): per pixel M*M connection slots [view length][light vertex], then M
        emitter-hit slots (M = max. path length); pixel index (-1: none) and (radiance rgb, lightness)."""
        w, h = self.current_resolution()
        m = max(1, max_path_length)
        n = w * h * (m * m + m)
        pix = np.zeros(n, np.int32)
        val = np.zeros((n, 4), np.float32)
        self._check(self.core.mufflon_get_lt_records(self.muffInst, _ptr(pix), _ptr(val), n), "mufflon_get_lt_records")
        return pix, val

    def vcm_records(self, max_path_length: int):
        """Vertex connection and merging's contributions of the last iteration (integer parameter
        "Record connections" set): per pixel M*M connection slots [view length][light vertex], then M
        emitter-hit and M merge slots [view length - 1] (M = max. path length); pixel index (-1: none)
        and (radiance rgb, lightness)."""
        w, h = self.current_resolution()
        m = max(1, max_path_length)
        n = w * h * (m * m + 2 * m)
        pix = np.zeros(n, np.int32)
        val = np.zeros((n, 4), np.float32)
        self._check(self.core.mufflon_get_lt_records(self.muffInst, _ptr(pix), _ptr(val), n), "mufflon_get_lt_records")
        return pix, val

    def light_tree(self):
        """The GPU-built light list and tree: (lights (n, 112) uint8, nodes (m, 20) uint8,
        area-light keys uint64, codes uint32, root flux); layout in include/mufflon_core.h."""
        nl, nn, na = c_uint32(), c_uint32(), c_uint32()
        rf = c_float()
        self._check(self.core.mufflon_get_light_tree(self.muffInst, byref(nl), byref(nn), byref(na), None, None, None,
                                                     None, byref(rf)), "mufflon_get_light_tree")
        lights = np.zeros((nl.value, 112), np.uint8)
        nodes = np.zeros((nn.value, 20), np.uint8)
        keys = np.zeros(na.value, np.uint64)
        codes = np.zeros(na.value, np.uint32)
        self._check(self.core.mufflon_get_light_tree(self.muffInst, byref(nl), byref(nn), byref(na), _ptr(lights),
                                                     _ptr(nodes), _ptr(keys), _ptr(codes), byref(rf)),
                    "mufflon_get_light_tree")
        return lights, nodes, keys, codes, rf.value

    def load_stats(self):
        s = MufflonLoadStats()
        self._check(self.core.mufflon_get_load_stats(self.muffInst, byref(s)), "mufflon_get_load_stats")
        return {k: getattr(s, k) for k, _ in MufflonLoadStats._fields_ if k != "pad"}

    def texture_update(self, texture, rgba):
        """Replaces a texture's texels ((H, W, 4) or (H, W, 3) float32) on host and device; resets the accumulation."""
        a = np.asarray(rgba, np.float32)
        if a.ndim == 3 and a.shape[2] == 3:
            a = np.concatenate([a, np.ones(a.shape[:2] + (1,), np.float32)], axis=2)
        a = np.ascontiguousarray(a)
        self._check(self.core.mufflon_texture_update(self.muffInst, texture, a.ctypes.data), "mufflon_texture_update")

    def albedo_gradient(self, texture, spp, image_grad, tex_shape):
        """dLoss/dTexel (H_t, W_t, 3) for imageGrad = dLoss/dImage (H, W, 3) of the spp-sample image."""
        g = np.ascontiguousarray(image_grad, np.float32)
        out = np.zeros((tex_shape[0], tex_shape[1], 3), np.float32)
        ms = c_float(0.0)
        self._check(self.core.mufflon_albedo_gradient(self.muffInst, texture, int(spp), g.ctypes.data, out.ctypes.data,
                                                      byref(ms)), "mufflon_albedo_gradient")
        return out, ms.value

    def emission_gradient(self, material, spp, image_grad):
        """dLoss/dL (3,) for the emitted radiance L (radiance x scale) of an emissive material, for
        imageGrad = dLoss/dImage (H, W, 3) of the spp-sample image; returns (gradient, device ms)."""
        g = np.ascontiguousarray(image_grad, np.float32)
        out = np.zeros(3, np.float32)
        ms = c_float(0.0)
        self._check(self.core.mufflon_emission_gradient(self.muffInst, material, int(spp), g.ctypes.data,
                                                        out.ctypes.data, byref(ms)), "mufflon_emission_gradient")
        return out, ms.value

    def set_emitted_radiance(self, material, rgb):
        """Replaces the emitted radiance (radiance x scale) of an emissive material; the scene is rebuilt
        before the next render."""
        a = np.ascontiguousarray(rgb, np.float32).reshape(3)
        self._check(self.core.mufflon_set_emitted_radiance(self.muffInst, material, a.ctypes.data),
                    "mufflon_set_emitted_radiance")

    def trace_rays(self, rays, tmax=1048576.0, geo_normals=None):
        rays = np.ascontiguousarray(rays, np.float32)
        n = len(rays)
        t = np.zeros(n, np.float32)
        inst = np.zeros(n, np.int32)
        prim = np.zeros(n, np.int32)
        sp = np.zeros((n, 2), np.float32)
        g = None if geo_normals is None else np.ascontiguousarray(geo_normals, np.float32)
        self._check(self.core.mufflon_trace_rays(self.muffInst, _ptr(rays), _ptr(g), tmax, n, _ptr(t), _ptr(inst),
                                                 _ptr(prim), _ptr(sp)), "mufflon_trace_rays")
        return t, inst, prim, sp

    def trace_occlusion(self, a, b):
        a = np.ascontiguousarray(a, np.float32)
        b = np.ascontiguousarray(b, np.float32)
        occ = np.zeros(len(a), np.uint8)
        self._check(self.core.mufflon_trace_occlusion(self.muffInst, _ptr(a), _ptr(b), len(a), _ptr(occ)),
                    "mufflon_trace_occlusion")
        return occ.astype(bool)

    def get_bvh(self, which: int):
        n, ni = c_int32(0), c_int32(0)
        self._check(self.core.mufflon_get_bvh(self.muffInst, which, byref(n), byref(ni), None, None), "mufflon_get_bvh")
        nodes = np.zeros((2 * ni.value, 8), np.float32)
        prim = np.zeros(n.value, np.int32)
        self._check(self.core.mufflon_get_bvh(self.muffInst, which, byref(n), byref(ni), _ptr(nodes), _ptr(prim)),
                    "mufflon_get_bvh")
        return nodes, prim, ni.value


def lbvh_build(dll: DllInterface, lod, morton_bits: int = 63):
    """GPU LBVH build of one LodSpec with 63- or 30-bit Morton codes:
    (morton_sorted, parents, nodes, prim_ids, num_internal, stage_ms)."""
    idx = np.concatenate([lod.triangles.reshape(-1), lod.quads.reshape(-1)]).astype(np.uint32)
    v = np.ascontiguousarray(lod.vertices, np.float32)
    s = np.ascontiguousarray(lod.spheres, np.float32)
    n = lod.num_prims
    morton = np.zeros(max(n, 1), np.uint64)
    parents = np.zeros(max(2 * n - 1, 1), np.int32)
    nodes = np.zeros((max(2 * (n - 1), 1), 8), np.float32)
    prim = np.zeros(max(n, 1), np.int32)
    ni = c_int32(0)
    ms = np.zeros(9, np.float32)
    ok = dll.core.mufflon_lbvh_build_ex(_ptr(v), len(v), _ptr(idx), len(lod.triangles), len(lod.quads), _ptr(s),
                                        len(s), morton_bits, _ptr(morton), _ptr(parents), _ptr(nodes), _ptr(prim),
                                        byref(ni), _ptr(ms))
    dll._check(ok, "mufflon_lbvh_build_ex")
    return morton[:n], parents[:max(2 * n - 1, 0)], nodes[:2 * ni.value], prim[:n], ni.value, ms


def sort_pairs(dll: DllInterface, keys: np.ndarray, values: np.ndarray):
    k = np.ascontiguousarray(keys, np.uint64).copy()
    v = np.ascontiguousarray(values, np.int32).copy()
    dll._check(dll.core.mufflon_sort_pairs(_ptr(k), _ptr(v), len(k)), "mufflon_sort_pairs")
    return k, v


def render_batch(jobs, use_graph=True, hit_ids=False):
    """Renders a batch with mufflon_render_batch.

    `jobs` is a list of dicts: instance (a DllInterface with a loaded
    scenario), width, height (0 = the scenario's), spp, seed, min_path,
    max_path, rr_start, nee. Returns (radiance images (H, W, 3), hit-id images
    or None, per-job completion ms, stats dict)."""
    if not jobs:
        raise ValueError("empty batch")
    core = jobs[0]["instance"].core
    arr = (MufflonBatchJob * len(jobs))()
    imgs, hits = [], []
    for j, d in enumerate(jobs):
        inst = d["instance"]
        w, h = d.get("width", 0), d.get("height", 0)
        if not w or not h:
            w, h = inst.resolution
        arr[j] = MufflonBatchJob(inst.muffInst, w, h, d["spp"], d.get("seed", 0), d.get("min_path", 0),
                                 d.get("max_path", 16), d.get("rr_start", 0), d.get("nee", 1))
        imgs.append(np.zeros((h, w, 3), np.float32))
        hits.append(np.zeros((h, w, 2), np.float32) if hit_ids else None)
    rad_ptrs = (c_void_p * len(jobs))(*[im.ctypes.data for im in imgs])
    hit_ptrs = (c_void_p * len(jobs))(*[(hm.ctypes.data if hm is not None else None) for hm in hits])
    done = (c_float * len(jobs))()
    st = MufflonBatchStats()
    if not core.mufflon_render_batch(arr, len(jobs), 1 if use_graph else 0, rad_ptrs, hit_ptrs if hit_ids else None,
                                     done, byref(st)):
        raise MufflonError(f"mufflon_render_batch failed: {core.core_get_dll_error().decode()}")
    return imgs, (hits if hit_ids else None), list(done), {k: getattr(st, k) for k, _ in MufflonBatchStats._fields_}


def load_scene_spec(dll: DllInterface, spec, scenario_name: str = None, texture_files=None, texture_callback=None):
    """Builds a SceneSpec through the world-building C API and loads it. With `texture_files`
    (a path per texture of the spec), the textures are read from those files with world_add_texture,
    passing `texture_callback` (a TextureCallback or None), instead of from the spec's arrays."""
    core, I = dll.core, dll.muffInst
    keep = []
    sc = core.world_create_scenario(I, (scenario_name or spec.name).encode())
    dll._check(sc, "world_create_scenario")

    def tex_value(vals):
        arr = (c_float * len(vals))(*[float(x) for x in vals])
        t = core.world_add_texture_value(I, arr, len(vals), 0)
        dll._check(t, "world_add_texture_value")
        return t

    textures = []
    for k, tex in enumerate(spec.textures):
        if texture_files is not None:
            t = core.world_add_texture(I, str(texture_files[k]).encode(), 0, 0,
                                       texture_callback or TextureCallback(), None)
            dll._check(t, "world_add_texture")
            textures.append(t)
            continue
        a = np.ascontiguousarray(tex, np.float32)
        keep.append(a)
        t = core.world_add_texture_rgba32f(I, f"texture{k}".encode(), a.shape[1], a.shape[0], _ptr(a), 0)
        dll._check(t, "world_add_texture_rgba32f")
        textures.append(t)
    dll.textures = textures
    dll.materials = []  # material handles in the spec's order (its slot indices)
    for i, m in enumerate(spec.materials):
        name = f"mat{i}".encode()
        slot = core.scenario_declare_material_slot(sc, name, len(name))
        p = MaterialParams()
        p.outerMedium.refractionIndex.u = 1.0
        if m.type == 0:
            p.innerType = MaterialParamType.LAMBERT
            p.inner.lambert.albedo = textures[m.albedo_texture] if m.albedo_texture >= 0 else tex_value(m.albedo)
        elif m.type == 1:
            p.innerType = MaterialParamType.TORRANCE
            p.inner.torrance.albedo = textures[m.albedo_texture] if m.albedo_texture >= 0 else tex_value(m.albedo)
            p.inner.torrance.roughness = tex_value(m.roughness)
            p.inner.torrance.shadowingModel = ShadowingModel.SMITH if m.shadowing == 1 else ShadowingModel.VCAVITY
            p.inner.torrance.ndf = NormalDistFunction.GGX
        else:
            p.innerType = MaterialParamType.EMISSIVE
            p.inner.emissive.radiance = tex_value(m.radiance)
            p.inner.emissive.scale = Vec3(*m.scale)
        if getattr(m, "alpha_texture", -1) >= 0:
            p.alpha = textures[m.alpha_texture]
        mh = core.world_add_material(I, name, byref(p))
        dll._check(mh, "world_add_material")
        dll.materials.append(mh)
        dll._check(core.scenario_assign_material(sc, slot, mh), "scenario_assign_material")
    objs = []
    for li, lod in enumerate(spec.lods):
        obj = core.world_create_object(I, lod.name.encode(), 0)
        dll._check(obj, "world_create_object")
        lh = core.object_add_lod(obj, 0, 0)
        dll._check(lh, "object_add_lod")
        nv = len(lod.vertices)
        if nv:
            pts = np.ascontiguousarray(lod.vertices, np.float32)
            nrm = np.ascontiguousarray(lod.normals, np.float32)
            uvs = np.ascontiguousarray(lod.uvs, np.float32)
            keep += [pts, nrm, uvs]
            bp, bn, bu = _bulk(pts), _bulk(nrm), _bulk(uvs)
            r = core.polygon_add_vertex_bulk(lh, nv, byref(bp), byref(bn), byref(bu), None, None, None, None)
            dll._check(r >= 0, "polygon_add_vertex_bulk")
        fm = np.ascontiguousarray(lod.face_materials, np.uint16)
        nt, nq = len(lod.triangles), len(lod.quads)
        if nt:
            t = np.ascontiguousarray(lod.triangles, np.uint32)
            dll._check(core.polygon_add_triangle_bulk(lh, nt, _ptr(t), _ptr(fm[:nt].copy())) >= 0, "polygon_add_triangle_bulk")
        if nq:
            q = np.ascontiguousarray(lod.quads, np.uint32)
            dll._check(core.polygon_add_quad_bulk(lh, nq, _ptr(q), _ptr(fm[nt:].copy())) >= 0, "polygon_add_quad_bulk")
        ns = len(lod.spheres)
        if ns:
            sph = np.ascontiguousarray(lod.spheres, np.float32)
            sm = np.ascontiguousarray(lod.sphere_materials, np.uint16)
            keep += [sph, sm]
            bs = _bulk(sph)
            dll._check(core.spheres_add_sphere_bulk(lh, ns, byref(bs), None, None) >= 0, "spheres_add_sphere_bulk")
            bm = _bulk(sm)
            dll._check(core.spheres_set_material_idx_bulk(lh, 0, ns, byref(bm)) == ns, "spheres_set_material_idx_bulk")
        objs.append(obj)
    for i in range(len(spec.instance_lod)):
        li = int(spec.instance_lod[i])
        masked = li == 0xFFFFFFFF
        ih = core.world_create_instance(I, objs[0 if masked else li], 0)
        dll._check(ih, "world_create_instance")
        m = Mat3x4()
        m.v[:] = [float(x) for x in spec.world_to_instance[i]]
        dll._check(core.instance_set_transformation_matrix(I, ih, byref(m), 1), "instance_set_transformation_matrix")
        if masked:
            core.scenario_mask_instance(sc, ih)
    cam = core.world_add_pinhole_camera(I, b"camera", byref(Vec3(*spec.cam_pos)), byref(Vec3(*spec.cam_dir)),
                                        byref(Vec3(*spec.cam_up)), 1, 1e-4, 1e10, spec.vfov)
    dll._check(cam, "world_add_pinhole_camera")
    dll._check(core.scenario_set_camera(I, sc, cam), "scenario_set_camera")
    dll._check(core.scenario_set_resolution(sc, spec.width, spec.height), "scenario_set_resolution")
    for k, pl in enumerate(spec.point_lights):
        h = core.world_add_light(I, f"point{k}".encode(), LightType.POINT, 1)
        core.world_set_point_light_position(I, h, Vec3(*pl[:3]), 0)
        core.world_set_point_light_intensity(I, h, Vec3(*pl[3:]), 0)
        dll._check(core.scenario_add_light(I, sc, h), "scenario_add_light")
    if spec.background is not None:
        h = core.world_add_background_light(I, b"background", BackgroundType.MONOCHROME)
        core.world_set_env_light_color(I, h, Vec3(*spec.background[0]))
        core.world_set_env_light_scale(I, h, Vec3(*spec.background[1]))
        dll._check(core.scenario_add_light(I, sc, h), "scenario_add_light")
    msg = c_char_p()
    dll._check(core.world_finalize_scenario(I, sc, byref(msg)), "world_finalize_scenario")
    dll._check(core.world_load_scenario(I, sc), "world_load_scenario")
    dll.resolution = (spec.width, spec.height)
    return sc


def load_scene_file(dll: DllInterface, path: str):
    """Loads a JSON scene file (and its binary) through loader_load_json; raises on failure."""
    if dll.loader is None:
        raise MufflonError("the DllInterface was created without the loader (useLoader=False)")
    status = dll.loader_load_json(path)
    if status != LoaderStatus.SUCCESS:
        raise MufflonError(f"Failed to load scene '{path}' ({status.name}): {dll.loader_get_dll_error()}")
    sc = dll.core.world_get_current_scenario(dll.muffInst)
    w, h = c_uint32(0), c_uint32(0)
    dll.core.scenario_get_resolution(sc, byref(w), byref(h))
    dll.resolution = (w.value, h.value)
    return sc


class RenderActions:
    """Convenience layer with the method names of Mufflon's RenderActions."""

    def __init__(self, binary_path=None, useLoader=True):
        self.dllInterface = DllInterface(binary_path, useLoader)
        self.activeRendererName = ""
        self.sceneName = ""

    def load_json(self, sceneJson, defaultRenderTarget="Radiance"):
        self.sceneName = os.path.splitext(os.path.basename(sceneJson))[0]
        load_scene_file(self.dllInterface, sceneJson)
        self.enable_render_target(defaultRenderTarget, False)

    def load_spec(self, spec, defaultRenderTarget="Radiance"):
        self.sceneName = spec.name
        load_scene_spec(self.dllInterface, spec)
        self.enable_render_target(defaultRenderTarget, False)

    def enable_renderer(self, rendererName, devices):
        d = self.dllInterface
        for i in range(d.render_get_renderer_count()):
            name = d.render_get_renderer_name(i)
            short = d.render_get_renderer_short_name(i)
            if name.lower() == rendererName.lower() or short.lower() == rendererName.lower():
                for v in range(d.render_get_renderer_variations(i)):
                    if int(devices) == d.render_get_renderer_devices(i, v):
                        self.activeRendererName = rendererName
                        d.render_enable_renderer(i, v)
                        return
        raise MufflonError(f"Could not find renderer '{rendererName}' for the devices {devices}")

    def load_scenario(self, scenarioName):
        d = self.dllInterface
        hdl = d.world_find_scenario(scenarioName)
        if not hdl:
            raise MufflonError(f"Failed to find scenario '{scenarioName}'")
        if not d.world_load_scenario(hdl):
            raise MufflonError(f"Failed to load scenario '{scenarioName}'")

    def enable_render_target(self, targetName, variance):
        if not self.dllInterface.render_enable_render_target(targetName, variance):
            raise MufflonError(f"Failed to enable render target {targetName} (variance: {variance})")

    def disable_render_target(self, targetName, variance):
        if not self.dllInterface.render_disable_render_target(targetName, variance):
            raise MufflonError(f"Failed to disable render target {targetName} (variance: {variance})")

    def renderer_set_parameter_int(self, parameterName, value):
        return self.dllInterface.renderer_set_parameter_int(parameterName, value)

    def renderer_set_parameter_bool(self, parameterName, value):
        return self.dllInterface.renderer_set_parameter_bool(parameterName, value)

    def render_reset(self):
        self.dllInterface.render_reset()

    def render_for_iterations(self, iterationCount, printProgress=False, progressSteps=1, takeScreenshot=False):
        acc = ProcessTime(0, 0)
        for i in range(iterationCount):
            if printProgress and (i % progressSteps == 0):
                print("--- ", (i + 1), " of ", iterationCount, " ---", flush=True)
            it, _, _ = self.dllInterface.render_iterate()
            acc.microseconds += it.microseconds
        return acc

    def get_target(self, targetName="Radiance"):
        return self.dllInterface.get_target_image(targetName)
