"""ctypes wrapper of the CPU oracle (liboracle.so): TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this
module, as a checker. The product library never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")
_lib = None


class OrLod(C.Structure):
    _fields_ = [("numVertices", C.c_uint32), ("numTriangles", C.c_uint32), ("numQuads", C.c_uint32),
                ("numSpheres", C.c_uint32), ("vertices", C.c_void_p), ("normals", C.c_void_p),
                ("uvs", C.c_void_p), ("indices", C.c_void_p), ("faceMaterials", C.c_void_p),
                ("spheres", C.c_void_p), ("sphereMaterials", C.c_void_p)]


class OrMaterial(C.Structure):
    _fields_ = [("type", C.c_int32), ("albedo", C.c_float * 3), ("roughness", C.c_float * 2),
                ("shadowing", C.c_int32), ("ndf", C.c_int32), ("radiance", C.c_float * 3),
                ("scale", C.c_float * 3), ("albedoTexture", C.c_int32), ("alphaTexture", C.c_int32)]


class OrTexture(C.Structure):
    _fields_ = [("width", C.c_uint32), ("height", C.c_uint32), ("texels", C.c_void_p)]


class OrSceneDesc(C.Structure):
    _fields_ = [("numLods", C.c_uint32), ("lods", C.POINTER(OrLod)), ("numInstances", C.c_uint32),
                ("worldToInstance", C.c_void_p), ("instanceLod", C.c_void_p), ("numMaterials", C.c_uint32),
                ("materials", C.POINTER(OrMaterial)), ("numTextures", C.c_uint32),
                ("textures", C.POINTER(OrTexture)), ("numPointLights", C.c_uint32),
                ("pointLights", C.c_void_p), ("hasBackground", C.c_int32), ("backgroundColor", C.c_float * 3),
                ("backgroundScale", C.c_float * 3), ("camPos", C.c_float * 3), ("camDir", C.c_float * 3),
                ("camUp", C.c_float * 3), ("vFov", C.c_float), ("nearPlane", C.c_float), ("farPlane", C.c_float),
                ("width", C.c_uint32), ("height", C.c_uint32)]


class OrPtParams(C.Structure):
    _fields_ = [("seed", C.c_int32), ("minPathLength", C.c_int32), ("maxPathLength", C.c_int32),
                ("neeCount", C.c_int32), ("neePositionGuide", C.c_int32), ("rrStartDepth", C.c_int32)]


class OrLtParams(C.Structure):
    _fields_ = [("seed", C.c_int32), ("minPathLength", C.c_int32), ("maxPathLength", C.c_int32),
                ("density", C.c_int32)]


class OrStats(C.Structure):
    _fields_ = [("rays", C.c_uint64), ("shadowRays", C.c_uint64), ("nodeVisits", C.c_uint64),
                ("instanceVisits", C.c_uint64), ("triTests", C.c_uint64), ("quadTests", C.c_uint64),
                ("sphereTests", C.c_uint64)]


def build():
    """Compile liboracle.so with the recipe in oracle/Makefile."""
    subprocess.check_call(["make", "-s", "-C", _HERE])


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        _lib = C.CDLL(_LIB_PATH)
        L = _lib
        L.oracle_scene_create.restype = C.c_void_p
        L.oracle_scene_create.argtypes = [C.POINTER(OrSceneDesc)]
        L.oracle_scene_destroy.argtypes = [C.c_void_p]
        L.oracle_bvh_info.argtypes = [C.c_void_p, C.c_int32, C.POINTER(C.c_int32), C.POINTER(C.c_int32)]
        L.oracle_bvh_get.argtypes = [C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        L.oracle_scene_aabb.argtypes = [C.c_void_p, C.c_void_p]
        L.oracle_light_tree.argtypes = [C.c_void_p] + [C.c_void_p] * 8
        L.oracle_light_build_ms.restype = C.c_double
        L.oracle_light_build_ms.argtypes = [C.c_void_p]
        L.oracle_trace_first.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_float, C.c_uint32,
                                         C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        L.oracle_trace_any.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p]
        L.oracle_pt_create.restype = C.c_void_p
        L.oracle_pt_create.argtypes = [C.c_void_p, C.POINTER(OrPtParams)]
        L.oracle_pt_destroy.argtypes = [C.c_void_p]
        L.oracle_albedo_gradient.argtypes = [C.c_void_p, C.c_int32, C.c_uint32, C.c_void_p, C.c_void_p, C.c_int32]
        L.oracle_albedo_gradient.restype = C.c_int
        L.oracle_emission_gradient.argtypes = [C.c_void_p, C.c_int32, C.c_uint32, C.c_void_p, C.c_void_p, C.c_int32]
        L.oracle_emission_gradient.restype = C.c_int
        L.oracle_pt_iterate.argtypes = [C.c_void_p, C.c_int32]
        L.oracle_pt_iterate_rows.argtypes = [C.c_void_p, C.c_int32, C.c_uint32, C.c_uint32]
        L.oracle_pt_get_target.argtypes = [C.c_void_p, C.c_int32, C.c_void_p]
        L.oracle_pt_stats.argtypes = [C.c_void_p, C.POINTER(OrStats)]
        L.oracle_lt_create.restype = C.c_void_p
        L.oracle_lt_create.argtypes = [C.c_void_p, C.POINTER(OrLtParams)]
        L.oracle_lt_destroy.argtypes = [C.c_void_p]
        L.oracle_lt_iterate.argtypes = [C.c_void_p, C.c_int32]
        L.oracle_lt_get_target.argtypes = [C.c_void_p, C.c_int32, C.c_void_p]
        L.oracle_lt_records.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        L.oracle_lt_stats.argtypes = [C.c_void_p, C.POINTER(OrStats)]
        L.oracle_bpt_create.restype = C.c_void_p
        L.oracle_bpt_create.argtypes = [C.c_void_p, C.POINTER(OrLtParams)]
        L.oracle_bpt_destroy.argtypes = [C.c_void_p]
        L.oracle_bpt_iterate.argtypes = [C.c_void_p, C.c_int32]
        L.oracle_bpt_get_target.argtypes = [C.c_void_p, C.c_int32, C.c_void_p]
        L.oracle_bpt_records.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        L.oracle_bpt_stats.argtypes = [C.c_void_p, C.POINTER(OrStats)]
        L.oracle_vcm_create.restype = C.c_void_p
        L.oracle_vcm_create.argtypes = [C.c_void_p, C.POINTER(OrLtParams), C.c_float, C.c_int32]
        L.oracle_vcm_destroy.argtypes = [C.c_void_p]
        L.oracle_vcm_iterate.argtypes = [C.c_void_p, C.c_int32]
        L.oracle_vcm_get_target.argtypes = [C.c_void_p, C.c_int32, C.c_void_p]
        L.oracle_vcm_records.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        L.oracle_vcm_stats.argtypes = [C.c_void_p, C.POINTER(OrStats)]
        L.oracle_vcm_map_size.restype = C.c_uint32
        L.oracle_vcm_map_size.argtypes = [C.c_uint32]
        L.oracle_wang_hash.restype = C.c_uint32
        L.oracle_wang_hash.argtypes = [C.c_uint32]
        L.oracle_wireframe_create.restype = C.c_void_p
        L.oracle_wireframe_create.argtypes = [C.c_void_p, C.c_float, C.c_int32]
        L.oracle_wireframe_destroy.argtypes = [C.c_void_p]
        L.oracle_wireframe_iterate.argtypes = [C.c_void_p, C.c_int32]
        L.oracle_wireframe_get_target.argtypes = [C.c_void_p, C.c_void_p]
        L.oracle_wireframe_get_variance.argtypes = [C.c_void_p, C.c_void_p]
        L.oracle_pcg64_seed.restype = C.c_uint64
        L.oracle_pcg64_seed.argtypes = [C.c_uint32]
        L.oracle_pcg64_next.restype = C.c_uint64
        L.oracle_pcg64_next.argtypes = [C.POINTER(C.c_uint64)]
        L.oracle_part_by_two21.restype = C.c_uint64
        L.oracle_part_by_two21.argtypes = [C.c_uint32]
        L.oracle_part_by_two10.restype = C.c_uint32
        L.oracle_part_by_two10.argtypes = [C.c_uint32]
        L.oracle_scene_rebuild_lod_bvhs.restype = C.c_int
        L.oracle_scene_rebuild_lod_bvhs.argtypes = [C.c_void_p, C.c_int32]
        L.oracle_scramble_seed.restype = C.c_uint64
        L.oracle_scramble_seed.argtypes = [C.c_uint32]
        L.oracle_golden_ratio2d.argtypes = [C.c_uint32, C.c_uint32, C.c_void_p]
        for f in ("oracle_part_by_two16",):
            getattr(L, f).restype = C.c_uint64
            getattr(L, f).argtypes = [C.c_uint32]
        for f in ("oracle_morton_code16", "oracle_hilbert_code16"):
            getattr(L, f).restype = C.c_uint64
            getattr(L, f).argtypes = [C.c_uint32, C.c_uint32, C.c_uint32]
        L.oracle_karras.argtypes = [C.c_void_p, C.c_int32, C.c_void_p]
        L.oracle_sincos.argtypes = [C.c_float, C.POINTER(C.c_float), C.POINTER(C.c_float)]
        L.oracle_atan2.restype = C.c_float
        L.oracle_atan2.argtypes = [C.c_float, C.c_float]
        L.oracle_acos.restype = C.c_float
        L.oracle_acos.argtypes = [C.c_float]
    return _lib


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p) if a is not None and a.size else None


class OracleScene:
    """Owns the numpy buffers referenced by the descriptor while the scene is built."""

    def __init__(self, spec):
        L = lib()
        self.spec = spec
        keep = []
        lods = (OrLod * max(1, len(spec.lods)))()
        for i, l in enumerate(spec.lods):
            idx = np.concatenate([l.triangles.reshape(-1), l.quads.reshape(-1)]).astype(np.uint32)
            arrs = [np.ascontiguousarray(l.vertices, np.float32), np.ascontiguousarray(l.normals, np.float32),
                    np.ascontiguousarray(l.uvs, np.float32), np.ascontiguousarray(idx),
                    np.ascontiguousarray(l.face_materials, np.uint16), np.ascontiguousarray(l.spheres, np.float32),
                    np.ascontiguousarray(l.sphere_materials, np.uint16)]
            keep += arrs
            lods[i] = OrLod(len(l.vertices), len(l.triangles), len(l.quads), len(l.spheres),
                            *[_ptr(a) for a in arrs])
        mats = (OrMaterial * max(1, len(spec.materials)))()
        for i, m in enumerate(spec.materials):
            mats[i] = OrMaterial(m.type, (C.c_float * 3)(*m.albedo), (C.c_float * 2)(*m.roughness),
                                 int(m.shadowing), 0,
                                 (C.c_float * 3)(*m.radiance), (C.c_float * 3)(*m.scale), m.albedo_texture,
                                 getattr(m, "alpha_texture", -1))
        texs = (OrTexture * max(1, len(spec.textures)))()
        for i, t in enumerate(spec.textures):
            a = np.ascontiguousarray(t, np.float32)
            keep.append(a)
            texs[i] = OrTexture(a.shape[1], a.shape[0], _ptr(a))
        w2i = np.ascontiguousarray(spec.world_to_instance, np.float32)
        il = np.ascontiguousarray(spec.instance_lod, np.uint32)
        pl = np.ascontiguousarray(spec.point_lights, np.float32)
        keep += [w2i, il, pl]
        d = OrSceneDesc()
        d.numLods = len(spec.lods)
        d.lods = lods
        d.numInstances = len(il)
        d.worldToInstance = _ptr(w2i)
        d.instanceLod = _ptr(il)
        d.numMaterials = len(spec.materials)
        d.materials = mats
        d.numTextures = len(spec.textures)
        d.textures = texs
        d.numPointLights = len(pl)
        d.pointLights = _ptr(pl)
        d.hasBackground = 1 if spec.background is not None else 0
        if spec.background is not None:
            d.backgroundColor = (C.c_float * 3)(*spec.background[0])
            d.backgroundScale = (C.c_float * 3)(*spec.background[1])
        d.camPos = (C.c_float * 3)(*spec.cam_pos)
        d.camDir = (C.c_float * 3)(*spec.cam_dir)
        d.camUp = (C.c_float * 3)(*spec.cam_up)
        d.vFov = spec.vfov
        d.nearPlane = 1e-4
        d.farPlane = 1e10
        d.width = spec.width
        d.height = spec.height
        self.handle = L.oracle_scene_create(C.byref(d))
        if not self.handle:
            raise RuntimeError("oracle_scene_create failed")

    def close(self):
        if self.handle:
            lib().oracle_scene_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def bvh(self, which: int):
        """(morton_sorted, parents, nodes (n,8) float32 view, prim_ids, num_internal); which=-1 is the TLAS."""
        L = lib()
        np_, ni = C.c_int32(), C.c_int32()
        if not L.oracle_bvh_info(self.handle, which, C.byref(np_), C.byref(ni)):
            raise IndexError(which)
        n = np_.value
        morton = np.zeros(max(n, 0), np.uint64)
        parents = np.zeros(max(2 * n - 1, 0), np.int32)
        nodes = np.zeros((2 * ni.value, 8), np.float32)
        prim = np.zeros(max(n, 0), np.int32)
        L.oracle_bvh_get(self.handle, which, _ptr(morton), _ptr(parents), _ptr(nodes), _ptr(prim))
        return morton, parents, nodes, prim, ni.value

    def rebuild_lod_bvhs(self, morton_bits: int):
        """Rebuilds the LoD hierarchies with 63- or 30-bit Morton codes."""
        if not lib().oracle_scene_rebuild_lod_bvhs(self.handle, morton_bits):
            raise ValueError(f"Morton codes have 63 or 30 bits, not {morton_bits}")

    def aabb(self):
        a = np.zeros(6, np.float32)
        lib().oracle_scene_aabb(self.handle, _ptr(a))
        return a

    def light_build_ms(self):
        """Host time of this scene's light list and tree build (one thread)."""
        return lib().oracle_light_build_ms(self.handle)

    def light_tree(self):
        """(lights (n, 112) uint8, nodes (m, 20) uint8, keys uint64, codes uint32, root flux) in the
        core's device layout."""
        nl, nn, nc = C.c_uint32(), C.c_uint32(), C.c_uint32()
        rf = C.c_float()
        lib().oracle_light_tree(self.handle, C.byref(nl), C.byref(nn), C.byref(nc), None, None, None, None, None)
        lights = np.zeros((nl.value, 112), np.uint8)
        nodes = np.zeros((nn.value, 20), np.uint8)
        keys = np.zeros(nc.value, np.uint64)
        codes = np.zeros(nc.value, np.uint32)
        lib().oracle_light_tree(self.handle, C.byref(nl), C.byref(nn), C.byref(nc), _ptr(lights), _ptr(nodes),
                                _ptr(keys), _ptr(codes), C.byref(rf))
        return lights, nodes, keys, codes, rf.value

    def trace_first(self, rays: np.ndarray, tmax: float = 1048576.0, geo_normals=None):
        rays = np.ascontiguousarray(rays, np.float32)
        n = len(rays)
        t = np.zeros(n, np.float32)
        inst = np.zeros(n, np.int32)
        prim = np.zeros(n, np.int32)
        sp = np.zeros((n, 2), np.float32)
        g = None if geo_normals is None else np.ascontiguousarray(geo_normals, np.float32)
        lib().oracle_trace_first(self.handle, _ptr(rays), _ptr(g), tmax, n, _ptr(t), _ptr(inst), _ptr(prim), _ptr(sp))
        return t, inst, prim, sp

    def trace_any(self, a: np.ndarray, b: np.ndarray):
        a = np.ascontiguousarray(a, np.float32)
        b = np.ascontiguousarray(b, np.float32)
        occ = np.zeros(len(a), np.uint8)
        lib().oracle_trace_any(self.handle, _ptr(a), _ptr(b), len(a), _ptr(occ))
        return occ.astype(bool)


class OraclePathTracer:
    def __init__(self, scene: OracleScene, seed=0, min_path=0, max_path=16, nee_count=1, rr_start=0):
        self.scene = scene
        p = OrPtParams(seed, min_path, max_path, nee_count, 0, rr_start)
        self.handle = lib().oracle_pt_create(scene.handle, C.byref(p))

    def iterate(self, threads: int = 0):
        if threads <= 0:
            threads = os.cpu_count() or 1
        lib().oracle_pt_iterate(self.handle, threads)

    def iterate_rows(self, y0: int, y1: int, threads: int = 0):
        """One untallied pass over rows [y0, y1) (CPU baseline timing)."""
        if threads <= 0:
            threads = os.cpu_count() or 1
        lib().oracle_pt_iterate_rows(self.handle, threads, y0, y1)

    # the auxiliary targets (pt_params.hpp:16-26): oracle target index, channels
    AUX = {"Position": (4, 3), "Depth": (5, 1), "Normal": (6, 3), "UV": (7, 2), "Albedo": (8, 3), "Lightness": (9, 1)}

    def target(self, name: str, variance: bool = False):
        """Cumulative target, or with variance=True its running variance."""
        w, h = self.scene.spec.width, self.scene.spec.height
        if name == "Radiance":
            out = np.zeros((h, w, 3), np.float32)
            lib().oracle_pt_get_target(self.handle, 2 if variance else 0, _ptr(out))
        elif name == "Hit ID":
            out = np.zeros((h, w, 2), np.float32)
            lib().oracle_pt_get_target(self.handle, 3 if variance else 1, _ptr(out))
        elif name in self.AUX:
            k, ch = self.AUX[name]
            out = np.zeros((h, w, ch), np.float32)
            lib().oracle_pt_get_target(self.handle, k + (6 if variance else 0), _ptr(out))
        else:
            raise KeyError(name)
        return out

    def albedo_gradient(self, texture_index: int, spp: int, image_grad, threads: int = 0) -> np.ndarray:
        """dLoss/dTexel (H_t, W_t, 3) in float64 for imageGrad = dLoss/dImage (H, W, 3), replaying spp
        samples per pixel from the seed (test reference of the GPU adjoint)."""
        if threads <= 0:
            threads = os.cpu_count() or 1
        tex = self.scene.spec.textures[texture_index]
        g = np.ascontiguousarray(image_grad, np.float32)
        out = np.zeros((tex.shape[0], tex.shape[1], 3), np.float64)
        if not lib().oracle_albedo_gradient(self.handle, texture_index, spp, _ptr(g), _ptr(out), threads):
            raise ValueError("oracle_albedo_gradient: invalid arguments (is Russian roulette off?)")
        return out

    def emission_gradient(self, material_index: int, spp: int, image_grad, threads: int = 0) -> np.ndarray:
        """dLoss/dL (3,) in float64 for the emitted radiance L = radiance x scale of emissive material
        `material_index` (index into the scene's material list), for imageGrad = dLoss/dImage (H, W, 3),
        replaying spp samples per pixel from the seed (test reference of the GPU emission adjoint)."""
        if threads <= 0:
            threads = os.cpu_count() or 1
        g = np.ascontiguousarray(image_grad, np.float32)
        out = np.zeros(3, np.float64)
        if not lib().oracle_emission_gradient(self.handle, material_index, spp, _ptr(g), _ptr(out), threads):
            raise ValueError("oracle_emission_gradient: invalid arguments (not an emissive material?)")
        return out

    def stats(self):
        s = OrStats()
        lib().oracle_pt_stats(self.handle, C.byref(s))
        return {k: getattr(s, k) for k, _ in OrStats._fields_}

    def close(self):
        if self.handle:
            lib().oracle_pt_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class OracleLightTracer:
    """CPU restatement of the light tracer (lt_common.hpp, cpu_lt.cpp): one photon per pixel index and
    iteration, every path vertex connected to the camera."""

    TARGETS = {"Radiance": (0, 3), "Lightness": (1, 1), "Density": (2, 1)}

    def __init__(self, scene: OracleScene, seed=0, min_path=0, max_path=16, density=False):
        self.scene = scene
        self.max_path = max(1, max_path)
        p = OrLtParams(seed, min_path, max_path, 1 if density else 0)
        self.handle = lib().oracle_lt_create(scene.handle, C.byref(p))
        if not self.handle:
            raise ValueError("oracle_lt_create failed")

    def iterate(self, threads: int = 0):
        if threads <= 0:
            threads = os.cpu_count() or 1
        lib().oracle_lt_iterate(self.handle, threads)

    def target(self, name: str, variance: bool = False):
        """Cumulative target (Density: the last iteration's), or with variance=True its variance
        buffer (Density: its running mean; the target reduces moments)."""
        w, h = self.scene.spec.width, self.scene.spec.height
        idx, ch = self.TARGETS[name]
        out = np.zeros((h, w, ch), np.float32)
        lib().oracle_lt_get_target(self.handle, idx + (3 if variance else 0), _ptr(out))
        return out

    def records(self):
        """The last iteration's camera connections: pixel index per (photon, path length) slot (-1: none)
        and (radiance rgb, lightness, density) as added."""
        n = self.scene.spec.width * self.scene.spec.height * self.max_path
        pix = np.zeros(n, np.int32)
        val = np.zeros((n, 5), np.float32)
        if not lib().oracle_lt_records(self.handle, _ptr(pix), _ptr(val)):
            raise RuntimeError("no iteration has run")
        return pix, val

    def stats(self):
        s = OrStats()
        lib().oracle_lt_stats(self.handle, C.byref(s))
        return {k: getattr(s, k) for k, _ in OrStats._fields_}

    def close(self):
        if self.handle:
            lib().oracle_lt_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class OracleBidirPathTracer:
    """CPU restatement of the bidirectional path tracer (cpu_bpt.cpp): per pixel and iteration one light
    subpath and one view subpath, all connections and emitter hits weighted by the balance heuristic."""

    TARGETS = {"Radiance": (0, 3), "Lightness": (1, 1)}

    def __init__(self, scene: OracleScene, seed=0, min_path=0, max_path=16):
        self.scene = scene
        self.max_path = max(1, max_path)
        p = OrLtParams(seed, min_path, max_path, 0)
        self.handle = lib().oracle_bpt_create(scene.handle, C.byref(p))
        if not self.handle:
            raise ValueError("oracle_bpt_create failed")

    def iterate(self, threads: int = 0):
        if threads <= 0:
            threads = os.cpu_count() or 1
        lib().oracle_bpt_iterate(self.handle, threads)

    def target(self, name: str, variance: bool = False):
        """Cumulative target, or with variance=True its running variance."""
        w, h = self.scene.spec.width, self.scene.spec.height
        idx, ch = self.TARGETS[name]
        out = np.zeros((h, w, ch), np.float32)
        lib().oracle_bpt_get_target(self.handle, idx + (2 if variance else 0), _ptr(out))
        return out

    def records(self):
        """The last iteration's contributions per pixel: M*M connection slots [view length][light vertex]
        then M emitter-hit slots (M = max. path length); pixel index (-1: none) and (radiance rgb,
        lightness) as added."""
        m = self.max_path
        n = self.scene.spec.width * self.scene.spec.height * (m * m + m)
        pix = np.zeros(n, np.int32)
        val = np.zeros((n, 4), np.float32)
        if not lib().oracle_bpt_records(self.handle, _ptr(pix), _ptr(val)):
            raise RuntimeError("no iteration has run")
        return pix, val

    def stats(self):
        s = OrStats()
        lib().oracle_bpt_stats(self.handle, C.byref(s))
        return {k: getattr(s, k) for k, _ in OrStats._fields_}

    def close(self):
        if self.handle:
            lib().oracle_bpt_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class OracleWireframe:
    """CPU restatement of the wireframe renderer (wireframe_common.hpp, cpu_wireframe.cpp)."""

    def __init__(self, scene: OracleScene, line_width=1.0, max_trace_depth=1000):
        self.scene = scene
        self.handle = lib().oracle_wireframe_create(scene.handle, float(line_width), int(max_trace_depth))

    def iterate(self, threads: int = 0):
        lib().oracle_wireframe_iterate(self.handle, threads if threads > 0 else (os.cpu_count() or 1))

    def target(self, variance: bool = False):
        w, h = self.scene.spec.width, self.scene.spec.height
        out = np.zeros((h, w, 3), np.float32)
        (lib().oracle_wireframe_get_variance if variance else lib().oracle_wireframe_get_target)(self.handle, _ptr(out))
        return out

    def close(self):
        if self.handle:
            lib().oracle_wireframe_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class OracleVcm:
    """CPU restatement of vertex connection and merging (cpu_vcm.cpp): per pixel and iteration one light
    subpath (all stored as photons in a hash grid) and one view subpath whose vertices connect to one
    light subpath, count emitter hits and merge with the photons within the merge radius."""

    TARGETS = {"Radiance": (0, 3), "Lightness": (1, 1)}

    def __init__(self, scene: OracleScene, seed=0, min_path=0, max_path=16, merge_radius=0.001, progressive=False):
        self.scene = scene
        self.max_path = max(1, max_path)
        p = OrLtParams(seed, min_path, max_path, 0)
        self.handle = lib().oracle_vcm_create(scene.handle, C.byref(p), float(merge_radius), int(progressive))
        if not self.handle:
            raise ValueError("oracle_vcm_create failed")

    def iterate(self, threads: int = 0):
        if threads <= 0:
            threads = os.cpu_count() or 1
        lib().oracle_vcm_iterate(self.handle, threads)

    def target(self, name: str, variance: bool = False):
        w, h = self.scene.spec.width, self.scene.spec.height
        idx, ch = self.TARGETS[name]
        out = np.zeros((h, w, ch), np.float32)
        lib().oracle_vcm_get_target(self.handle, idx + (2 if variance else 0), _ptr(out))
        return out

    def records(self):
        """The last iteration's contributions per pixel: M*M connection slots [view length][light vertex],
        M emitter-hit slots and M merge slots [view length - 1] (M = max. path length); pixel index (-1:
        none) and (radiance rgb, lightness) as added."""
        m = self.max_path
        n = self.scene.spec.width * self.scene.spec.height * (m * m + 2 * m)
        pix = np.zeros(n, np.int32)
        val = np.zeros((n, 4), np.float32)
        if not lib().oracle_vcm_records(self.handle, _ptr(pix), _ptr(val)):
            raise RuntimeError("no iteration has run")
        return pix, val

    def stats(self):
        s = OrStats()
        lib().oracle_vcm_stats(self.handle, C.byref(s))
        return {k: getattr(s, k) for k, _ in OrStats._fields_}

    def close(self):
        if self.handle:
            lib().oracle_vcm_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def vcm_map_size(capacity: int) -> int:
    return int(lib().oracle_vcm_map_size(capacity))


def wang_hash(x: int) -> int:
    return int(lib().oracle_wang_hash(x))
