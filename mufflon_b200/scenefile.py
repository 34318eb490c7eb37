"""Writer of Mufflon scene files: a JSON scene description plus its binary
geometry file (*.mff), in the layout of doc/FileFormat.md that
libmufflon_loader.so (loader_load_json) reads.

`write_scene(spec, path)` turns a SceneSpec into such a pair. The world the
loader builds from the files is the one `bindings.load_scene_spec` builds from
the spec it returns (bit for bit: the returned spec carries the camera's field
of view as the loader computes it from degrees, and quantised normals when
`compressed_normals` is set), so renders of both can be compared exactly.

`write_mff` / `write_json` are the lower-level pieces for files with several
LoDs per object, named instances, scenarios with LoD overrides and masks.
"""
from __future__ import annotations

import dataclasses
import json
import math
import os
import struct
import zlib
from typing import Dict, List, Optional, Sequence

import numpy as np

MAGIC = {k: struct.unpack("<I", k.encode())[0] for k in ("Mats", "Bone", "Objs", "Obj_", "LOD_", "Attr", "Inst")}
DEFLATE = 1
COMPRESSED_NORMALS = 2
NO_FRAME = 0xFFFFFFFF
FILE_VERSION = "1.7"


def pack_normal32(n: np.ndarray) -> np.ndarray:
    """Octahedral packing of unit normals (V, 3) into uint32 (doc/FileFormat.md packNormal32)."""
    n = np.asarray(n, np.float64)
    l1 = np.abs(n).sum(1)
    l1 = np.where(l1 > 0, l1, 1.0)
    up = n[:, 2] >= 0
    u = np.where(up, n[:, 0] / l1, (1 - np.abs(n[:, 1]) / l1) * np.where(n[:, 0] >= 0, 1.0, -1.0))
    v = np.where(up, n[:, 1] / l1, (1 - np.abs(n[:, 0]) / l1) * np.where(n[:, 1] >= 0, 1.0, -1.0))
    ui = np.floor(u * 32767.0 + 0.5).astype(np.int64) & 0xFFFF
    vi = np.floor(v * 32767.0 + 0.5).astype(np.int64) & 0xFFFF
    return (ui | (vi << 16)).astype(np.uint32)


def unpack_normal32(p: np.ndarray) -> np.ndarray:
    """Inverse of pack_normal32, normalised, in float32 with the loader's
    operation order (so the result equals the loader's bit for bit)."""
    p = np.asarray(p, np.uint32)
    f32 = np.float32
    u = (p & 0xFFFF).astype(np.uint16).view(np.int16).astype(f32) / f32(32767.0)
    v = (p >> 16).astype(np.uint16).view(np.int16).astype(f32) / f32(32767.0)
    z = (f32(1.0) - np.abs(u)) - np.abs(v)
    low = z < 0
    x = np.where(low, (f32(1.0) - np.abs(v)) * np.where(u >= 0, f32(1.0), f32(-1.0)), u).astype(f32)
    y = np.where(low, (f32(1.0) - np.abs(u)) * np.where(v >= 0, f32(1.0), f32(-1.0)), v).astype(f32)
    length = np.sqrt((x * x + y * y) + z * z).astype(f32)
    return np.stack([x / length, y / length, z / length], 1).astype(f32)


def loaded_fov(degrees: float) -> float:
    """The vertical field of view in radians that the loader derives from `degrees`."""
    return float(np.float32(degrees) * (np.float32(math.pi) / np.float32(180.0)))


# ---------------------------------------------------------------- binary file
@dataclasses.dataclass
class MffObject:
    name: str
    lods: list                      # LodSpec per level (0: most detailed)
    flags: int = 0
    keyframe: int = NO_FRAME
    prev_anim_object: int = NO_FRAME


@dataclasses.dataclass
class MffInstance:
    name: str
    object: int
    transform: np.ndarray           # 12 float32, world-to-instance (file version >= 1.4)
    keyframe: int = NO_FRAME
    prev_anim_instance: int = NO_FRAME


def _string(s: str) -> bytes:
    b = s.encode("utf-8")
    return struct.pack("<I", len(b)) + b


def _block(data: bytes, deflate: bool) -> bytes:
    if not deflate:
        return data
    c = zlib.compress(data, 6)
    return struct.pack("<II", len(c), len(data)) + c


def _attributes(attrs, deflate: bool) -> bytes:
    """<ATTRIBUTE> list: (name, meta, flags, type, bytes) tuples."""
    body = b"".join(_string(n) + _string(m) + struct.pack("<IIQ", f, t, len(d)) + d for n, m, f, t, d in attrs)
    return struct.pack("<I", MAGIC["Attr"]) + _block(body, deflate)


def _lod_bytes(lod, flags: int, attributes: Optional[dict] = None) -> bytes:
    deflate = bool(flags & DEFLATE)
    attributes = attributes or {}
    V, T, Q, S = len(lod.vertices), len(lod.triangles), len(lod.quads), len(lod.spheres)
    va, fa, sa = attributes.get("vertex", []), attributes.get("face", []), attributes.get("sphere", [])
    out = [struct.pack("<9I", MAGIC["LOD_"], T, Q, S, V, 0, len(va), len(fa), len(sa))]
    if V:
        pos = np.ascontiguousarray(lod.vertices, "<f4").tobytes()
        if flags & COMPRESSED_NORMALS:
            nrm = pack_normal32(lod.normals).astype("<u4").tobytes()
        else:
            nrm = np.ascontiguousarray(lod.normals, "<f4").tobytes()
        uvs = np.ascontiguousarray(lod.uvs, "<f4").tobytes()
        out.append(_block(pos + nrm + uvs, deflate))
        if va:
            out.append(_attributes(va, deflate))
    if T:
        out.append(_block(np.ascontiguousarray(lod.triangles, "<u4").reshape(-1).tobytes(), deflate))
    if Q:
        out.append(_block(np.ascontiguousarray(lod.quads, "<u4").reshape(-1).tobytes(), deflate))
    if T + Q:
        out.append(_block(np.ascontiguousarray(lod.face_materials, "<u2").tobytes(), deflate))
        if fa:
            out.append(_attributes(fa, deflate))
    if S:
        sph = np.ascontiguousarray(lod.spheres, "<f4").tobytes() + np.ascontiguousarray(lod.sphere_materials, "<u2").tobytes()
        out.append(_block(sph, deflate))
        if sa:
            out.append(_attributes(sa, deflate))
    return b"".join(out)


def _aabb(lods) -> tuple:
    pts = []
    for lod in lods:
        if len(lod.vertices):
            pts.append(np.asarray(lod.vertices, np.float32))
        if len(lod.spheres):
            s = np.asarray(lod.spheres, np.float32)
            pts += [s[:, :3] - s[:, 3:], s[:, :3] + s[:, 3:]]
    if not pts:
        return (0.0, 0.0, 0.0), (0.0, 0.0, 0.0)
    p = np.concatenate(pts)
    return tuple(float(x) for x in p.min(0)), tuple(float(x) for x in p.max(0))


def write_mff(path: str, materials: Sequence[str], objects: Sequence[MffObject], instances: Sequence[MffInstance],
              flags: int = 0, unique_materials: bool = True, bones: Optional[tuple] = None,
              attributes: Optional[Dict[int, dict]] = None) -> None:
    """Writes a binary geometry file. `materials` are the binary material
    names (index = material index of faces and spheres). `bones` = (numBones,
    numFrames) adds a 'Bone' section of identity transforms. `attributes`
    maps an object index to {"vertex"|"face"|"sphere": [(name, meta, flags,
    type, bytes), ...]} written into each of its LoDs."""
    mats = struct.pack("<I", len(materials)) + b"".join(_string(m) for m in materials)
    head = bytearray()
    head += struct.pack("<IQ", MAGIC["Mats"], 0) + mats
    struct.pack_into("<Q", head, 4, len(head))
    if bones is not None:
        nb, nf = bones
        start = len(head)
        dq = np.tile(np.array([0, 0, 0, 1, 0, 0, 0, 0], "<f4"), nb * nf).tobytes()
        sec = bytearray(struct.pack("<IQII", MAGIC["Bone"], 0, nb, nf) + dq)
        struct.pack_into("<Q", sec, 4, start + len(sec))
        head += sec
    objs_start = len(head)
    # objects: header, jump table, then each object with its LoDs
    obj_blobs = []
    for oi, o in enumerate(objects):
        lods = [_lod_bytes(l, flags, (attributes or {}).get(oi)) for l in o.lods]
        mn, mx = _aabb(o.lods)
        prefix = struct.pack("<I", MAGIC["Obj_"]) + _string(o.name) + struct.pack("<III6f", o.flags, o.keyframe,
                                                                                   o.prev_anim_object, *mn, *mx)
        uniq = b""
        if unique_materials:
            ids = sorted({int(m) for l in o.lods for m in np.concatenate([np.asarray(l.face_materials, np.int64).reshape(-1),
                                                                          np.asarray(l.sphere_materials, np.int64).reshape(-1)])})
            uniq = struct.pack("<I", len(ids)) + struct.pack(f"<{len(ids)}H", *ids)
        obj_blobs.append((prefix, uniq, lods))
    table_len = 4 + 8 + 4 + 4 + 8 * len(objects)
    pos = objs_start + table_len
    offsets, body = [], bytearray()
    for prefix, uniq, lods in obj_blobs:
        offsets.append(pos)
        jt_len = 4 + 8 * len(lods)
        lod_pos = pos + len(prefix) + jt_len + len(uniq)
        lod_offs = []
        for lb in lods:
            lod_offs.append(lod_pos)
            lod_pos += len(lb)
        blob = prefix + struct.pack(f"<I{len(lods)}Q", len(lods), *lod_offs) + uniq + b"".join(lods)
        body += blob
        pos += len(blob)
    inst_start = pos
    objs = struct.pack("<IQII", MAGIC["Objs"], inst_start, flags, len(objects)) + struct.pack(f"<{len(objects)}Q", *offsets)
    inst = bytearray(struct.pack("<II", MAGIC["Inst"], len(instances)))
    for i in instances:
        inst += _string(i.name) + struct.pack("<III", i.object, i.keyframe, i.prev_anim_instance)
        inst += np.asarray(i.transform, "<f4").reshape(12).tobytes()
    with open(path, "wb") as f:
        f.write(bytes(head) + objs + bytes(body) + bytes(inst))


# ---------------------------------------------------------------- JSON file
def _floats(x) -> list:
    return [float(v) for v in np.asarray(x, np.float64).reshape(-1)]


def write_pfm(path: str, rgb: np.ndarray) -> None:
    """RGB float image (H, W, >=3) as a little-endian PFM, rows as given."""
    a = np.ascontiguousarray(np.asarray(rgb, np.float32)[..., :3], "<f4")
    with open(path, "wb") as f:
        f.write(f"PF\n{a.shape[1]} {a.shape[0]}\n-1.0\n".encode())
        f.write(a.tobytes())


def material_json(m, texture_file: Optional[str] = None, alpha_file: Optional[str] = None) -> dict:
    """JSON material of a MaterialSpec (types 0 Lambert, 1 Torrance GGX/Smith, 2 emissive), with its
    alpha texture file if it has one."""
    if m.type == 0:
        out = {"type": "lambert", "albedo": texture_file or _floats(m.albedo)}
    elif m.type == 1:
        out = {"type": "torrance", "ndf": "GGX", "shadowingModel": "smith" if m.shadowing == 1 else "vcavity",
               "roughness": _floats(m.roughness),
               "albedo": texture_file or _floats(m.albedo)}
    else:
        return {"type": "emissive", "radiance": _floats(m.radiance), "scale": _floats(m.scale)}
    if alpha_file:
        out["alpha"] = alpha_file
    return out


def write_json(path: str, document: dict) -> None:
    with open(path, "w") as f:
        json.dump(document, f, indent=1)


def write_scene(spec, json_path: str, *, deflate: bool = False, compressed_normals: bool = False,
                version: str = FILE_VERSION, scenario: str = None, binary_name: str = None):
    """Writes `spec` as `json_path` plus its binary file (and PFM files for
    textures) and returns the spec the loaded world equals (see the module
    docstring). Masked instances (instance_lod 0xFFFFFFFF) become instances of
    object 0 masked by the scenario."""
    if spec.background is not None and tuple(float(x) for x in spec.background[1]) != (1.0, 1.0, 1.0):
        raise ValueError("a monochrome background of the file format has no separate scale")
    base = os.path.splitext(json_path)[0]
    directory = os.path.dirname(os.path.abspath(json_path))
    binary_name = binary_name or os.path.basename(base) + ".mff"
    flags = (DEFLATE if deflate else 0) | (COMPRESSED_NORMALS if compressed_normals else 0)
    lods = list(spec.lods)
    if compressed_normals:
        lods = [dataclasses.replace(l, normals=unpack_normal32(pack_normal32(l.normals)) if len(l.normals) else l.normals)
                for l in lods]
    mat_names = [f"mat{i}" for i in range(len(spec.materials))]
    objects = [MffObject(f"obj{i}_{l.name}", [l]) for i, l in enumerate(spec.lods)]
    instances, masked = [], []
    for i, li in enumerate(np.asarray(spec.instance_lod, np.uint32)):
        if int(li) == 0xFFFFFFFF:
            masked.append(f"inst{i}")
            li = 0
        instances.append(MffInstance(f"inst{i}", int(li), np.asarray(spec.world_to_instance[i], np.float32)))
    write_mff(os.path.join(directory, binary_name), mat_names, objects, instances, flags)
    tex_files = {}
    for k, tex in enumerate(spec.textures):
        name = f"{os.path.basename(base)}_tex{k}.pfm"
        write_pfm(os.path.join(directory, name), tex)
        tex_files[k] = name
    materials = {mat_names[i]: material_json(m, tex_files.get(m.albedo_texture) if m.albedo_texture >= 0 else None,
                                             tex_files.get(getattr(m, "alpha_texture", -1)))
                 for i, m in enumerate(spec.materials)}
    deg = math.degrees(spec.vfov)
    lights = {f"point{k}": {"type": "point", "position": _floats(pl[:3]), "intensity": _floats(pl[3:])}
              for k, pl in enumerate(np.asarray(spec.point_lights, np.float32).reshape(-1, 6))}
    if spec.background is not None:
        lights["background"] = {"type": "envmap", "scale": _floats(spec.background[0])}
    scen = scenario or spec.name
    doc = {
        "version": version,
        "binary": binary_name,
        "defaultScenario": scen,
        "noDefaultInstances": any(o not in {i.object for i in instances} for o in range(len(objects))),
        "cameras": {"camera": {"type": "pinhole", "path": [_floats(spec.cam_pos)], "viewDir": [_floats(spec.cam_dir)],
                               "up": [_floats(spec.cam_up)], "fov": deg}},
        "lights": lights,
        "materials": materials,
        "scenarios": {scen: {
            "camera": "camera", "resolution": [int(spec.width), int(spec.height)], "lights": list(lights),
            "materialAssignments": {n: n for n in mat_names},
            "instanceProperties": {n: {"mask": True} for n in masked},
        }},
    }
    write_json(json_path, doc)
    return dataclasses.replace(spec, lods=lods, vfov=loaded_fov(deg))
