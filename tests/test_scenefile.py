"""Scene files on the CPU: the writer's layout against doc/FileFormat.md, and
the loader's own JSON parser and binary reader (built from the library's
sources into a small driver, tests/cpp/mff_dump.cpp) against what was written.
Floats are compared as bit patterns."""
import json
import os
import struct
import subprocess
import zlib

import numpy as np
import pytest

from mufflon_b200 import scenefile, scenes

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LOADER = os.path.join(ROOT, "mufflon_b200", "csrc", "loader")


@pytest.fixture(scope="session")
def mff_dump(tmp_path_factory):
    exe = str(tmp_path_factory.mktemp("mff_dump") / "mff_dump")
    # the product's host flags (mufflon_b200/build.py CXX_FLAGS)
    cmd = ["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-fno-fast-math", "-Wall",
           os.path.join(ROOT, "tests", "cpp", "mff_dump.cpp"), os.path.join(LOADER, "json.cpp"),
           os.path.join(LOADER, "mff_binary.cpp"), "-lz", "-o", exe]
    subprocess.run(cmd, check=True, capture_output=True)

    def run(*args):
        r = subprocess.run([exe] + [str(a) for a in args], capture_output=True, text=True)
        assert r.returncode in (0, 2), f"driver crashed ({r.returncode}): {r.stderr}"
        if r.returncode == 2:
            return r.stdout.strip()
        return json.loads(r.stdout)
    return run


def bits(a):
    return np.asarray(a, np.float32).reshape(-1).view(np.uint32).tolist()


# ---------------------------------------------------------------- JSON parser
def test_json_parser_matches_python(tmp_path, mff_dump):
    doc = {"b": [1, -0.0, 2.5e-300, 1e300, 123456789012, -7, 0.1, 3.0, 1.7976931348623157e308],
           "a": {"nested": {"deep": [True, False, None, "x"]}}, "s": "tab\t quote\" slash\\ é ☃ 😀 \u0001",
           "empty": {}, "list": [], "z": 0}
    p = tmp_path / "doc.json"
    p.write_text(json.dumps(doc, indent=2, ensure_ascii=True))
    out = mff_dump("json", p)
    assert out == doc
    assert list(out) == list(doc)  # member order is kept
    p.write_text(json.dumps(doc, ensure_ascii=False))
    assert mff_dump("json", p) == doc


@pytest.mark.parametrize("text,where", [
    ('{"a": [1, 2,]}', "line 1"), ('{"a": 1', "end of input"), ('{"a": "\\q"}', "invalid escape"),
    ('{"a": "\\ud800"}', "surrogate"), ('{"a": 01}', "expected ','"), ('{\n"a": tru}', "line 2"),
    ('{"a": 1} x', "after the document"), ('[' * 300 + ']' * 300, "nesting"), ('{"a": 1e999}', "out of range"),
])
def test_json_parser_errors(tmp_path, mff_dump, text, where):
    p = tmp_path / "bad.json"
    p.write_text(text)
    out = mff_dump("json", p)
    assert isinstance(out, str) and out.startswith("ERROR: JSON parse error") and where in out, out


# ---------------------------------------------------------------- normals
def test_normal_packing_matches_the_loader(mff_dump):
    rng = np.random.default_rng(3)
    n = rng.normal(size=(200, 3))
    n /= np.linalg.norm(n, axis=1, keepdims=True)
    n = np.concatenate([n, np.eye(3), -np.eye(3), [[1, 1, 0], [0, -1, -1]] / np.sqrt(2)])
    packed = scenefile.pack_normal32(n)
    py = scenefile.unpack_normal32(packed)
    cpp = np.array(mff_dump("unpack", *packed.tolist()), np.uint32).view(np.float32)
    assert np.array_equal(bits(py), bits(cpp))
    # 16-bit octahedral quantisation: better than 1e-4 rad
    p64 = py.astype(np.float64)
    angle = np.arctan2(np.linalg.norm(np.cross(p64, n), axis=1), np.sum(p64 * n, 1))
    assert np.max(angle) < 1e-4
    assert np.allclose(np.linalg.norm(py, axis=1), 1.0, atol=1e-6)


# ---------------------------------------------------------------- binary layout
def _parse_header(buf):
    """Independent reading of the section headers (doc/FileFormat.md)."""
    magic, nxt, nmat = struct.unpack_from("<IQI", buf, 0)
    assert magic == scenefile.MAGIC["Mats"]
    pos, names = 16, []
    for _ in range(nmat):
        (n,) = struct.unpack_from("<I", buf, pos)
        names.append(buf[pos + 4:pos + 4 + n].decode())
        pos += 4 + n
    assert pos == nxt
    magic, = struct.unpack_from("<I", buf, nxt)
    if magic == scenefile.MAGIC["Bone"]:
        _, nxt, nb, nf = struct.unpack_from("<IQII", buf, nxt)
        magic, = struct.unpack_from("<I", buf, nxt)
    assert magic == scenefile.MAGIC["Objs"]
    _, inst, flags, nobj = struct.unpack_from("<IQII", buf, nxt)
    jump = struct.unpack_from(f"<{nobj}Q", buf, nxt + 20)
    for off in jump:
        assert struct.unpack_from("<I", buf, off)[0] == scenefile.MAGIC["Obj_"]
    assert struct.unpack_from("<I", buf, inst)[0] == scenefile.MAGIC["Inst"]
    return names, flags, jump, inst


def _scene_specs():
    tex = scenes.smooth_noise_texture(1, 8)
    return {
        "cornell": scenes.cornell_box(1, 16, 16),
        "ico": scenes.displaced_icosphere(1, subdiv=2, width=16, height=9),
        "inst": scenes.instanced_scene(2, num_meshes=2, num_instances=5, num_spheres=7, tri_range=(50, 200),
                                       width=16, height=9),
        "tex": scenes.cornell_box_textured(1, 16, 16, texture=tex),
    }


@pytest.mark.parametrize("deflate", [False, True])
@pytest.mark.parametrize("packed", [False, True])
def test_reader_returns_what_was_written(tmp_path, mff_dump, deflate, packed):
    for name, spec in _scene_specs().items():
        jp = tmp_path / f"{name}_{int(deflate)}{int(packed)}.json"
        loaded = scenefile.write_scene(spec, str(jp), deflate=deflate, compressed_normals=packed)
        doc = json.loads(jp.read_text())
        binp = tmp_path / doc["binary"]
        names, flags, jump, _ = _parse_header(binp.read_bytes())
        assert flags == (1 if deflate else 0) | (2 if packed else 0)
        out = mff_dump("mff", binp)
        assert out["materials"] == names == [f"mat{i}" for i in range(len(spec.materials))]
        assert out["flags"] == flags and out["bones"] == [0, 0]
        assert len(out["objects"]) == len(spec.lods)
        for o, (lod, lod_loaded) in zip(out["objects"], zip(spec.lods, loaded.lods)):
            (L,) = o["lods"]
            V, T, Q, S = len(lod.vertices), len(lod.triangles), len(lod.quads), len(lod.spheres)
            assert L["header"] == [T, Q, S, V, 0, 0, 0, 0]
            assert L["positions"] == bits(lod.vertices)
            assert L["normals"] == bits(lod_loaded.normals)
            if not packed:
                assert L["normals"] == bits(lod.normals)
            assert L["uvs"] == bits(lod.uvs)
            assert L["triangles"] == np.asarray(lod.triangles, np.uint32).reshape(-1).tolist()
            assert L["quads"] == np.asarray(lod.quads, np.uint32).reshape(-1).tolist()
            assert L["faceMaterials"] == np.asarray(lod.face_materials).tolist()
            assert L["spheres"] == bits(lod.spheres)
            assert L["sphereMaterials"] == np.asarray(lod.sphere_materials).tolist()
            used = sorted(set(np.asarray(lod.face_materials).tolist()) | set(np.asarray(lod.sphere_materials).tolist()))
            assert o["unique"] == used
        assert len(out["instances"]) == len(spec.instance_lod)
        for k, inst in enumerate(out["instances"]):
            assert inst["name"] == f"inst{k}" and inst["keyframe"] == 0xFFFFFFFF
            li = int(spec.instance_lod[k])
            assert inst["object"] == (0 if li == 0xFFFFFFFF else li)
            assert inst["transform"] == bits(spec.world_to_instance[k])
        # the JSON side
        assert doc["version"] == "1.7" and doc["defaultScenario"] == spec.name
        cam = doc["cameras"]["camera"]
        assert cam["type"] == "pinhole"
        assert loaded.vfov == pytest.approx(spec.vfov, rel=1e-6)


def test_attributes_and_bones_are_skipped(tmp_path, mff_dump):
    spec = scenes.instanced_scene(2, num_meshes=2, num_instances=3, num_spheres=4, tri_range=(50, 100), width=8, height=8)
    objs = [scenefile.MffObject(f"o{i}", [l]) for i, l in enumerate(spec.lods)]
    insts = [scenefile.MffInstance(f"i{k}", int(li), spec.world_to_instance[k]) for k, li in enumerate(spec.instance_lod)]
    attrs = {}
    for i, l in enumerate(spec.lods):
        a = {}
        if len(l.vertices):
            a["vertex"] = [("AdditionalUV2D", "AdditionalUV2D", 0, 16, np.zeros((len(l.vertices), 2), "<f4").tobytes()),
                           ("Color", "Color", 0, 17, np.ones((len(l.vertices), 3), "<f4").tobytes())]
        if len(l.triangles) + len(l.quads):
            a["face"] = [("FaceId", "", 0, 5, np.arange(len(l.triangles) + len(l.quads), dtype="<u4").tobytes())]
        if len(l.spheres):
            a["sphere"] = [("Tag", "meta", 7, 1, bytes(len(l.spheres)))]
        attrs[i] = a
    for deflate in (0, 1):
        p = tmp_path / f"attr{deflate}.mff"
        scenefile.write_mff(str(p), ["a", "b", "c"], objs, insts, flags=deflate, bones=(2, 3), attributes=attrs)
        out = mff_dump("mff", p)
        assert out["bones"] == [2, 3]
        for o, l in zip(out["objects"], spec.lods):
            assert o["lods"][0]["positions"] == bits(l.vertices)
            assert o["lods"][0]["spheres"] == bits(l.spheres)
            assert o["lods"][0]["faceMaterials"] == np.asarray(l.face_materials).tolist()
        assert [i["object"] for i in out["instances"]] == [int(x) for x in spec.instance_lod]


def _small_file(tmp_path, deflate):
    spec = scenes.cornell_box(1, 8, 8)
    p = tmp_path / f"small{deflate}.json"
    scenefile.write_scene(spec, str(p), deflate=bool(deflate))
    return tmp_path / json.loads(p.read_text())["binary"]


@pytest.mark.parametrize("deflate", [0, 1])
def test_truncated_files_fail_cleanly(tmp_path, mff_dump, deflate):
    """Every prefix of a valid file either reads (the cut is past the data the
    reader needs) or fails with a message; the driver never crashes."""
    good = _small_file(tmp_path, deflate).read_bytes()
    cut = tmp_path / "cut.mff"
    failures = 0
    for n in list(range(0, 64)) + list(range(64, len(good), 23)):
        cut.write_bytes(good[:n])
        out = mff_dump("mff", cut)
        if isinstance(out, str):
            assert out.startswith("ERROR: "), out
            failures += 1
    assert failures > 0


def test_corrupt_fields_fail_cleanly(tmp_path, mff_dump):
    src = _small_file(tmp_path, 0)
    good = bytearray(src.read_bytes())
    names, flags, jump, inst = _parse_header(bytes(good))

    def run_with(mutate, expect):
        b = bytearray(good)
        mutate(b)
        p = tmp_path / "bad.mff"
        p.write_bytes(bytes(b))
        out = mff_dump("mff", p)
        assert isinstance(out, str) and expect in out, out

    run_with(lambda b: struct.pack_into("<I", b, 0, 0x12345678), "materials header magic")
    run_with(lambda b: struct.pack_into("<I", b, jump[0], 0), "object magic")
    run_with(lambda b: struct.pack_into("<I", b, inst, 0), "instance magic")
    run_with(lambda b: struct.pack_into("<Q", b, 4, len(good) + 100), "beyond the end")
    # a LoD's vertex count far beyond the file
    o = jump[0]
    (nlen,) = struct.unpack_from("<I", good, o + 4)
    jt = o + 8 + nlen + 36
    (lod_off,) = struct.unpack_from("<Q", good, jt + 4)
    run_with(lambda b: struct.pack_into("<I", b, lod_off + 16, 0x7FFFFFFF), "past the end")
    run_with(lambda b: struct.pack_into("<I", b, lod_off, 0), "LoD magic")
    # a face material beyond the material table
    out = mff_dump("mff", src)
    (L,) = out["objects"][0]["lods"]
    T, Q, S, V = L["header"][:4]
    mat_off = lod_off + 36 + V * 32 + T * 12 + Q * 16
    run_with(lambda b: struct.pack_into("<H", b, mat_off, 999), "exceeds the")
    # an instance naming an object that does not exist
    (inl,) = struct.unpack_from("<I", good, inst + 8)
    run_with(lambda b: struct.pack_into("<I", b, inst + 12 + inl, 77), "names object")


def test_deflate_block_sizes_are_checked(tmp_path, mff_dump):
    src = _small_file(tmp_path, 1)
    good = bytearray(src.read_bytes())
    names, flags, jump, inst = _parse_header(bytes(good))
    o = jump[0]
    (nlen,) = struct.unpack_from("<I", good, o + 4)
    (lod_off,) = struct.unpack_from("<Q", good, o + 8 + nlen + 36 + 4)
    blk = lod_off + 36
    packed, unpacked = struct.unpack_from("<II", good, blk)
    assert zlib.decompress(bytes(good[blk + 8:blk + 8 + packed])).__len__() == unpacked
    for field, val, expect in [(4, unpacked + 4, "expected"), (0, packed - 3, "inflate"),
                               (4, 0xFFFFFFF0, "expected")]:
        b = bytearray(good)
        struct.pack_into("<I", b, blk + field, val)
        p = tmp_path / "badz.mff"
        p.write_bytes(bytes(b))
        out = mff_dump("mff", p)
        assert isinstance(out, str) and out.startswith("ERROR"), out
