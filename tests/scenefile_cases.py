"""Scene-file cases shared by the loader tests on the GPU (test_gpu_loader.py)
and on the CPU against a host-only fake core (test_loader_host.py)."""
import dataclasses
import json

import numpy as np

from mufflon_b200 import scenefile, scenes


def lod_scene(tmp_path):
    """Object A with two LoDs (fine, coarse icosphere), a ground quad B and a
    sphere cloud C; instances a0, a1 (of A), b, c; five scenarios."""
    def ico(sub, seed):
        v, f = scenes.displaced_sphere_mesh(sub, seed)
        return scenes._lod(v, scenes.vertex_normals(v, f), scenes.spherical_uv(v), tris=f.astype(np.uint32),
                           mats=np.zeros(len(f), np.uint16), name="A")
    a_fine, a_coarse = ico(4, 1), ico(1, 1)
    gp, gn = scenes._quad((-6, -1.2, -6), (-6, -1.2, 6), (6, -1.2, 6), (6, -1.2, -6))
    ground = scenes._lod(gp, gn, np.array([(0, 0), (1, 0), (1, 1), (0, 1)], np.float32),
                         quads=np.arange(4, dtype=np.uint32).reshape(1, 4), mats=np.array([1], np.uint16), name="B")
    rng = np.random.default_rng(5)
    sph = np.concatenate([rng.uniform(-3, 3, (40, 3)), rng.uniform(0.05, 0.25, (40, 1))], 1).astype(np.float32)
    cloud = scenes._lod(np.zeros((0, 3)), np.zeros((0, 3)), np.zeros((0, 2)), spheres=sph,
                        sphere_mats=np.full(40, 2, np.uint16), name="C")
    mats = [scenes.MaterialSpec(1, albedo=(0.7, 0.5, 0.3), roughness=(0.3, 0.3)),
            scenes.MaterialSpec(0, albedo=(0.6, 0.6, 0.6)), scenes.MaterialSpec(0, albedo=(0.2, 0.5, 0.8))]
    left = scenes._w2i_from_rt(np.eye(3), np.array([-1.3, 0.0, 0.0]))
    right = scenes._w2i_from_rt(np.eye(3), np.array([1.3, 0.0, 0.0]))
    ident = scenes.identity34()
    base = scenes.SceneSpec([a_fine, ground, cloud], np.array([left, right, ident, ident], np.float32),
                            np.array([0, 0, 1, 2], np.uint32), mats, np.array([[2, 4, 3, 30, 30, 30]], np.float32),
                            ((0.2, 0.25, 0.3), (1.0, 1.0, 1.0)), (0.0, 0.8, 6.0), (0.0, -0.15, -1.0), (0.0, 1.0, 0.0),
                            scenefile.loaded_fov(40.0), 48, 36, name="lods")
    names = ["mat0", "mat1", "mat2"]
    objs = [scenefile.MffObject("A", [a_fine, a_coarse]), scenefile.MffObject("B", [ground]),
            scenefile.MffObject("C", [cloud])]
    insts = [scenefile.MffInstance(n, o, base.world_to_instance[i]) for i, (n, o) in
             enumerate([("a0", 0), ("a1", 0), ("b", 1), ("c", 2)])]
    scenefile.write_mff(str(tmp_path / "lods.mff"), names, objs, insts, flags=scenefile.DEFLATE)
    common = {"camera": "cam", "resolution": [48, 36], "lights": ["sun", "sky"],
              "materialAssignments": {n: n for n in names}}
    doc = {
        "version": "1.7", "binary": "lods.mff", "defaultScenario": "fine",
        "cameras": {"cam": {"type": "pinhole", "path": [list(base.cam_pos)], "viewDir": [list(base.cam_dir)],
                            "up": [[0.0, 1.0, 0.0]], "fov": 40.0}},
        "lights": {"sun": {"type": "point", "position": [2, 4, 3], "intensity": [30, 30, 30]},
                   "sky": {"type": "envmap", "scale": [0.2, 0.25, 0.3]}},
        "materials": {n: scenefile.material_json(m) for n, m in zip(names, mats)},
        "scenarios": {
            "fine": dict(common),
            "coarse": dict(common, lod=1),
            "mixed": {"parentScenario": "fine", "instanceProperties": {"a1": {"lod": 1}},
                      "objectProperties": {"C": {"mask": True}}},
            "objlod": dict(common, objectProperties={"A": {"lod": 1}}, instanceProperties={"a0": {"lod": 0}}),
            "masked": dict(common, lod=1, instanceProperties={"b": {"mask": True}, "unknown": {"mask": True}}),
        },
    }
    scenefile.write_json(str(tmp_path / "lods.json"), doc)
    M = 0xFFFFFFFF
    expect = {  # spec LoD list and the LoD index of each instance a0, a1, b, c
        "fine": ([a_fine, ground, cloud], [0, 0, 1, 2]),
        "coarse": ([a_coarse, ground, cloud], [0, 0, 1, 2]),
        "mixed": ([a_fine, a_coarse, ground], [0, 1, 2, M]),
        "objlod": ([a_fine, a_coarse, ground, cloud], [0, 1, 2, 3]),
        "masked": ([a_coarse, cloud], [0, 0, M, 1]),
    }
    return base, expect


WALTER = {"type": "walter", "ndf": "GGX", "roughness": 0.2, "absorption": [0, 0, 0], "ior": 1.5}


def failure_files(tmp_path):
    """Yields (path, expectation) for scene files that must not load: the
    expectation is a tuple of words the error message contains. One good
    file is yielded with None, and files that load with warnings with a list
    of words the warnings contain."""
    spec = scenes.cornell_box(1, 16, 16)
    good = tmp_path / "good.json"
    scenefile.write_scene(spec, str(good))
    doc = json.loads(good.read_text())
    scen = doc["defaultScenario"]
    yield good, None
    yield tmp_path / "nope.json", ("does not exist",)
    yield tmp_path, ("is a directory",)
    bad = tmp_path / "bad.json"
    bad.write_text('{"version": "1.7",\n "binary": }')
    yield bad, ("JSON parse error", "line 2")

    counter = [0]

    def variant(mutate):
        d = json.loads(json.dumps(doc))
        mutate(d)
        counter[0] += 1
        p = tmp_path / f"variant{counter[0]}.json"
        scenefile.write_json(str(p), d)
        return p

    yield variant(lambda x: x.update(binary="missing.mff")), ("does not exist",)
    yield variant(lambda x: x.pop("cameras")), ("missing 'cameras'",)
    yield variant(lambda x: x.update(defaultScenario="nope")), ("default scenario 'nope'",)
    yield variant(lambda x: x["scenarios"][scen]["materialAssignments"].pop("mat0")), ("missing 'mat0'",)
    yield variant(lambda x: x["scenarios"][scen]["materialAssignments"].update(mat0="nope")), ("unknown material name 'nope'",)
    yield variant(lambda x: x["scenarios"][scen].update(camera="nope")), ("camera 'nope' does not exist",)
    yield variant(lambda x: x["scenarios"][scen].update(resolution=[0, 4])), ("resolution",)
    yield variant(lambda x: x["scenarios"][scen].update(parentScenario=scen)), ("loop in scenario inheritance",)
    yield variant(lambda x: x["scenarios"][scen].update(lod=-1)), ("lod", "non-negative integer")
    yield variant(lambda x: x["cameras"]["camera"].update(path=[[0, 0]])), ("path", "3 numbers")
    # models the CUDA path tracer does not implement: an error when a scenario uses them ...
    yield variant(lambda x: x["materials"].update(mat0=WALTER)), ("mat0", "not implemented")
    yield variant(lambda x: x["materials"]["mat1"].update(type="torrance", ndf="BS", roughness=0.3)), ("GGX",)
    yield variant(lambda x: x["materials"]["mat0"].update(type="blend")), ("factorA",)
    yield variant(lambda x: x["materials"]["mat0"].update(type="glass")), ("'glass' is not supported",)
    yield variant(lambda x: x["materials"]["mat0"].update(alpha=[1, 2, 3])), ("alpha", "texture path")
    yield variant(lambda x: (x["lights"].update(spot={"type": "spot", "position": [0, 1, 0], "direction": [0, -1, 0],
                                                      "intensity": [1, 1, 1], "width": 0.5}),
                            x["scenarios"][scen]["lights"].append("spot"))), ("spot",)
    yield variant(lambda x: (x["lights"].update(env={"type": "envmap", "map": "sky.pfm"}),
                            x["scenarios"][scen]["lights"].append("env"))), ("env",)
    yield variant(lambda x: (x["cameras"].update(lens={"type": "focus", "path": [[0, 0, 5]], "viewDir": [[0, 0, -1]],
                                                       "focusDistance": 5.0}),
                            x["scenarios"][scen].update(camera="lens"))), ("focus",)
    yield variant(lambda x: x["materials"]["mat0"].update(type="emissive", temperature=3000)), ("temperature",)
    yield variant(lambda x: x["materials"]["mat0"].update(albedo="missing.pfm")), ("cannot find texture",)
    (tmp_path / "gray.pfm").write_bytes(b"Pf\n1 1\n-1.0\n" + np.zeros(1, "<f4").tobytes())
    yield variant(lambda x: x["materials"]["mat0"].update(albedo="gray.pfm")), ("single-channel",)
    (tmp_path / "short.pfm").write_bytes(b"PF\n4 4\n-1.0\n" + np.zeros(5, "<f4").tobytes())
    yield variant(lambda x: x["materials"]["mat0"].update(albedo="short.pfm")), ("shorter than",)
    # ... and ignored when unused, or ignored with a warning
    yield variant(lambda x: (x["materials"].update(unused=WALTER),
                             x["lights"].update(g={"type": "goniometric", "position": [0, 1, 0], "map": "x.pfm"}),
                             x["scenarios"][scen]["lights"].append("g"),
                             x["scenarios"][scen]["lights"].append("ghost"),
                             x["cameras"].update(o={"type": "ortho", "path": [0, 0, 1], "viewDir": [0, 0, -1]}),
                             x.update(deinstance=True))), ["goniometric", "ghost", "orthographic", "deinstance"]
    # corrupt binaries
    raw = (tmp_path / doc["binary"]).read_bytes()
    (tmp_path / "trunc.mff").write_bytes(raw[: len(raw) // 2])
    yield variant(lambda x: x.update(binary="trunc.mff")), ("binary file", "end of the file")
    (tmp_path / "magic.mff").write_bytes(b"XXXX" + raw[4:])
    yield variant(lambda x: x.update(binary="magic.mff")), ("magic",)
    scenefile.write_mff(str(tmp_path / "bones.mff"), ["mat0"], [scenefile.MffObject("o", [spec.lods[0]])], [],
                        bones=(2, 1))
    yield variant(lambda x: x.update(binary="bones.mff")), ("skeletal animation",)
    # a face material index beyond the file's material names
    lod = dataclasses.replace(spec.lods[0], face_materials=np.full_like(spec.lods[0].face_materials, 5))
    scenefile.write_mff(str(tmp_path / "mats.mff"), ["mat0", "mat1"], [scenefile.MffObject("o", [lod])], [])
    yield variant(lambda x: (x.update(binary="mats.mff"),
                             x["scenarios"][scen].update(materialAssignments={"mat0": "mat0", "mat1": "mat1"}))), \
        ("exceeds the 2 materials",)
