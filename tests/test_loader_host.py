"""The scene-file loader's control flow on the CPU: libmufflon_loader.so's
sources linked against a host-only fake of the core's world API
(tests/cpp/fake_core.cpp), built with AddressSanitizer and UBSan. Checks the
world the loader builds from a file, scenario settings, on-demand LoDs, and
every failure case of the GPU tests (tests/scenefile_cases.py) without a GPU."""
import json
import os
import subprocess

import numpy as np
import pytest

from mufflon_b200 import scenefile, scenes
from tests import scenefile_cases as cases

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LOADER = os.path.join(ROOT, "mufflon_b200", "csrc", "loader")


@pytest.fixture(scope="session")
def harness(tmp_path_factory):
    exe = str(tmp_path_factory.mktemp("harness") / "loader_harness")
    srcs = [os.path.join(LOADER, f) for f in ("json.cpp", "mff_binary.cpp", "scene_loader.cpp", "interface.cpp")]
    srcs += [os.path.join(ROOT, "tests", "cpp", f) for f in ("fake_core.cpp", "loader_harness.cpp")]
    cmd = ["g++", "-O1", "-g", "-std=c++17", "-ffp-contract=off", "-fno-fast-math", "-Wall",
           "-fsanitize=address,undefined", "-fno-sanitize-recover=all", "-fno-omit-frame-pointer"] + srcs + ["-lz", "-o", exe]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr

    def run(path, scenario=None):
        args = [exe, str(path)] + ([scenario] if scenario else [])
        env = dict(os.environ, ASAN_OPTIONS="detect_leaks=1:abort_on_error=0", UBSAN_OPTIONS="print_stacktrace=1")
        r = subprocess.run(args, capture_output=True, text=True, env=env, timeout=120)
        assert r.returncode == 0 and "Sanitizer" not in r.stderr and "runtime error" not in r.stderr, r.stderr[-4000:]
        return json.loads(r.stdout)
    return run


def bits(a):
    return np.asarray(a, np.float32).reshape(-1).view(np.uint32).tolist()


@pytest.mark.parametrize("deflate,packed", [(False, False), (True, True)])
def test_world_from_a_file(tmp_path, harness, deflate, packed):
    spec = scenes.instanced_scene(4, num_meshes=2, num_instances=6, num_spheres=5, tri_range=(100, 300),
                                  width=32, height=24)
    jp = tmp_path / "s.json"
    loaded = scenefile.write_scene(spec, str(jp), deflate=deflate, compressed_normals=packed)
    out = harness(jp)
    assert out["status"] == 0, out["error"]
    w = out["world"]
    assert [o["name"] for o in w["objects"]] == [f"obj{i}_{l.name}" for i, l in enumerate(spec.lods)]
    used = {int(x) for x in spec.instance_lod}
    for k, (o, lod) in enumerate(zip(w["objects"], loaded.lods)):
        assert o["slots"] == 1
        if k not in used:  # no instance: its geometry is never requested
            assert o["lods"] == {}
            continue
        assert list(o["lods"]) == ["0"]
        L = o["lods"]["0"]
        assert L["v"] == bits(lod.vertices) and L["n"] == bits(lod.normals)
        assert (L["tri"], L["quad"], L["sph"]) == (len(lod.triangles), len(lod.quads), len(lod.spheres))
    assert [i["object"] for i in w["instances"]] == [int(x) for x in spec.instance_lod]
    assert [i["w2i"] for i in w["instances"]] == [bits(m) for m in spec.world_to_instance]
    assert all(i["frame"] == 0xFFFFFFFF for i in w["instances"])
    (cam,) = w["cameras"]
    assert cam["fov"] == bits([loaded.vfov])[0]
    assert cam["near"] == bits([0.01])[0] and cam["far"] == bits([500.0])[0]
    (sc,) = w["scenarios"]
    assert sc["name"] == spec.name and sc["res"] == [32, 24] and sc["lod"] == 0
    assert sc["slots"] == [[f"mat{i}", f"mat{i}"] for i in range(len(spec.materials))]
    types = {0: 1, 1: 3, 2: 0}  # MaterialSpec type -> MaterialParamType
    assert [m[1] for m in w["materials"]] == [types[m.type] for m in spec.materials]
    (pl, bg) = w["lights"]
    assert pl["a"] == bits(spec.point_lights[0][:3]) and pl["b"] == bits(spec.point_lights[0][3:])
    assert bg["kind"] == 1 and bg["a"] == bits(spec.background[0])
    assert w["loaded"] == [spec.name]
    assert out["abortIdle"] == 0 and out["warnings"] == ""


def test_scenarios_and_on_demand_lods(tmp_path, harness):
    cases.lod_scene(tmp_path)
    out = harness(tmp_path / "lods.json")
    assert out["status"] == 0, out["error"]
    w = out["world"]
    A, B, C = w["objects"]
    assert (A["slots"], B["slots"], C["slots"]) == (2, 1, 1)
    assert list(A["lods"]) == ["0"]  # the default scenario needs the fine LoD only
    sc = {s["name"]: s for s in w["scenarios"]}
    assert list(sc) == ["fine", "coarse", "mixed", "objlod", "masked"]
    assert sc["coarse"]["lod"] == 1 and sc["fine"]["lod"] == 0
    # "mixed" inherits camera, lights and materials from "fine"
    assert sc["mixed"]["camera"] == "cam" and sc["mixed"]["lights"] == sc["fine"]["lights"]
    assert sc["mixed"]["instanceLods"] == {"1": 1} and sc["mixed"]["maskedObjects"] == [2]
    assert sc["objlod"]["objectLods"] == {"0": 1} and sc["objlod"]["instanceLods"] == {"0": 0}
    assert sc["masked"]["maskedInstances"] == [2]  # "unknown" names no instance and is skipped
    for name, lods in [("coarse", ["0", "1"]), ("masked", ["0", "1"]), ("fine", ["0"])]:
        out = harness(tmp_path / "lods.json", name)
        assert out["switched"], out["error"]
        assert list(out["world"]["objects"][0]["lods"]) == lods, name


def test_failure_cases(tmp_path, harness):
    good = None
    for path, needles in cases.failure_files(tmp_path):
        out = harness(path)
        if needles is None:
            good = path
            assert out["status"] == 0, out["error"]
        elif isinstance(needles, list):
            assert out["status"] == 0, out["error"]
            for n in needles:
                assert n in out["warnings"], (n, out["warnings"])
        else:
            assert out["status"] == 1, (path, out)
            for n in needles:
                assert n in out["error"], (n, out["error"])
    assert good is not None


def test_old_version_defaults(tmp_path, harness):
    """Before version 1.5 camera planes default to fractions of the scene diagonal."""
    spec = scenes.cornell_box(1, 16, 16)
    jp = tmp_path / "c.json"
    scenefile.write_scene(spec, str(jp))
    doc = json.loads(jp.read_text())
    doc["version"] = "1.4"
    scenefile.write_json(str(jp), doc)
    out = harness(jp)
    assert out["status"] == 0, out["error"]
    (cam,) = out["world"]["cameras"]
    near = np.array([cam["near"]], np.uint32).view(np.float32)[0]
    far = np.array([cam["far"]], np.uint32).view(np.float32)[0]
    assert near != np.float32(0.01) and far / near == pytest.approx(2e4, rel=1e-5)
    del doc["version"]
    scenefile.write_json(str(jp), doc)
    out = harness(jp)
    assert out["status"] == 0 and "no version" in out["warnings"]
