"""Scene-file import on the GPU (libmufflon_loader.so through its C ABI).

A scene written to JSON + binary and loaded with loader_load_json must give
the same world as the same scene built through the world API
(bindings.load_scene_spec): identical images and hit ids, bit for bit, for
uncompressed, DEFLATE and packed-normal files. Scenario features (global,
per-object and per-instance LoD, masks, parent scenarios) are checked the
same way against equivalent specs, LoDs must arrive on demand through the
core's LoD-loader callback, and broken or unsupported files must fail with a
message and leave the instance usable."""
import dataclasses
import json
import os
import subprocess

import numpy as np
import pytest

from mufflon_b200 import bindings, scenefile, scenes
from tests import scenefile_cases as cases

pytestmark = pytest.mark.gpu

PARAMS = {"Seed": 3, "Max. path length": 6, "Min. path length": 0, "NEE count": 1, "RR start depth": 2}
ITER = 3


def _render(d, iterations=ITER, hit=True):
    assert d.render_enable_renderer(0, 0)
    for k, v in PARAMS.items():
        assert d.renderer_set_parameter_int(k, v)
    d.render_enable_render_target("Radiance", False)
    if hit:
        d.render_enable_render_target("Hit ID", False)
    d.render_reset()
    for _ in range(iterations):
        d.render_iterate()
    img = d.get_target_image("Radiance").copy()
    hid = d.get_target_image("Hit ID").copy() if hit else None
    return img, hid


def _render_spec(spec, iterations=ITER):
    d = bindings.DllInterface()
    try:
        bindings.load_scene_spec(d, spec)
        return _render(d, iterations)
    finally:
        d.close()


@pytest.fixture
def loader_dll():
    d = bindings.DllInterface(useLoader=True)
    yield d
    d.close()


def _specs():
    tex = scenes.smooth_noise_texture(2, 16)
    return {
        "cornell": scenes.cornell_box(2, 40, 40),
        "ico": scenes.displaced_icosphere(2, subdiv=4, width=48, height=27),
        "inst": scenes.instanced_scene(3, num_meshes=3, num_instances=30, num_spheres=60, tri_range=(500, 2000),
                                       width=48, height=27),
        "tex": scenes.cornell_box_textured(2, 40, 40, texture=tex),
        "vcavity": _vcavity(scenes.displaced_icosphere(4, subdiv=3, width=40, height=24)),
        "alpha": scenes.alpha_cutouts(2, 40, 40),
    }


def _vcavity(spec):
    """Torrance materials with the file format's default shadowing model (V-cavity)."""
    return dataclasses.replace(spec, materials=[dataclasses.replace(m, shadowing=0) if m.type == scenes.MAT_TORRANCE
                                                else m for m in spec.materials])


@pytest.mark.parametrize("name", ["cornell", "ico", "inst", "tex", "vcavity", "alpha"])
@pytest.mark.parametrize("deflate,packed", [(False, False), (True, False), (True, True)])
def test_loaded_file_equals_api_built_scene(tmp_path, loader_dll, name, deflate, packed):
    spec = _specs()[name]
    jp = tmp_path / f"{name}.json"
    loaded_spec = scenefile.write_scene(spec, str(jp), deflate=deflate, compressed_normals=packed)
    bindings.load_scene_file(loader_dll, str(jp))
    img, hid = _render(loader_dll)
    ref_img, ref_hid = _render_spec(loaded_spec)
    assert np.array_equal(hid, ref_hid), "hit ids differ"
    assert np.array_equal(img, ref_img), "radiance differs"
    assert loader_dll.loader_get_loading_status() == ""  # no load running


def test_loaded_file_matches_oracle(tmp_path, loader_dll, oracle):
    spec = scenes.cornell_box(4, 48, 48)
    jp = tmp_path / "c.json"
    loaded_spec = scenefile.write_scene(spec, str(jp), deflate=True, compressed_normals=True)
    bindings.load_scene_file(loader_dll, str(jp))
    img, hid = _render(loader_dll, iterations=2)
    pt = oracle.OraclePathTracer(oracle.OracleScene(loaded_spec), seed=PARAMS["Seed"], min_path=0,
                                 max_path=PARAMS["Max. path length"], nee_count=1, rr_start=PARAMS["RR start depth"])
    for _ in range(2):
        pt.iterate()
    ref = pt.target("Radiance")
    assert np.array_equal(hid, pt.target("Hit ID"))
    err = np.sqrt(np.mean((img - ref) ** 2)) / np.sqrt(np.mean(ref ** 2))
    assert err <= 1e-4, err


# ---------------------------------------------------------------- scenarios and LoDs
def test_scenario_lods_masks_and_on_demand_loading(tmp_path, loader_dll):
    base, expect = cases.lod_scene(tmp_path)
    d = loader_dll
    bindings.load_scene_file(d, str(tmp_path / "lods.json"))
    A = d.core.world_get_object(d.muffInst, b"A")
    assert A
    assert d.core.object_has_lod(A, 0) and not d.core.object_has_lod(A, 1)  # only what "fine" needs
    assert d.core.world_get_instance_count(d.muffInst, 0xFFFFFFFF) == 4
    meta = d.loader_load_lod_metadatas(4)
    assert [m[1] for m in meta[:2]] == [len(expect["fine"][0][0].triangles), len(expect["coarse"][0][0].triangles)]
    assert meta[2][2] == 1 and meta[3][4] == 40
    assert d.loader_load_object_material_indices(2) == [2]
    for name in ["fine", "coarse", "mixed", "objlod", "masked", "fine"]:
        sc = d.world_find_scenario(name)
        assert sc and d.world_load_scenario(sc), d.core_get_dll_error()
        img, hid = _render(d)
        lods, inst = expect[name]
        spec = dataclasses.replace(base, lods=lods, instance_lod=np.array(inst, np.uint32))
        ref_img, ref_hid = _render_spec(spec)
        assert np.array_equal(hid, ref_hid), name
        assert np.array_equal(img, ref_img), name
    assert d.core.object_has_lod(A, 1)  # brought in by the "coarse" scenario


def _exact_transforms(n, seed):
    """World-to-instance matrices s*P | t (P a signed permutation, s a power of
    two, t on a 1/4 grid) whose inverses are exact in float32."""
    rng = np.random.default_rng(seed)
    w2i, i2w = [], []
    for _ in range(n):
        P = np.eye(3)[rng.permutation(3)] * rng.choice([-1.0, 1.0], 3)[:, None]
        s = float(rng.choice([0.5, 1.0, 2.0]))
        t = np.round(rng.uniform(-40, 40, 3) * 4) / 4
        A = s * P
        w2i.append(np.concatenate([A, t[:, None]], 1).reshape(12))
        Ai = P.T / s
        i2w.append(np.concatenate([Ai, (-Ai @ t)[:, None]], 1).reshape(12))
    return np.array(w2i, np.float32), np.array(i2w, np.float32)


def test_old_versions_use_instance_to_world_matrices(tmp_path, loader_dll):
    """Files before version 1.4 store instance-to-world matrices; the core
    inverts them. With exactly invertible transforms both files give the same
    world as the API-built scene."""
    spec = scenes.instanced_scene(6, num_meshes=2, num_instances=12, num_spheres=10, tri_range=(300, 900),
                                  width=40, height=30)
    w2i, i2w = _exact_transforms(len(spec.instance_lod), 9)
    w2i[-1] = scenes.identity34()
    i2w[-1] = scenes.identity34()
    spec = dataclasses.replace(spec, world_to_instance=w2i)
    new = tmp_path / "new.json"
    loaded_spec = scenefile.write_scene(spec, str(new))
    doc = json.loads(new.read_text())
    doc["version"] = "1.3"
    doc["binary"] = "old.mff"
    scenefile.write_json(str(tmp_path / "old.json"), doc)
    objs = [scenefile.MffObject(f"obj{i}_{l.name}", [l]) for i, l in enumerate(spec.lods)]
    insts = [scenefile.MffInstance(f"inst{i}", int(li), i2w[i]) for i, li in enumerate(spec.instance_lod)]
    scenefile.write_mff(str(tmp_path / "old.mff"), [f"mat{i}" for i in range(len(spec.materials))], objs, insts)
    ref_img, ref_hid = _render_spec(loaded_spec)
    for f in (new, tmp_path / "old.json"):
        bindings.load_scene_file(loader_dll, str(f))
        img, hid = _render(loader_dll)
        assert np.array_equal(hid, ref_hid), f
        assert np.array_equal(img, ref_img), f


# ---------------------------------------------------------------- failures
def _expect_error(d, path, *needles):
    st = d.loader_load_json(str(path))
    assert st == bindings.LoaderStatus.ERROR, st
    msg = d.loader_get_dll_error()
    for n in needles:
        assert n in msg, msg
    return msg


def test_broken_and_unsupported_files_fail_with_a_message(tmp_path, loader_dll):
    d = loader_dll
    good = None
    for path, needles in cases.failure_files(tmp_path):
        if needles is None:
            good = path
        elif isinstance(needles, list):  # loads, with warnings containing these words
            assert d.loader_load_json(str(path)) == bindings.LoaderStatus.SUCCESS, d.loader_get_dll_error()
            w = d.loader_get_warnings()
            for n in needles:
                assert any(n in x for x in w), (n, w)
        else:
            _expect_error(d, path, *needles)
    # the instance recovers: the good file still loads and renders
    bindings.load_scene_file(d, str(good))
    img, _ = _render(d, iterations=1, hit=False)
    assert np.isfinite(img).all() and img.max() > 0
    assert not d.loader_abort()  # nothing running
    assert "no load is running" in d.loader_get_dll_error()


def test_core_rejects_material_indices_beyond_the_slots():
    """The core refuses a LoD whose material index names no material slot of
    the scenario (the device indexes the material table with it); the file
    reader's own check is among the failure cases above."""
    spec = scenes.cornell_box(1, 16, 16)
    lod = dataclasses.replace(spec.lods[0], face_materials=np.full_like(spec.lods[0].face_materials, 50))
    d = bindings.DllInterface()
    try:
        with pytest.raises(bindings.MufflonError, match="material slots"):
            bindings.load_scene_spec(d, dataclasses.replace(spec, lods=[lod] + list(spec.lods[1:])))
    finally:
        d.close()


def test_c_program_renders_a_scene_file(tmp_path, core_lib_path):
    """The example.c flow in C, end to end: the saved PFM equals the image
    the Python binding renders from the same file with the default parameters."""
    from tests.conftest import build_c_example
    exe = build_c_example(core_lib_path, str(tmp_path))
    spec = scenes.cornell_box(7, 32, 24)
    jp = tmp_path / "scene.json"
    scenefile.write_scene(spec, str(jp), deflate=True)
    out = tmp_path / "out.pfm"
    r = subprocess.run([exe, "PT", "Radiance", str(jp), "4", str(out)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    data = out.read_bytes()
    header_end = data.index(b"-1.0\n") + 5
    assert data[:header_end].split()[:3] == [b"PF", b"32", b"24"]
    pfm = np.frombuffer(data[header_end:], "<f4").reshape(24, 32, 3)
    d = bindings.DllInterface(useLoader=True)
    try:
        bindings.load_scene_file(d, str(jp))
        assert d.render_enable_renderer(0, 0)
        d.render_enable_render_target("Radiance", False)
        for _ in range(4):
            d.render_iterate()
        assert np.array_equal(pfm, d.get_target_image("Radiance"))
    finally:
        d.close()
