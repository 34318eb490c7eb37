"""The CUDA "Lighttracer" (core/lt.cu) against the oracle's light tracer
(lt_common.hpp:19-77 restated).

Every camera connection of an iteration is recorded per photon and path
length (pixel and added radiance, lightness, density) and compared bit for
bit: emission from point, triangle and quad lights and the colored
background picked through the light tree, the camera projection, adjoint BSDF evaluation and sampling of Lambert
and both Torrance shadowing models, the walk through single- and
multi-level hierarchies and the generator stream across iterations. The
images differ only in the order the atomics add the same terms: relative
RMSE within 1e-5. The renderer registry and the target checks are tested too."""
import dataclasses

import numpy as np
import pytest

from mufflon_b200 import bindings, scenes

pytestmark = pytest.mark.gpu


def _glossy_icosphere(shadowing):
    spec = scenes.displaced_icosphere(3, subdiv=4, width=64, height=36)
    mats = [dataclasses.replace(m, shadowing=shadowing) if m.type == scenes.MAT_TORRANCE else m for m in spec.materials]
    mats[1] = scenes.MaterialSpec(scenes.MAT_TORRANCE, albedo=(0.7, 0.7, 0.6), roughness=(0.3, 0.2), shadowing=shadowing)
    return dataclasses.replace(spec, materials=mats, background=None)


def _instanced():
    """Instances with a point light in front of the camera (the scene's own
    light is far from what the camera sees)."""
    spec = scenes.instanced_scene(0, num_meshes=3, num_instances=64, num_spheres=300, tri_range=(500, 3000),
                                  width=64, height=48)
    p = np.asarray(spec.cam_pos, np.float32) + 15.0 * np.asarray(spec.cam_dir, np.float32)
    lights = np.array([[p[0], p[1] + 3.0, p[2], 3000.0, 3000.0, 3000.0]], np.float32)
    return dataclasses.replace(spec, background=None, point_lights=lights)


CASES = {
    "panels": lambda: scenes.emissive_panels(5, 6, 40, 2, width=64, height=48, emissive_triangles=12),
    "sphere_lights": lambda: scenes.emissive_panels(7, 4, 10, 1, width=64, height=48, emissive_triangles=2,
                                                    emissive_spheres=6),
    "cornell": lambda: scenes.cornell_box(1, width=64, height=64),
    "icosphere_smith": lambda: _glossy_icosphere(1),
    "icosphere_vcavity": lambda: _glossy_icosphere(0),
    "instanced": _instanced,
    # a colored background next to a point light: photons from the environment too
    "icosphere_env": lambda: scenes.displaced_icosphere(2, subdiv=4, width=64, height=36),
}


def _gpu_lt(spec, params, iterations, density, per_iteration=None):
    d = bindings.DllInterface()
    try:
        bindings.load_scene_spec(d, spec)
        assert d.render_enable_renderer(1, 0)
        for k, v in params.items():
            assert d.renderer_set_parameter_int(k, v)
        assert d.renderer_set_parameter_int("Record connections", 1)
        d.render_enable_render_target("Radiance", False)
        d.render_enable_render_target("Lightness", False)
        if density:
            d.render_enable_render_target("Density", False)
        for it in range(iterations):
            d.render_iterate()
            if per_iteration:
                per_iteration(it, d.lt_records(params["Max. path length"]))
        out = {t: d.get_target_image(t) for t in (["Radiance", "Lightness"] + (["Density"] if density else []))}
        stats = d.render_stats()
        return out, stats
    finally:
        d.close()


def _rel_rmse(a, b):
    return float(np.sqrt(np.mean((a.astype(np.float64) - b) ** 2)) / max(np.sqrt(np.mean(b.astype(np.float64) ** 2)), 1e-30))


@pytest.mark.parametrize("case", list(CASES))
@pytest.mark.parametrize("density", [False, True], ids=["plain", "density"])
@pytest.mark.parametrize("megakernel", [0, 1], ids=["stages", "single_kernel"])
def test_lt_connections_and_image_match_oracle(oracle, case, density, megakernel):
    """Both schedules: the stages per path length (default) and the single
    persistent kernel ("Megakernel" 1)."""
    spec = CASES[case]()
    params = {"Seed": 4, "Min. path length": 0, "Max. path length": 6, "Megakernel": megakernel}
    lt = oracle.OracleLightTracer(oracle.OracleScene(spec), seed=4, min_path=0, max_path=6, density=density)
    seen = []

    def check(it, rec):
        lt.iterate()
        gp, gv = rec
        op, ov = lt.records()
        assert np.array_equal(gp, op), f"iteration {it}: connection pixels differ ({np.sum(gp != op)} slots)"
        assert np.array_equal(gv.view(np.uint32), ov.view(np.uint32)), f"iteration {it}: connection values differ"
        seen.append(int((gp >= 0).sum()))

    out, stats = _gpu_lt(spec, params, 2, density, check)
    assert min(seen) > 50, seen
    assert stats["errors"] == 0 and stats["rays"] > 0
    for name, img in out.items():
        ref = lt.target(name)
        assert img.shape == ref.shape
        assert _rel_rmse(img, ref) <= 1e-5, (name, _rel_rmse(img, ref))


def test_lt_min_path_length(oracle):
    spec = CASES["panels"]()
    params = {"Seed": 9, "Min. path length": 2, "Max. path length": 4}
    lt = oracle.OracleLightTracer(oracle.OracleScene(spec), seed=9, min_path=2, max_path=4)

    def check(it, rec):
        lt.iterate()
        op, ov = lt.records()
        assert np.array_equal(rec[0], op) and np.array_equal(rec[1].view(np.uint32), ov.view(np.uint32))
        # slot 0 (the light vertex, path length 1) is below the minimum
        assert np.all(rec[0].reshape(-1, 4)[:, 0] == -1)

    out, _ = _gpu_lt(spec, params, 2, False, check)
    assert _rel_rmse(out["Radiance"], lt.target("Radiance")) <= 1e-5


def test_renderer_registry_lists_the_light_tracer():
    d = bindings.DllInterface()
    try:
        assert d.render_get_renderer_count() == 5
        assert [d.render_get_renderer_name(i) for i in range(5)] == \
            ["Pathtracer", "Lighttracer", "Wireframe", "Bidirectional Pathtracer", "Vertex Connection and Merging"]
        assert [d.render_get_renderer_short_name(i) for i in range(5)] == ["PT", "LT", "WF", "BPT", "VCM"]
        core, I = d.core, d.muffInst
        assert core.render_get_renderer_variations(I, 1) == 1
        assert core.render_get_renderer_devices(I, 1, 0) == 2  # DEVICE_CUDA
        assert not d.render_enable_renderer(5, 0)
        assert d.render_enable_renderer(1, 0)
        assert core.render_get_render_target_count(I) == 3
        assert [core.render_get_render_target_name(I, i).decode() for i in range(3)] == ["Radiance", "Lightness", "Density"]
        names = [core.renderer_get_parameter_desc(I, i, None).decode() for i in range(core.renderer_get_num_parameters(I))]
        assert names[:3] == ["Seed", "Min. path length", "Max. path length"]
        assert not d.renderer_set_parameter_int("NEE count", 1)  # a path-tracer parameter
        assert d.render_enable_renderer(0, 0)
        assert core.render_get_render_target_count(I) == 8
        assert d.renderer_set_parameter_int("NEE count", 1)
    finally:
        d.close()


def test_lt_and_pt_keep_separate_parameters():
    d = bindings.DllInterface()
    try:
        assert d.render_enable_renderer(1, 0)
        assert d.renderer_set_parameter_int("Seed", 77)
        assert d.render_enable_renderer(0, 0)
        assert d.renderer_get_parameter_int("Seed") == 0
        assert d.render_enable_renderer(1, 0)
        assert d.renderer_get_parameter_int("Seed") == 77
    finally:
        d.close()


def test_hit_id_is_not_a_light_tracer_target():
    spec = CASES["panels"]()
    d = bindings.DllInterface()
    try:
        bindings.load_scene_spec(d, spec)
        assert d.render_enable_renderer(1, 0)
        d.render_enable_render_target("Hit ID", False)
        d.render_iterate()
        with pytest.raises(bindings.MufflonError, match="not produced by the CUDA light tracer"):
            d.get_target_image("Hit ID")
    finally:
        d.close()


def _dark_icosphere():
    """No light at all: no point light, no emitter, no background."""
    spec = scenes.displaced_icosphere(4, subdiv=3, width=24, height=16)
    return dataclasses.replace(spec, background=None, point_lights=np.zeros((0, 6), np.float32))


@pytest.mark.parametrize("case,max_path", [("panels", 1), ("cornell", 2), ("dark", 4)])
def test_lt_edge_cases_match_oracle(oracle, case, max_path):
    """Path length 1 (only the light vertices' own connections), 2, and a
    scene without lights (no photon starts; the image stays black)."""
    spec = _dark_icosphere() if case == "dark" else CASES[case]()
    params = {"Seed": 1, "Min. path length": 0, "Max. path length": max_path}
    lt = oracle.OracleLightTracer(oracle.OracleScene(spec), seed=1, min_path=0, max_path=max_path)

    def check(it, rec):
        lt.iterate()
        op, ov = lt.records()
        assert np.array_equal(rec[0], op) and np.array_equal(rec[1].view(np.uint32), ov.view(np.uint32))

    out, stats = _gpu_lt(spec, params, 2, False, check)
    if case == "dark":
        assert not out["Radiance"].any() and stats["rays"] == 0
    else:
        assert out["Radiance"].any()
        assert _rel_rmse(out["Radiance"], lt.target("Radiance")) <= 1e-5
