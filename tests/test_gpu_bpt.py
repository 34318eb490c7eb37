"""The CUDA "Bidirectional Pathtracer" (core/bpt.cu) against the oracle's
restatement of the reference's CPU one (cpu_bpt.cpp:170-232).

Every contribution of an iteration is recorded per pixel and slot (each
connection of a view vertex with a light vertex, and each emitter the view
subpath hits: the pixel it lands in, radiance and lightness) and compared
bit for bit over two iterations: light subpaths from point, triangle and quad
lights and the colored background, the balance-heuristic weights from the
vertices' cached MIS sums, Lambert and both Torrance shadowing models, single-
and multi-level hierarchies. The images then differ only in the order the
atomics add the same terms."""
import dataclasses

import numpy as np
import pytest

from mufflon_b200 import bindings, scenes

pytestmark = pytest.mark.gpu


def _glossy_icosphere(shadowing, background=False):
    spec = scenes.displaced_icosphere(3, subdiv=4, width=48, height=32)
    mats = [dataclasses.replace(m, shadowing=shadowing) if m.type == scenes.MAT_TORRANCE else m for m in spec.materials]
    mats[1] = scenes.MaterialSpec(scenes.MAT_TORRANCE, albedo=(0.7, 0.7, 0.6), roughness=(0.3, 0.2), shadowing=shadowing)
    return dataclasses.replace(spec, materials=mats, background=spec.background if background else None)


def _instanced():
    spec = scenes.instanced_scene(0, num_meshes=3, num_instances=64, num_spheres=300, tri_range=(500, 3000),
                                  width=48, height=32)
    p = np.asarray(spec.cam_pos, np.float32) + 15.0 * np.asarray(spec.cam_dir, np.float32)
    lights = np.array([[p[0], p[1] + 3.0, p[2], 3000.0, 3000.0, 3000.0]], np.float32)
    return dataclasses.replace(spec, background=None, point_lights=lights)


CASES = {
    "panels": lambda: scenes.emissive_panels(5, 6, 40, 2, width=48, height=32, emissive_triangles=12),
    "sphere_lights": lambda: scenes.emissive_panels(7, 4, 10, 1, width=48, height=32, emissive_triangles=2,
                                                    emissive_spheres=6),
    "cornell": lambda: scenes.cornell_box(1, width=40, height=40),
    "icosphere_smith": lambda: _glossy_icosphere(1),
    "icosphere_vcavity_env": lambda: _glossy_icosphere(0, background=True),
    "instanced": _instanced,
}


def _gpu_bpt(spec, params, iterations, per_iteration=None):
    d = bindings.DllInterface()
    try:
        bindings.load_scene_spec(d, spec)
        assert d.render_enable_renderer(3, 0)
        for k, v in params.items():
            assert d.renderer_set_parameter_int(k, v)
        assert d.renderer_set_parameter_int("Record connections", 1)
        d.render_enable_render_target("Radiance", False)
        d.render_enable_render_target("Lightness", False)
        for it in range(iterations):
            d.render_iterate()
            if per_iteration:
                per_iteration(it, d.bpt_records(params["Max. path length"]))
        return {t: d.get_target_image(t) for t in ("Radiance", "Lightness")}, d.render_stats()
    finally:
        d.close()


def _rel_rmse(a, b):
    return float(np.sqrt(np.mean((a.astype(np.float64) - b) ** 2)) / max(np.sqrt(np.mean(b.astype(np.float64) ** 2)), 1e-30))


SCHEDULES = pytest.mark.parametrize("megakernel", [0, 1], ids=["stages", "single_kernel"])


@SCHEDULES
@pytest.mark.parametrize("case", list(CASES))
def test_bpt_contributions_and_image_match_oracle(oracle, case, megakernel):
    """Both schedules: stages per path length (the default) and the persistent
    kernel ("Megakernel" 1)."""
    spec = CASES[case]()
    params = {"Seed": 6, "Min. path length": 0, "Max. path length": 5, "Megakernel": megakernel}
    ob = oracle.OracleBidirPathTracer(oracle.OracleScene(spec), seed=6, min_path=0, max_path=5)
    seen = []

    def check(it, rec):
        ob.iterate()
        gp, gv = rec
        op, ov = ob.records()
        assert np.array_equal(gp, op), f"iteration {it}: contribution pixels differ ({np.sum(gp != op)} slots)"
        bad = np.nonzero(np.any(gv.view(np.uint32) != ov.view(np.uint32), axis=1))[0]
        assert len(bad) == 0, f"iteration {it}: {len(bad)} contributions differ, first slot {bad[0]}: {gv[bad[0]]} vs {ov[bad[0]]}"
        seen.append(int(np.count_nonzero(np.any(gv != 0, axis=1))))

    out, stats = _gpu_bpt(spec, params, 2, check)
    assert min(seen) > 50, seen
    assert stats["errors"] == 0 and stats["rays"] > 0
    for name, img in out.items():
        assert _rel_rmse(img, ob.target(name)) <= 1e-5, (name, _rel_rmse(img, ob.target(name)))


@SCHEDULES
def test_bpt_min_path_length(oracle, megakernel):
    spec = CASES["cornell"]()
    params = {"Seed": 2, "Min. path length": 3, "Max. path length": 4, "Megakernel": megakernel}
    ob = oracle.OracleBidirPathTracer(oracle.OracleScene(spec), seed=2, min_path=3, max_path=4)

    def check(it, rec):
        ob.iterate()
        op, ov = ob.records()
        assert np.array_equal(rec[0], op) and np.array_equal(rec[1].view(np.uint32), ov.view(np.uint32))

    out, _ = _gpu_bpt(spec, params, 2, check)
    assert _rel_rmse(out["Radiance"], ob.target("Radiance")) <= 1e-5


def test_bpt_in_the_registry():
    d = bindings.DllInterface()
    try:
        core, I = d.core, d.muffInst
        assert d.render_get_renderer_count() == 5
        assert d.render_get_renderer_name(3) == "Bidirectional Pathtracer"
        assert d.render_get_renderer_short_name(3) == "BPT"
        assert core.render_get_renderer_devices(I, 3, 0) == 2  # DEVICE_CUDA
        assert d.render_enable_renderer(3, 0)
        assert [core.render_get_render_target_name(I, i).decode() for i in range(core.render_get_render_target_count(I))] == \
            ["Radiance", "Lightness"]
        assert d.renderer_set_parameter_int("Seed", 5)
        assert d.render_enable_renderer(1, 0)
        assert d.renderer_get_parameter_int("Seed") == 0
    finally:
        d.close()


def _dark_icosphere():
    """No light at all: no point light, no emitter, no background."""
    spec = scenes.displaced_icosphere(4, subdiv=3, width=24, height=16)
    return dataclasses.replace(spec, background=None, point_lights=np.zeros((0, 6), np.float32))


@SCHEDULES
@pytest.mark.parametrize("case,max_path", [("panels", 1), ("cornell", 2), ("dark", 4)])
def test_bpt_edge_cases_match_oracle(oracle, case, max_path, megakernel):
    """Path length 1 (no light-subpath walk), 2, and a scene without lights
    (no light subpath; only the view subpath runs and the image stays black)."""
    spec = _dark_icosphere() if case == "dark" else CASES[case]()
    params = {"Seed": 1, "Min. path length": 0, "Max. path length": max_path, "Megakernel": megakernel}
    ob = oracle.OracleBidirPathTracer(oracle.OracleScene(spec), seed=1, min_path=0, max_path=max_path)

    def check(it, rec):
        ob.iterate()
        op, ov = ob.records()
        assert np.array_equal(rec[0], op) and np.array_equal(rec[1].view(np.uint32), ov.view(np.uint32))

    out, stats = _gpu_bpt(spec, params, 2, check)
    if case == "dark":
        assert not out["Radiance"].any() and stats["rays"] > 0
    else:
        assert out["Radiance"].any()
        assert _rel_rmse(out["Radiance"], ob.target("Radiance")) <= 1e-5


@pytest.mark.parametrize("renderer", [1, 3, 4], ids=["lt", "bpt", "vcm"])
def test_stages_refuse_paths_beyond_their_launch_count(renderer):
    """The staged schedules launch a fixed number of generations; a longer
    max. path length fails the iteration with a message (for the light and
    bidirectional tracers naming the switch to the persistent kernel, and
    "Megakernel" 1 renders it; vertex connection and merging has only the
    stages)."""
    spec = scenes.cornell_box(1, width=8, height=8)
    d = bindings.DllInterface()
    try:
        bindings.load_scene_spec(d, spec)
        assert d.render_enable_renderer(renderer, 0)
        assert d.renderer_set_parameter_int("Max. path length", 65)
        with pytest.raises(bindings.MufflonError, match="at most 64 path lengths"):
            d.render_iterate()
        if renderer == 4:
            return
        assert d.renderer_set_parameter_int("Megakernel", 1)
        d.render_iterate()
        assert d.render_stats()["rays"] > 0
    finally:
        d.close()
