"""The CUDA "Vertex Connection and Merging" renderer (core/vcm.cu) against the
oracle's restatement of the reference's CPU one (cpu_vcm.cpp:148-290).

Every contribution of an iteration is recorded per pixel and slot (each
connection of a view vertex with a vertex of its light subpath, each emitter
the view subpath hits, and each view vertex's merges with the photons of all
light subpaths: the pixel it lands in, radiance and lightness) and compared
bit for bit over two iterations. The merges follow the photon map's bucket
order, so their sums are the oracle's to the last bit as well; the images then
differ only in the order the atomics add the same terms."""
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


def _gpu_vcm(spec, params, iterations, radius, progressive=False, per_iteration=None):
    d = bindings.DllInterface()
    try:
        bindings.load_scene_spec(d, spec)
        assert d.render_enable_renderer(4, 0)
        for k, v in params.items():
            assert d.renderer_set_parameter_int(k, v)
        assert d.renderer_set_parameter_float("Relative merge radius", radius)
        assert d.renderer_set_parameter_bool("Progressive", progressive)
        assert d.renderer_set_parameter_int("Record connections", 1)
        d.render_enable_render_target("Radiance", False)
        d.render_enable_render_target("Lightness", False)
        for it in range(iterations):
            d.render_iterate()
            if per_iteration:
                per_iteration(it, d.vcm_records(params["Max. path length"]))
        return {t: d.get_target_image(t) for t in ("Radiance", "Lightness")}, d.render_stats()
    finally:
        d.close()


def _rel_rmse(a, b):
    return float(np.sqrt(np.mean((a.astype(np.float64) - b) ** 2)) / max(np.sqrt(np.mean(b.astype(np.float64) ** 2)), 1e-30))


def _compare(ob, seen=None, m=None):
    def check(it, rec):
        ob.iterate()
        gp, gv = rec
        op, ov = ob.records()
        assert np.array_equal(gp, op), f"iteration {it}: contribution pixels differ ({np.sum(gp != op)} slots)"
        bad = np.nonzero(np.any(gv.view(np.uint32) != ov.view(np.uint32), axis=1))[0]
        assert len(bad) == 0, f"iteration {it}: {len(bad)} contributions differ, first slot {bad[0]}: {gv[bad[0]]} vs {ov[bad[0]]}"
        if seen is not None:
            per = gv.reshape(-1, m * m + 2 * m, 4)
            seen.append((int(np.count_nonzero(np.any(per[:, :m * m] != 0, axis=2))),
                         int(np.count_nonzero(np.any(per[:, m * m + m:] != 0, axis=2)))))
    return check


@pytest.mark.parametrize("case", list(CASES))
def test_vcm_contributions_and_image_match_oracle(oracle, case):
    """Connections, emitter hits and merges bit for bit over two iterations;
    a merge radius of 2 % of the scene's diagonal gives every case many
    merges."""
    spec = CASES[case]()
    m = 5
    params = {"Seed": 6, "Min. path length": 0, "Max. path length": m}
    ob = oracle.OracleVcm(oracle.OracleScene(spec), seed=6, min_path=0, max_path=m, merge_radius=0.02)
    seen = []
    out, stats = _gpu_vcm(spec, params, 2, 0.02, per_iteration=_compare(ob, seen, m))
    assert min(c for c, _ in seen) > 50, seen
    assert min(mg for _, mg in seen) > 10, seen
    assert stats["errors"] == 0 and stats["rays"] > 0
    for name, img in out.items():
        assert _rel_rmse(img, ob.target(name)) <= 1e-5, (name, _rel_rmse(img, ob.target(name)))


def test_vcm_min_path_length_and_progressive_radius(oracle):
    """A minimum path length filters connections, hits and merges; the
    progressive radius shrinks with the iteration (three iterations)."""
    spec = CASES["cornell"]()
    params = {"Seed": 2, "Min. path length": 3, "Max. path length": 4}
    ob = oracle.OracleVcm(oracle.OracleScene(spec), seed=2, min_path=3, max_path=4, merge_radius=0.03, progressive=True)
    out, _ = _gpu_vcm(spec, params, 3, 0.03, progressive=True, per_iteration=_compare(ob))
    assert _rel_rmse(out["Radiance"], ob.target("Radiance")) <= 1e-5


def _dark_icosphere():
    """No light at all: no point light, no emitter, no background."""
    spec = scenes.displaced_icosphere(4, subdiv=3, width=24, height=16)
    return dataclasses.replace(spec, background=None, point_lights=np.zeros((0, 6), np.float32))


@pytest.mark.parametrize("case,max_path", [("panels", 1), ("cornell", 2), ("dark", 4)])
def test_vcm_edge_cases_match_oracle(oracle, case, max_path):
    """Path length 1 (no light-subpath walk, no merge fits), 2, and a scene
    without lights (no light subpaths, no photons; the image stays black)."""
    spec = _dark_icosphere() if case == "dark" else CASES[case]()
    params = {"Seed": 1, "Min. path length": 0, "Max. path length": max_path}
    ob = oracle.OracleVcm(oracle.OracleScene(spec), seed=1, min_path=0, max_path=max_path, merge_radius=0.02)
    out, stats = _gpu_vcm(spec, params, 2, 0.02, per_iteration=_compare(ob))
    if case == "dark":
        assert not out["Radiance"].any() and stats["rays"] > 0
    else:
        assert out["Radiance"].any()
        assert _rel_rmse(out["Radiance"], ob.target("Radiance")) <= 1e-5


def test_vcm_in_the_registry():
    """Renderer 4 with the reference's parameters (vcm_params.hpp) and targets."""
    d = bindings.DllInterface()
    try:
        core, I = d.core, d.muffInst
        assert d.render_get_renderer_name(4) == "Vertex Connection and Merging"
        assert d.render_get_renderer_short_name(4) == "VCM"
        assert core.render_get_renderer_devices(I, 4, 0) == 2  # DEVICE_CUDA
        assert d.render_enable_renderer(4, 0)
        assert [core.render_get_render_target_name(I, i).decode() for i in range(core.render_get_render_target_count(I))] == \
            ["Radiance", "Lightness"]
        names = [core.renderer_get_parameter_desc(I, i, None).decode() for i in range(core.renderer_get_num_parameters(I))]
        assert names[:5] == ["Seed", "Min. path length", "Max. path length", "Relative merge radius", "Progressive"]
        assert d.renderer_get_parameter_float("Relative merge radius") == pytest.approx(0.001)
        assert d.renderer_get_parameter_bool("Progressive") is False
        assert d.renderer_set_parameter_float("Relative merge radius", 0.01)
        assert d.renderer_get_parameter_float("Relative merge radius") == pytest.approx(0.01)
        assert not d.renderer_set_parameter_float("Relative merge radius", 0.0)
        assert d.renderer_set_parameter_bool("Progressive", True)
        assert d.renderer_get_parameter_bool("Progressive") is True
        assert not d.renderer_set_parameter_int("Megakernel", 1)
        assert d.render_enable_renderer(3, 0)
        assert not d.renderer_set_parameter_float("Relative merge radius", 0.01)
    finally:
        d.close()
