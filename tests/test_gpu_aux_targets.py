"""The path tracer's auxiliary targets against the oracle.

"Position", "Depth", "Normal", "UV", "Albedo" and "Lightness" (pt_params.hpp:
16-26) are contributed as pt_common.hpp:105-152 does: at every vertex from the
minimum path length on, weighted by the guide weight of the camera path's
footprint (footprint.hpp:137-165), and "Lightness" also at every unoccluded
next-event sample. Each pixel's terms are added in the path's own order on
both sides, so the cumulative images (and their variances) are compared bit for
bit, for both schedules, over several iterations with Russian roulette, a
minimum path length and two next-event samples per vertex.
"""
import numpy as np
import pytest

from mufflon_b200 import bindings, scenes

pytestmark = pytest.mark.gpu

AUX = ["Position", "Depth", "Normal", "UV", "Albedo", "Lightness"]
CASES = {
    "cornell": lambda: scenes.cornell_box(2, 48, 48),
    "icosphere_env": lambda: scenes.displaced_icosphere(1, subdiv=4, width=64, height=36),
    "instanced": lambda: scenes.instanced_scene(1, num_meshes=3, num_instances=48, num_spheres=200,
                                                tri_range=(500, 3000), width=48, height=32),
}


@pytest.mark.parametrize("megakernel", [0, 1], ids=["wavefront", "megakernel"])
@pytest.mark.parametrize("case", list(CASES))
def test_aux_targets_match_oracle(oracle, case, megakernel):
    spec = CASES[case]()
    params = {"Seed": 3, "Max. path length": 7, "Min. path length": 1, "NEE count": 2, "RR start depth": 2,
              "Megakernel": megakernel}
    d = bindings.DllInterface()
    try:
        bindings.load_scene_spec(d, spec)
        assert d.render_enable_renderer(0, 0)
        for k, v in params.items():
            assert d.renderer_set_parameter_int(k, v)
        for name in AUX:
            assert d.render_enable_render_target(name, name in ("Depth", "Lightness"))
        d.render_enable_render_target("Hit ID", False)
        for _ in range(3):
            d.render_iterate()
        got = {name: d.get_target_image(name) for name in AUX}
        got_var = {name: d.get_target_image(name, variance=True) for name in ("Depth", "Lightness")}
        rad, hid = d.get_target_image("Radiance"), d.get_target_image("Hit ID")
    finally:
        d.close()
    pt = oracle.OraclePathTracer(oracle.OracleScene(spec), seed=3, min_path=1, max_path=7, nee_count=2, rr_start=2)
    for _ in range(3):
        pt.iterate()
    assert np.array_equal(rad.view(np.uint32), pt.target("Radiance").view(np.uint32))
    assert np.array_equal(hid, pt.target("Hit ID"))
    for name in AUX:
        ref = pt.target(name)
        assert got[name].shape == ref.shape, name
        assert np.array_equal(got[name].view(np.uint32), ref.view(np.uint32)), \
            (name, int(np.sum(got[name].view(np.uint32) != ref.view(np.uint32))))
    for name, img in got_var.items():
        assert np.array_equal(img.view(np.uint32), pt.target(name, variance=True).view(np.uint32)), name
    # the targets are not trivial
    assert float(got["Depth"].max()) > 0.0 and float(np.abs(got["Normal"]).max()) > 0.0
    assert float(got["Lightness"].max()) > 0.0 and float(got["Albedo"].max()) > 0.0


def test_first_hit_depth_and_albedo_of_a_direct_view(oracle):
    """With a path length of 1 a pixel's Depth is its camera ray's hit distance times the first
    vertex's guide weight (1 / (1 + 1 / pdf) for the pinhole's pdf), the same on both sides."""
    spec = scenes.cornell_box(0, 32, 32)
    d = bindings.DllInterface()
    try:
        bindings.load_scene_spec(d, spec)
        assert d.render_enable_renderer(0, 0)
        assert d.renderer_set_parameter_int("Max. path length", 1)
        for name in ("Depth", "Albedo"):
            assert d.render_enable_render_target(name, False)
        d.render_iterate()
        depth, albedo = d.get_target_image("Depth"), d.get_target_image("Albedo")
    finally:
        d.close()
    pt = oracle.OraclePathTracer(oracle.OracleScene(spec), seed=0, max_path=1)
    pt.iterate()
    assert np.array_equal(depth, pt.target("Depth")) and np.array_equal(albedo, pt.target("Albedo"))
    assert 2.0 < float(np.median(depth)) < 5.0  # the camera stands 3.6 in front of the box
