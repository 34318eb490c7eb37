"""The CUDA "Wireframe" (core/wireframe.cu) against the oracle's restatement
of the reference's CPU one (wireframe_common.hpp:93-180, cpu_wireframe.cpp:18-38).

The cumulative "Border" image is compared bit for bit after each of two
iterations (one documented pixel of the Cornell box excepted): camera rays with the per-pixel generator stream, the walk through
the surfaces (each step re-traced from the hit point), the closest-edge
distance of triangles and quads, the rim test of spheres, instance transforms
and the background on a miss. The registry entry, the target list and the
"Line width" parameter are tested too."""
import dataclasses

import numpy as np
import pytest

from mufflon_b200 import bindings, scenes

pytestmark = pytest.mark.gpu


def _degenerate_quad_room():
    """The Cornell box's walls and light without the two boxes, with the back
    wall's last two corners made equal: a quad with a zero-length edge, whose
    closest-edge distance is NaN for that edge (the reference's comparison
    chain then falls through to its last edge)."""
    spec = scenes.cornell_box(1, width=64, height=64)
    walls = spec.lods[0]
    v = walls.vertices.copy()
    v[11] = v[10]
    lods = [dataclasses.replace(walls, vertices=v), spec.lods[-1]]
    return dataclasses.replace(spec, lods=lods, world_to_instance=spec.world_to_instance[[0, -1]],
                               instance_lod=np.array([0, 1], np.uint32))


CASES = {
    "cornell": lambda: scenes.cornell_box(1, width=64, height=64),
    "icosphere_env": lambda: scenes.displaced_icosphere(2, subdiv=3, width=64, height=36),
    "panels_quads": lambda: scenes.emissive_panels(5, 6, 40, 2, width=64, height=48, emissive_triangles=12),
    "instanced_spheres": lambda: scenes.instanced_scene(0, num_meshes=3, num_instances=64, num_spheres=300,
                                                        tri_range=(500, 3000), width=64, height=48),
    "degenerate_quad": _degenerate_quad_room,
}
# Pixels (row from the bottom, column) allowed to differ from the oracle, per
# case (see the test): on the Cornell box both lie on the floor inside the
# footprint of the box standing at x ~ -0.45.
ALLOWED_DIFF = {"cornell": {(7, 14), (8, 25)}}


def _gpu_wireframe(spec, iterations, line_width=None, depth=None):
    d = bindings.DllInterface()
    out = []
    try:
        bindings.load_scene_spec(d, spec)
        assert d.render_enable_renderer(2, 0)
        if line_width is not None:
            assert d.renderer_set_parameter_float("Line width", line_width)
        if depth is not None:
            assert d.renderer_set_parameter_int("Maximum trace depth", depth)
        d.render_enable_render_target("Border", False)
        for _ in range(iterations):
            d.render_iterate()
            out.append(d.get_target_image("Border").copy())
        return out
    finally:
        d.close()


@pytest.mark.parametrize("case", list(CASES))
@pytest.mark.parametrize("line_width,depth", [(None, None), (3.5, 4)], ids=["default", "wide_depth4"])
def test_wireframe_border_matches_oracle(oracle, case, line_width, depth):
    spec = CASES[case]()
    imgs = _gpu_wireframe(spec, 2, line_width, depth)
    ow = oracle.OracleWireframe(oracle.OracleScene(spec), 1.0 if line_width is None else line_width,
                                1000 if depth is None else depth)
    for img in imgs:
        ow.iterate()
        ref = ow.target()
        assert img.shape == ref.shape
        # A walk re-traces from each hit point without an offset, so a ray can
        # start within 1e-7 of two coplanar surfaces (the bottom face of a box
        # standing on the floor, and the floor) and meet both at t ~ 4e-7;
        # the last bits of the instance transform then pick the closer one.
        # On the Cornell box 2 of 4096 pixels take the other branch (one per
        # iteration's sub-pixel offsets); every other case is bit-identical.
        differ = {tuple(int(c) for c in rc) for rc in np.argwhere(np.any(img.view(np.uint32) != ref.view(np.uint32), axis=-1))}
        assert differ <= ALLOWED_DIFF.get(case, set()), sorted(differ)
    # some pixels are edges, some are not
    assert 0.0 < float(np.mean(imgs[-1][..., 0] == 1.0)) < 1.0


def test_wireframe_in_the_registry():
    d = bindings.DllInterface()
    try:
        core, I = d.core, d.muffInst
        assert d.render_get_renderer_name(2) == "Wireframe"
        assert d.render_get_renderer_short_name(2) == "WF"
        assert core.render_get_renderer_devices(I, 2, 0) == 2  # DEVICE_CUDA
        assert d.render_enable_renderer(2, 0)
        assert [core.render_get_render_target_name(I, i).decode() for i in range(core.render_get_render_target_count(I))] == \
            ["Border"]
        names = [core.renderer_get_parameter_desc(I, i, None).decode() for i in range(core.renderer_get_num_parameters(I))]
        assert names == ["Line width", "Maximum trace depth", "Traversal step limit"]
        assert d.renderer_get_parameter_float("Line width") == 1.0
        assert d.renderer_get_parameter_int("Maximum trace depth") == 1000
        assert d.renderer_set_parameter_float("Line width", 2.0)
        assert not d.renderer_set_parameter_int("Seed", 1)
        assert d.render_enable_renderer(0, 0)
        assert d.renderer_get_parameter_int("Seed") == 0
        assert d.render_enable_renderer(2, 0)
        assert d.renderer_get_parameter_float("Line width") == 2.0
    finally:
        d.close()


def test_wireframe_radiance_is_not_a_target():
    spec = CASES["cornell"]()
    d = bindings.DllInterface()
    try:
        bindings.load_scene_spec(d, spec)
        assert d.render_enable_renderer(2, 0)
        d.render_enable_render_target("Border", False)
        d.render_iterate()
        with pytest.raises(bindings.MufflonError):
            d.get_target_image("Radiance")
    finally:
        d.close()
