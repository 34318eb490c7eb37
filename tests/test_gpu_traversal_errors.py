"""Abandoned traversals fail the call instead of returning silently wrong pixels.

Every traversal loop is bounded: a ray that exceeds the step limit (or the
traversal stack) is abandoned and counted. Following the reference's error
convention (interface.cpp:53-83: a failing call returns false and leaves a
message for core_get_dll_error), render_iterate then returns false. The test
forces the exit with a tiny "Traversal step limit" (a bounded-loop exit, not a
fault), checks the failure and its message for each renderer and schedule, and
checks that with the limit back at its default the same instance renders the
oracle's image again.
"""
import numpy as np
import pytest

from mufflon_b200 import bindings, scenes

pytestmark = pytest.mark.gpu


def _iterate_ok(d):
    return d.core.render_iterate(d.muffInst, None, None, None) != 0


@pytest.mark.parametrize("renderer,extra", [(0, {"Megakernel": 0}), (0, {"Megakernel": 1}), (1, {"Megakernel": 0}),
                                            (1, {"Megakernel": 1}), (2, {}), (3, {"Megakernel": 0}), (3, {"Megakernel": 1}),
                                            (4, {})],
                         ids=["pt-wavefront", "pt-megakernel", "lt-stages", "lt-single-kernel", "wireframe", "bpt-stages",
                              "bpt-single-kernel", "vcm"])
def test_step_limit_fails_the_iteration(renderer, extra):
    spec = scenes.displaced_icosphere(0, subdiv=4, width=48, height=27)
    d = bindings.DllInterface()
    try:
        bindings.load_scene_spec(d, spec)
        assert d.render_enable_renderer(renderer, 0)
        for k, v in extra.items():
            assert d.renderer_set_parameter_int(k, v)
        assert d.renderer_set_parameter_int("Traversal step limit", 2)
        assert d.renderer_get_parameter_int("Traversal step limit") == 2
        assert not _iterate_ok(d)
        msg = d.core_get_dll_error()
        assert "traversal abandoned" in msg and "step limit of 2" in msg, msg
        assert d.renderer_set_parameter_int("Traversal step limit", 0)
        assert _iterate_ok(d), d.core_get_dll_error()
        assert d.render_stats()["errors"] == 0
    finally:
        d.close()


def test_default_limit_renders_the_oracle_image_after_a_failure(oracle):
    spec = scenes.cornell_box(1, 64, 64)
    d = bindings.DllInterface()
    try:
        bindings.load_scene_spec(d, spec)
        assert d.render_enable_renderer(0, 0)
        assert d.renderer_set_parameter_int("Max. path length", 8)
        d.render_enable_render_target("Hit ID", False)
        assert d.renderer_set_parameter_int("Traversal step limit", 1)
        assert not _iterate_ok(d)
        assert d.renderer_set_parameter_int("Traversal step limit", 0)  # resets the accumulation
        assert _iterate_ok(d), d.core_get_dll_error()
        img = d.get_target_image("Radiance").copy()
        hid = d.get_target_image("Hit ID").copy()
    finally:
        d.close()
    pt = oracle.OraclePathTracer(oracle.OracleScene(spec), seed=0, max_path=8)
    pt.iterate()
    assert np.array_equal(hid, pt.target("Hit ID"))
    assert np.array_equal(img.view(np.uint32), pt.target("Radiance").view(np.uint32))


def test_batch_with_step_limit_fails():
    spec = scenes.cornell_box(2, 32, 32)
    d = bindings.DllInterface()
    try:
        bindings.load_scene_spec(d, spec)
        assert d.render_enable_renderer(0, 0)
        assert d.renderer_set_parameter_int("Traversal step limit", 1)
        with pytest.raises(bindings.MufflonError, match="traversal abandoned"):
            bindings.render_batch([dict(instance=d, spp=1, max_path=4)])
    finally:
        d.close()
