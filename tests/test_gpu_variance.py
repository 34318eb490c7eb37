"""Variance targets (render_enable_render_target(name, variance=true)).

The reference keeps, per recorded target, a running mean and (when asked) a
running variance, updated once per iteration by the stable scheme of
output_handler_variance.hpp:7-31; targets that reduce moments (the light
tracer's Density, render_targets.hpp:68-74) keep the iteration's value and,
in the variance slot, the running mean. Enabling a variance also records its
target; disabling with variance=true stops only the variance
(output_handler.hpp:391-431); reading a variance that is not recorded fails
(output_handler.hpp:303-306).

The GPU's variance buffers are compared with the oracle's after several
iterations: bit for bit for the path tracer (whose per-pixel sums are
sequential on both sides) and the wireframe renderer, and within relative
RMSE 1e-5 for the light tracer and the bidirectional path tracer, whose
images are summed with atomics in no fixed order.
"""
import numpy as np
import pytest

from mufflon_b200 import bindings, scenes

pytestmark = pytest.mark.gpu

ITERATIONS = 5


def _rel_rmse(a, b):
    a = a.astype(np.float64)
    b = b.astype(np.float64)
    return float(np.sqrt(np.mean((a - b) ** 2)) / max(np.sqrt(np.mean(b ** 2)), 1e-30))


def _render(spec, renderer, params, targets, iterations=ITERATIONS):
    d = bindings.DllInterface()
    try:
        bindings.load_scene_spec(d, spec)
        assert d.render_enable_renderer(renderer, 0)
        for k, v in params.items():
            assert d.renderer_set_parameter_int(k, v)
        for t in targets:
            assert d.render_enable_render_target(t, True)
        for _ in range(iterations):
            d.render_iterate()
        return {t: (d.get_target_image(t), d.get_target_image(t, variance=True)) for t in targets}
    finally:
        d.close()


@pytest.mark.parametrize("megakernel", [0, 1], ids=["wavefront", "megakernel"])
def test_pt_variance_matches_oracle(oracle, megakernel):
    spec = scenes.cornell_box(3, 64, 64)
    out = _render(spec, 0, {"Max. path length": 8, "Seed": 5, "Megakernel": megakernel}, ["Radiance", "Hit ID"])
    pt = oracle.OraclePathTracer(oracle.OracleScene(spec), seed=5, max_path=8)
    for _ in range(ITERATIONS):
        pt.iterate()
    for name, (mean, var) in out.items():
        assert np.array_equal(mean.view(np.uint32), pt.target(name).view(np.uint32)), name
        ref = pt.target(name, variance=True)
        assert np.array_equal(var.view(np.uint32), ref.view(np.uint32)), (name, _rel_rmse(var, ref))
    # a noisy image has a non-trivial variance; the hit ids of a static camera vary only at edges
    assert float(out["Radiance"][1].mean()) > 0.0
    assert 0.0 < float(np.mean(out["Hit ID"][1] > 0)) < 0.5


def test_lt_variance_and_density_mean_match_oracle(oracle):
    spec = scenes.emissive_panels(5, 6, 40, 2, width=64, height=48, emissive_triangles=12)
    out = _render(spec, 1, {"Max. path length": 6, "Seed": 2}, ["Radiance", "Lightness", "Density"])
    lt = oracle.OracleLightTracer(oracle.OracleScene(spec), seed=2, max_path=6, density=True)
    for _ in range(ITERATIONS):
        lt.iterate()
    for name, (cum, var) in out.items():
        assert _rel_rmse(cum, lt.target(name)) <= 1e-5, name
        assert _rel_rmse(var, lt.target(name, variance=True)) <= 1e-5, name
    # Density reduces moments: the target is the last iteration's value and
    # its variance slot the running mean, which is smoother than one iteration
    dens, dens_mean = out["Density"]
    assert float(dens_mean.sum()) > 0.0 and not np.array_equal(dens, dens_mean)


def test_bpt_variance_matches_oracle(oracle):
    spec = scenes.cornell_box(2, 48, 48)
    out = _render(spec, 3, {"Max. path length": 5, "Seed": 1}, ["Radiance", "Lightness"], iterations=3)
    bpt = oracle.OracleBidirPathTracer(oracle.OracleScene(spec), seed=1, max_path=5)
    for _ in range(3):
        bpt.iterate()
    for name, (cum, var) in out.items():
        assert _rel_rmse(cum, bpt.target(name)) <= 1e-5, name
        assert _rel_rmse(var, bpt.target(name, variance=True)) <= 1e-5, name


def test_vcm_variance_matches_oracle(oracle):
    spec = scenes.cornell_box(2, 48, 48)
    d = bindings.DllInterface()
    try:
        bindings.load_scene_spec(d, spec)
        assert d.render_enable_renderer(4, 0)
        for k, v in {"Max. path length": 5, "Seed": 1}.items():
            assert d.renderer_set_parameter_int(k, v)
        assert d.renderer_set_parameter_float("Relative merge radius", 0.02)
        for t in ("Radiance", "Lightness"):
            assert d.render_enable_render_target(t, True)
        for _ in range(3):
            d.render_iterate()
        out = {t: (d.get_target_image(t), d.get_target_image(t, variance=True)) for t in ("Radiance", "Lightness")}
    finally:
        d.close()
    vcm = oracle.OracleVcm(oracle.OracleScene(spec), seed=1, max_path=5, merge_radius=0.02)
    for _ in range(3):
        vcm.iterate()
    for name, (cum, var) in out.items():
        assert _rel_rmse(cum, vcm.target(name)) <= 1e-5, name
        assert _rel_rmse(var, vcm.target(name, variance=True)) <= 1e-5, name


def test_wireframe_border_variance_matches_oracle(oracle):
    spec = scenes.displaced_icosphere(2, subdiv=3, width=64, height=36)
    out = _render(spec, 2, {}, ["Border"], iterations=3)
    ow = oracle.OracleWireframe(oracle.OracleScene(spec), 1.0, 1000)
    for _ in range(3):
        ow.iterate()
    cum, var = out["Border"]
    assert np.array_equal(cum.view(np.uint32), ow.target().view(np.uint32))
    assert np.array_equal(var.view(np.uint32), ow.target(variance=True).view(np.uint32))
    assert float(var.max()) > 0.0


def test_variance_enable_disable_semantics():
    spec = scenes.cornell_box(0, 32, 32)
    d = bindings.DllInterface()
    try:
        bindings.load_scene_spec(d, spec)
        assert d.render_enable_renderer(0, 0)
        core, I = d.core, d.muffInst
        # enabling a variance records the target too
        assert d.render_disable_render_target("Hit ID", False)
        assert d.render_enable_render_target("Hit ID", True)
        assert core.render_is_render_target_enabled(I, b"Hit ID", 0) and core.render_is_render_target_enabled(I, b"Hit ID", 1)
        d.render_iterate()
        d.render_iterate()
        assert d.get_target_image("Hit ID", variance=True) is not None
        # disabling the variance keeps the target
        assert d.render_disable_render_target("Hit ID", True)
        assert core.render_is_render_target_enabled(I, b"Hit ID", 0)
        assert not core.render_is_render_target_enabled(I, b"Hit ID", 1)
        d.render_iterate()
        assert d.get_target_image("Hit ID") is not None
        with pytest.raises(bindings.MufflonError, match="does not record variance"):
            d.get_target_image("Hit ID", variance=True)
        # disabling without variance stops both
        assert d.render_enable_render_target("Hit ID", True)
        assert d.render_disable_render_target("Hit ID", False)
        assert not core.render_is_render_target_enabled(I, b"Hit ID", 0)
        assert not core.render_is_render_target_enabled(I, b"Hit ID", 1)
    finally:
        d.close()
