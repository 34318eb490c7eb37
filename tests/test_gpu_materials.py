"""Torrance (GGX) with both shadowing models of the reference
(microfacet_specular.hpp:26-110): Smith with visible-normal sampling and
V-cavity with NDF sampling plus the mirrored-cavity choice and the
multi-bounce compensation. GPU renders against the oracle at several
roughnesses; hit ids exact, radiance within relative RMSE 1e-4."""
import dataclasses

import numpy as np
import pytest

from mufflon_b200 import bindings, scenes

pytestmark = pytest.mark.gpu


def _render_gpu(spec, params, iterations):
    d = bindings.DllInterface()
    try:
        bindings.load_scene_spec(d, spec)
        assert d.render_enable_renderer(0, 0)
        for k, v in params.items():
            assert d.renderer_set_parameter_int(k, v)
        d.render_enable_render_target("Radiance", False)
        d.render_enable_render_target("Hit ID", False)
        for _ in range(iterations):
            d.render_iterate()
        return d.get_target_image("Radiance").copy(), d.get_target_image("Hit ID").copy()
    finally:
        d.close()


@pytest.mark.parametrize("shadowing", [0, 1], ids=["vcavity", "smith"])
@pytest.mark.parametrize("roughness", [0.04, 0.3, 0.8])
@pytest.mark.parametrize("megakernel", [0, 1])
def test_torrance_shadowing_models_match_oracle(oracle, shadowing, roughness, megakernel):
    spec = scenes.displaced_icosphere(3, subdiv=4, width=64, height=36)
    mats = [dataclasses.replace(m, shadowing=shadowing, roughness=(roughness, roughness * 0.7))
            if m.type == scenes.MAT_TORRANCE else m for m in spec.materials]
    # the ground becomes glossy too, so paths bounce between two Torrance surfaces
    mats[1] = scenes.MaterialSpec(scenes.MAT_TORRANCE, albedo=(0.7, 0.7, 0.6), roughness=(roughness, roughness),
                                  shadowing=shadowing)
    spec = dataclasses.replace(spec, materials=mats)
    params = {"Seed": 2, "Max. path length": 6, "RR start depth": 3, "Megakernel": megakernel}
    img, hid = _render_gpu(spec, params, 2)
    pt = oracle.OraclePathTracer(oracle.OracleScene(spec), seed=2, max_path=6, rr_start=3)
    for _ in range(2):
        pt.iterate()
    ref = pt.target("Radiance")
    assert np.array_equal(hid, pt.target("Hit ID"))
    err = np.sqrt(np.mean((img - ref) ** 2)) / np.sqrt(np.mean(ref ** 2))
    assert err <= 1e-4, err


def test_vcavity_differs_from_smith():
    """The two models are different BRDFs: same scene, different images."""
    spec = scenes.displaced_icosphere(3, subdiv=4, width=48, height=27)
    imgs = []
    for sh in (0, 1):
        mats = [dataclasses.replace(m, shadowing=sh, roughness=(0.5, 0.5)) if m.type == scenes.MAT_TORRANCE else m
                for m in spec.materials]
        imgs.append(_render_gpu(dataclasses.replace(spec, materials=mats), {"Seed": 1}, 2)[0])
    assert not np.array_equal(imgs[0], imgs[1])
    assert np.isfinite(imgs[0]).all()
