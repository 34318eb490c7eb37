"""The light list and light tree built on the GPU (core/light_build.cu) against
the oracle's CPU build (light_tree.cpp:120-447 restated), byte for byte:
lights in Hilbert order, node fluxes, indices and types, the sorted
(instance, primitive) -> node-path codes and the root flux. Light counts cover
the tree's shapes: one leaf, powers of two, odd and even numbers of extra
bottom nodes, point lights only, area lights only, triangle and quad emitters,
a mirroring instance."""
import numpy as np
import pytest

from mufflon_b200 import bindings, scenes

pytestmark = pytest.mark.gpu

# (instances, emissive quads per instance, point lights, emissive triangles per instance,
#  emissive spheres per instance)
CASES = [(0, 0, 1, 0, 0), (0, 0, 2, 0, 0), (1, 1, 0, 0, 0), (1, 1, 1, 0, 0), (2, 1, 1, 0, 0), (1, 7, 0, 0, 0),
         (2, 4, 1, 0, 0), (1, 8, 0, 0, 0), (3, 17, 3, 0, 0), (5, 3, 0, 0, 0), (8, 125, 1, 0, 0), (16, 256, 1, 0, 0),
         (64, 1024, 2, 0, 0), (1, 0, 0, 1, 0), (2, 3, 1, 5, 0), (5, 40, 2, 17, 0), (32, 100, 1, 37, 0),
         (1, 0, 0, 0, 1), (3, 2, 1, 1, 4), (16, 20, 1, 3, 11)]


def _gpu_tree(spec):
    d = bindings.DllInterface()
    try:
        bindings.load_scene_spec(d, spec)
        return d.light_tree()
    finally:
        d.close()


@pytest.mark.parametrize("case", CASES, ids=[f"{m}x({k}q+{t}t+{sp}s)+{p}" for m, k, p, t, sp in CASES])
def test_gpu_light_tree_equals_oracle(oracle, case):
    m, k, p, t, sp = case
    spec = scenes.emissive_panels(11 + m + k + p + t + sp, m, k, p, width=16, height=16, emissive_triangles=t,
                                  emissive_spheres=sp)
    gl, gn, gk, gc, grf = _gpu_tree(spec)
    ol, on, ok, oc, orf = oracle.OracleScene(spec).light_tree()
    n = m * (k + t + sp) + p
    assert len(gl) == len(ol) == n
    assert len(gn) == len(on) == max(n - 1, 0)
    assert len(gk) == len(ok) == m * (k + t + sp)
    assert np.array_equal(gl, ol), "lights differ (order or values)"
    assert np.array_equal(gn, on), "tree nodes differ"
    assert np.array_equal(gk, ok) and np.array_equal(gc, oc), "node-path codes differ"
    assert np.float32(grf).view(np.uint32) == np.float32(orf).view(np.uint32)


@pytest.mark.parametrize("tris,spheres,megakernel", [(0, 0, 0), (12, 0, 0), (3, 9, 0), (3, 9, 1)],
                         ids=["quads", "quads_tris", "spheres_wavefront", "spheres_megakernel"])
def test_render_with_many_area_lights_matches_oracle(oracle, tris, spheres, megakernel):
    spec = scenes.emissive_panels(5, 6, 40, 2, width=64, height=48, emissive_triangles=tris, emissive_spheres=spheres)
    d = bindings.DllInterface()
    try:
        bindings.load_scene_spec(d, spec)
        assert d.render_enable_renderer(0, 0)
        for name, v in {"Seed": 4, "Max. path length": 5, "RR start depth": 2, "Megakernel": megakernel}.items():
            assert d.renderer_set_parameter_int(name, v)
        d.render_enable_render_target("Radiance", False)
        d.render_enable_render_target("Hit ID", False)
        for _ in range(2):
            d.render_iterate()
        img, hid = d.get_target_image("Radiance"), d.get_target_image("Hit ID")
    finally:
        d.close()
    pt = oracle.OraclePathTracer(oracle.OracleScene(spec), seed=4, max_path=5, rr_start=2)
    for _ in range(2):
        pt.iterate()
    ref = pt.target("Radiance")
    assert np.array_equal(hid, pt.target("Hit ID"))
    assert np.sqrt(np.mean((img - ref) ** 2)) <= 1e-4 * np.sqrt(np.mean(ref ** 2))


def test_sphere_lights_in_the_light_tree():
    """Emissive spheres become area lights (world_container.cpp:966-990): one
    sphere light per emissive sphere of every instance, its radius scaled by
    the instance (the instances of emissive_panels are scaled by 0.7-1.5)."""
    spec = scenes.emissive_panels(2, 2, 3, 1, width=16, height=16, emissive_spheres=2)
    lights = _gpu_tree(spec)[0]
    types = lights[:, 0:2].copy().view(np.uint16).ravel()
    radius = lights[:, 108:112].copy().view(np.float32).ravel()[types == 4]
    assert len(radius) == 2 * 2
    sph = spec.lods[1].spheres[[1, 2], 3]  # the two emissive spheres of the panel set
    scales = [1.0 / np.linalg.norm(spec.world_to_instance[i].reshape(3, 4)[:, 0]) for i in (1, 2)]
    expect = np.array([s * r for s in scales for r in sph])
    assert np.allclose(np.sort(radius), np.sort(expect), rtol=1e-5)
