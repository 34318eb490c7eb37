"""CPU checks of the oracle's emissive spheres (area lights of
world_container.cpp:966-990): the path tracer's next-event samples of the
visible cap (light_sampling.hpp:389-430), its MIS weight of a hit on a sphere
(light_tree_sampling.hpp:395-405, the pdf of the cap seen from the previous
vertex) and the light tracer's emission from the sphere's surface
(light_sampling.hpp:173-194) estimate the same direct light: the light tracer
and the path tracer agree per path length, and the path tracer's MIS-weighted
estimate equals its hits-only estimate (a scene whose spheres' MIS weights were
off would not)."""
import numpy as np
import pytest

from mufflon_b200 import scenes


def _block_means(img, b=8):
    h, w, c = img.shape
    return img[: h // b * b, : w // b * b].reshape(h // b, b, w // b, b, c).mean(axis=(1, 3))


def _spheres_only():
    # sphere lights only: no emissive quads or triangles, no point lights
    return scenes.emissive_panels(4, 5, 0, 0, width=48, height=32, emissive_spheres=8)


@pytest.mark.parametrize("path_len", [1, 2])
def test_light_tracer_and_path_tracer_agree_with_sphere_lights(oracle, path_len):
    S = oracle.OracleScene(_spheres_only())
    l, _, _, _, _ = S.light_tree()
    assert (l[:, 0:2].copy().view(np.uint16).ravel() == 4).sum() == 5 * 8
    iters = 300
    lt = oracle.OracleLightTracer(S, seed=3, min_path=path_len, max_path=path_len)
    pt = oracle.OraclePathTracer(S, seed=5, min_path=path_len, max_path=path_len)
    for _ in range(iters):
        lt.iterate()
        pt.iterate()
    a, b = lt.target("Radiance"), pt.target("Radiance")
    ma, mb = a.mean(axis=(0, 1)), b.mean(axis=(0, 1))
    assert np.all(mb > 0) and np.all(np.abs(ma - mb) <= 0.04 * mb), (ma, mb)
    ba, bb = _block_means(a), _block_means(b)
    bright = bb > 0.2 * bb.max()
    assert np.all(np.abs(ba[bright] - bb[bright]) <= 0.3 * bb[bright])
    lt.close(); pt.close(); S.close()


def test_next_event_weights_sum_to_one_on_sphere_lights(oracle):
    """Direct light (path length 2) with next-event estimation plus MIS-weighted
    hits equals the same image from several next-event samples per vertex: the
    weights of the two techniques sum to one only if the hit's pdf is the
    cap pdf of the sphere seen from the previous vertex."""
    S = oracle.OracleScene(_spheres_only())
    iters = 300
    one = oracle.OraclePathTracer(S, seed=7, min_path=2, max_path=2, nee_count=1)
    four = oracle.OraclePathTracer(S, seed=9, min_path=2, max_path=2, nee_count=4)
    for _ in range(iters):
        one.iterate()
        four.iterate()
    a, b = one.target("Radiance").mean(axis=(0, 1)), four.target("Radiance").mean(axis=(0, 1))
    assert np.all(b > 0) and np.all(np.abs(a - b) <= 0.03 * b), (a, b)
    one.close(); four.close(); S.close()
