"""The oracle's light tracer (lt_common.hpp restated) on its own, without a GPU.

* Light tracing and path tracing estimate the same image: without point
  lights (which the light tracer shows where they are seen, the path tracer
  never) the two oracles agree per path length within the noise of a few
  hundred iterations. This checks the restated emission sampling, camera
  projection and importance, the adjoint BSDF evaluation and the walk
  against an independent estimator.
* The connection records and the image agree: the first iteration's
  radiance is the records added per pixel in photon order.
* Photons from the environment light estimate the same image as the path
  tracer's background hits and next-event estimation.
"""
import dataclasses

import numpy as np
import pytest

from mufflon_b200 import scenes


def _block_means(img, b=8):
    h, w, c = img.shape
    return img[: h // b * b, : w // b * b].reshape(h // b, b, w // b, b, c).mean(axis=(1, 3))


@pytest.mark.parametrize("path_len", [1, 2])
def test_light_tracer_and_path_tracer_estimate_the_same_image(oracle, path_len):
    spec = scenes.emissive_panels(5, 6, 40, 0, width=48, height=32, emissive_triangles=12)
    S = oracle.OracleScene(spec)
    iters = 400
    lt = oracle.OracleLightTracer(S, seed=3, min_path=path_len, max_path=path_len)
    pt = oracle.OraclePathTracer(S, seed=5, min_path=path_len, max_path=path_len)
    for _ in range(iters):
        lt.iterate()
        pt.iterate()
    a, b = lt.target("Radiance"), pt.target("Radiance")
    # the mean over the image within 3 %
    ma, mb = a.mean(axis=(0, 1)), b.mean(axis=(0, 1))
    assert np.all(np.abs(ma - mb) <= 0.03 * mb), (ma, mb)
    # and 8x8-pixel block means within 25 % where the blocks are bright
    ba, bb = _block_means(a), _block_means(b)
    bright = bb > 0.2 * bb.max()
    assert np.all(np.abs(ba[bright] - bb[bright]) <= 0.25 * bb[bright])
    lt.close(); pt.close(); S.close()


def test_records_add_up_to_the_first_iteration(oracle):
    spec = scenes.emissive_panels(2, 3, 20, 2, width=40, height=30, emissive_triangles=5)
    S = oracle.OracleScene(spec)
    lt = oracle.OracleLightTracer(S, seed=1, max_path=5, density=True)
    lt.iterate()
    pix, val = lt.records()
    assert (pix >= 0).sum() > 100
    acc = np.zeros((30 * 40, 5), np.float32)
    np.add.at(acc, pix[pix >= 0], val[pix >= 0])
    assert np.array_equal(lt.target("Radiance").reshape(-1, 3), acc[:, :3])
    assert np.array_equal(lt.target("Lightness").reshape(-1), acc[:, 3])
    assert np.array_equal(lt.target("Density").reshape(-1), acc[:, 4])
    # a connection's path length never exceeds the maximum; slots past a photon's end stay empty
    assert pix.reshape(-1, 5).shape[0] == 30 * 40
    lt.close(); S.close()


def test_point_lights_are_seen_by_the_light_tracer_only(oracle):
    """The light vertex of a point light is connected to the camera
    (lights.hpp:263-265 evaluate_point), so a point light in view adds
    radiance at path length 1; the path tracer has nothing there."""
    spec = scenes.emissive_panels(5, 0, 0, 3, width=48, height=32)
    S = oracle.OracleScene(spec)
    lt = oracle.OracleLightTracer(S, seed=2, min_path=1, max_path=1)
    lt.iterate()
    pix, _ = lt.records()
    pt = oracle.OraclePathTracer(S, seed=2, min_path=1, max_path=1)
    pt.iterate()
    assert np.all(pt.target("Radiance") == 0.0)
    assert (pix >= 0).sum() > 100 and lt.target("Radiance").sum() > 0.0
    lt.close(); pt.close(); S.close()


def test_environment_photons_match_the_path_tracer(oracle):
    """With a colored background, photons also leave the environment
    (light_sampling.hpp:292-306): at path length 1 they show the background
    itself, at length 2 the ground lit by it; both estimates agree with the
    path tracer's."""
    spec = dataclasses.replace(scenes.emissive_panels(5, 0, 0, 0, width=48, height=32),
                               background=((0.3, 0.4, 0.5), (1.0, 1.0, 1.0)))
    S = oracle.OracleScene(spec)
    for path_len in (1, 2):
        lt = oracle.OracleLightTracer(S, seed=3, min_path=path_len, max_path=path_len)
        pt = oracle.OraclePathTracer(S, seed=5, min_path=path_len, max_path=path_len)
        for _ in range(300):
            lt.iterate()
            pt.iterate()
        ma, mb = lt.target("Radiance").mean(axis=(0, 1)), pt.target("Radiance").mean(axis=(0, 1))
        assert np.all(mb > 0.0) and np.all(np.abs(ma - mb) <= 0.03 * mb), (path_len, ma, mb)
        lt.close(); pt.close()
    S.close()
