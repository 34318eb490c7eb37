"""The oracle's wireframe renderer (wireframe_common.hpp:93-180) on the CPU:
limiting cases of its two parameters, and the per-pixel generator stream."""
import numpy as np

from mufflon_b200 import scenes


def _border(oracle, spec, line_width, depth, iterations=1):
    w = oracle.OracleWireframe(oracle.OracleScene(spec), line_width, depth)
    for _ in range(iterations):
        w.iterate(2)
    return w.target()


def test_wide_line_paints_every_hit_pixel(oracle):
    """With a line wider than the image every first hit is an edge: the
    Cornell box is closed around the camera's view, so all pixels are white."""
    spec = scenes.cornell_box(1, width=32, height=32)
    img = _border(oracle, spec, 1e9, 1000)
    assert np.all(img == 1.0)


def test_zero_depth_is_black_and_edges_are_sparse(oracle):
    spec = scenes.cornell_box(1, width=32, height=32)
    assert np.all(_border(oracle, spec, 1.0, 0) == 0.0)
    img = _border(oracle, spec, 1.0, 1000)
    white = float(np.mean(img[..., 0] == 1.0))
    assert 0.0 < white < 0.5
    assert set(np.unique(img)) <= {0.0, 1.0}


def test_running_mean_over_iterations(oracle):
    """Jittered camera rays move across edges between iterations: the mean
    of two iterations takes the values 0, 1/2 and 1."""
    spec = scenes.cornell_box(1, width=32, height=32)
    img = _border(oracle, spec, 1.0, 1000, iterations=2)
    assert set(np.unique(img)) <= {0.0, 0.5, 1.0}
    assert np.any(img == 0.5)
