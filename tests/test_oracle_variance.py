"""The oracle's variance targets follow output_handler_variance.hpp:7-31.

After n iterations the recorded variance of a channel is the unbiased sample
variance of its n per-iteration values (Welford's update, divided by n - 1),
and the light tracer's Density (a target that reduces moments,
render_targets.hpp:68-74) holds the last iteration's value with the running
mean in its variance slot. The per-iteration values are recovered from the
running means in float64, so the comparison allows for float32 rounding.
"""
import numpy as np

from mufflon_b200 import scenes


def _per_iteration(means):
    """x_k = (k + 1) * M_k - k * M_(k-1) from the running means M_0..M_n."""
    m = [np.asarray(a, np.float64) for a in means]
    return [m[0]] + [(k + 1) * m[k] - k * m[k - 1] for k in range(1, len(m))]


def _rel_rmse(a, b):
    return float(np.sqrt(np.mean((a - b) ** 2)) / max(np.sqrt(np.mean(b ** 2)), 1e-30))


def test_pt_variance_is_the_sample_variance(oracle):
    spec = scenes.cornell_box(1, 32, 32)
    pt = oracle.OraclePathTracer(oracle.OracleScene(spec), seed=3, max_path=6)
    means = []
    for _ in range(6):
        pt.iterate()
        means.append(pt.target("Radiance"))
    xs = np.stack(_per_iteration(means))
    expected = xs.var(axis=0, ddof=1)
    got = pt.target("Radiance", variance=True).astype(np.float64)
    assert expected.max() > 0
    assert _rel_rmse(got, expected) <= 1e-3


def test_first_iteration_variance_is_zero(oracle):
    spec = scenes.cornell_box(1, 16, 16)
    pt = oracle.OraclePathTracer(oracle.OracleScene(spec), seed=0, max_path=4)
    pt.iterate()
    assert np.all(pt.target("Radiance", variance=True) == 0.0)
    assert np.all(pt.target("Hit ID", variance=True) == 0.0)


def test_lt_density_reduces_moments(oracle):
    spec = scenes.emissive_panels(2, 3, 20, 2, width=40, height=30, emissive_triangles=5)
    lt = oracle.OracleLightTracer(oracle.OracleScene(spec), seed=1, max_path=5, density=True)
    dens = []
    for _ in range(4):
        lt.iterate()
        pix, val = lt.records()
        acc = np.zeros(30 * 40, np.float32)
        np.add.at(acc, pix[pix >= 0], val[pix >= 0][:, 4])
        assert np.array_equal(lt.target("Density").reshape(-1), acc)  # the iteration's value
        dens.append(acc.astype(np.float64))
    mean = lt.target("Density", variance=True).reshape(-1).astype(np.float64)
    assert _rel_rmse(mean, np.mean(dens, axis=0)) <= 1e-5
