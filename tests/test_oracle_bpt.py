"""The oracle's bidirectional path tracer (cpu_bpt.cpp restated) on its own,
without a GPU: it estimates the same image as the path tracer per path
length, and its recorded contributions add up to the image."""
import numpy as np
import pytest

from mufflon_b200 import scenes


@pytest.mark.parametrize("path_len", [1, 2, 3])
def test_bpt_and_pt_estimate_the_same_image(oracle, path_len):
    spec = scenes.cornell_box(1, width=32, height=32)
    S = oracle.OracleScene(spec)
    b = oracle.OracleBidirPathTracer(S, seed=3, min_path=path_len, max_path=path_len)
    p = oracle.OraclePathTracer(S, seed=5, min_path=path_len, max_path=path_len)
    for _ in range(200):
        b.iterate()
        p.iterate()
    mb, mp = b.target("Radiance").mean(axis=(0, 1)), p.target("Radiance").mean(axis=(0, 1))
    assert np.all(np.abs(mb - mp) <= 0.03 * mp), (mb, mp)
    b.close(); p.close(); S.close()


def test_bpt_records_add_up_to_the_first_iteration(oracle):
    spec = scenes.emissive_panels(2, 3, 20, 2, width=24, height=16, emissive_triangles=5)
    S = oracle.OracleScene(spec)
    b = oracle.OracleBidirPathTracer(S, seed=1, max_path=4)
    b.iterate()
    pix, val = b.records()
    assert (pix >= 0).sum() > 100
    acc = np.zeros((16 * 24, 4), np.float32)
    np.add.at(acc, pix[pix >= 0], val[pix >= 0])
    assert np.array_equal(b.target("Radiance").reshape(-1, 3), acc[:, :3])
    assert np.array_equal(b.target("Lightness").reshape(-1), acc[:, 3])
    b.close(); S.close()
