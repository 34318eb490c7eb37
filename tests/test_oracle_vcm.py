"""The oracle's vertex connection and merging (cpu_vcm.cpp restated) on its own,
on the CPU: it estimates the same image as the oracle's bidirectional path
tracer, its records add up to its image, merges carry light, the progressive
radius follows iteration^(-1/6), and the photon map's hash pieces (the bucket
count and the Wang hash that pairs a pixel with a light subpath) follow their
published definitions."""
import numpy as np
import pytest

from mufflon_b200 import scenes


def _wang(x):
    """Thomas Wang's 32-bit integer hash, written from its published steps."""
    m = 0xFFFFFFFF
    x = ((x ^ 61) ^ (x >> 16)) & m
    x = (x * 9) & m
    x = x ^ (x >> 4)
    x = (x * 0x27D4EB2D) & m
    return x ^ (x >> 15)


def test_wang_hash_matches_its_published_steps(oracle):
    rng = np.random.default_rng(5)
    xs = [0, 1, 2, 61, 65535, 65536, 0x7FFFFFFF, 0xFFFFFFFF] + [int(v) for v in rng.integers(0, 2**32, 200)]
    for x in xs:
        assert oracle.wang_hash(x) == _wang(x), x


def _is_prime(v):
    if v < 2:
        return False
    d = 2
    while d * d <= v:
        if v % d == 0:
            return False
        d += 1
    return True


@pytest.mark.parametrize("capacity", [1, 7, 100, 1536, 40 * 40 * 5, 480 * 270 * 10])
def test_photon_map_bucket_count(oracle, capacity):
    """The next prime above 1.15 x the capacity that is 3 mod 4
    (photon_map.hpp:216-229)."""
    v = oracle.vcm_map_size(capacity)
    base = int(np.float32(capacity) * np.float32(1.15))
    assert v > base and v % 4 == 3 and _is_prime(v)
    assert not any(_is_prime(u) and u % 4 == 3 for u in range(base + 1, v))


def _cornell(size=40):
    return scenes.cornell_box(1, width=size, height=size)


def test_vcm_estimates_the_bidirectional_image(oracle):
    """Connections, hits and merges weighted by the VCM balance heuristic sum
    to the same image as the bidirectional path tracer (200 iterations)."""
    sc = oracle.OracleScene(_cornell())
    v = oracle.OracleVcm(sc, seed=3, max_path=5, merge_radius=0.01)
    b = oracle.OracleBidirPathTracer(sc, seed=3, max_path=5)
    for _ in range(200):
        v.iterate()
        b.iterate()
    mv = v.target("Radiance").reshape(-1, 3).mean(0)
    mb = b.target("Radiance").reshape(-1, 3).mean(0)
    assert np.all(np.abs(mv / mb - 1.0) < 0.01), (mv, mb)
    lv = float(v.target("Lightness").mean())
    lb = float(b.target("Lightness").mean())
    assert lv > 0 and lb > 0


def test_vcm_records_add_up_and_merges_carry_light(oracle):
    spec = _cornell(24)
    m = 4
    v = oracle.OracleVcm(oracle.OracleScene(spec), seed=1, max_path=m, merge_radius=0.03)
    v.iterate()
    pix, val = v.records()
    img = np.zeros((spec.width * spec.height, 4), np.float64)
    for p, x in zip(pix, val):
        if p >= 0:
            img[p] += x
    got = v.target("Radiance").reshape(-1, 3)
    assert np.allclose(img[:, :3], got, rtol=1e-5, atol=1e-7)
    per = val.reshape(spec.width * spec.height, m * m + 2 * m, 4)
    merges = per[:, m * m + m:, :3]
    assert np.count_nonzero(np.any(merges > 0, axis=2)) > 20
    assert float(merges.sum()) > 0.01 * float(per[:, :, :3].sum())


def test_progressive_radius_changes_from_the_second_iteration(oracle):
    """iteration^(-1/6) is 1 for the first iteration: the records agree; the
    second iteration merges within a smaller radius."""
    spec = _cornell(24)
    a = oracle.OracleVcm(oracle.OracleScene(spec), seed=2, max_path=4, merge_radius=0.05, progressive=True)
    b = oracle.OracleVcm(oracle.OracleScene(spec), seed=2, max_path=4, merge_radius=0.05, progressive=False)
    a.iterate()
    b.iterate()
    assert np.array_equal(a.records()[1], b.records()[1])
    a.iterate()
    b.iterate()
    assert not np.array_equal(a.records()[1], b.records()[1])


def test_no_light_gives_no_photons(oracle):
    """Without any light there is no light subpath (the reference's emission
    is undefined there: its light choice divides by a zero flux); the view
    subpaths still run and the image stays black."""
    import dataclasses
    spec = scenes.displaced_icosphere(4, subdiv=3, width=16, height=12)
    spec = dataclasses.replace(spec, background=None, point_lights=np.zeros((0, 6), np.float32))
    v = oracle.OracleVcm(oracle.OracleScene(spec), seed=1, max_path=4, merge_radius=0.05)
    v.iterate()
    assert not v.target("Radiance").any()
    assert v.stats()["rays"] > 0
