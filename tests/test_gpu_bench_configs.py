"""Parity at the benchmark workloads' own sizes.

The bench's headline number is measured on the 1 310 720-triangle displaced
icosphere at 1920x1080 (16 spp, path length 10, point light + environment),
and its instanced workload on 4 096 instances of 10 meshes plus 20 000 spheres
at 1920x1080 (path length 12, Russian roulette from length 3). These tests
render exactly those scenes with exactly those settings through the C API and
compare them with the oracle (the CPU restatement of the reference's path
tracer, cpu_pt.cpp:18-45 and pt_common.hpp:75-156):

  * the first-hit ids of the first iteration bit for bit;
  * the cumulative radiance and hit ids after the last iteration, radiance
    within relative RMSE 1e-4.

The icosphere runs all 16 samples of a bench frame; the instanced scene runs
2 samples (about 7 s of oracle time per sample on 16 host cores).
"""
import numpy as np
import pytest

from mufflon_b200 import bindings, scenes

pytestmark = pytest.mark.gpu


def _rel_rmse(a, b):
    a = a.astype(np.float64)
    b = b.astype(np.float64)
    return float(np.sqrt(np.mean((a - b) ** 2)) / np.sqrt(np.mean(b ** 2)))


def _compare(oracle, spec, params, spp):
    d = bindings.DllInterface()
    try:
        bindings.load_scene_spec(d, spec)
        assert d.render_enable_renderer(0, 0)
        for k, v in params.items():
            assert d.renderer_set_parameter_int(k, v)
        d.render_enable_render_target("Hit ID", False)
        d.render_iterate()
        first_hits = d.get_target_image("Hit ID").copy()
        for _ in range(spp - 1):
            d.render_iterate()
        img = d.get_target_image("Radiance").copy()
        hid = d.get_target_image("Hit ID").copy()
        assert d.render_stats()["errors"] == 0
    finally:
        d.close()
    pt = oracle.OraclePathTracer(oracle.OracleScene(spec), seed=params.get("Seed", 0),
                                 max_path=params["Max. path length"], rr_start=params.get("RR start depth", 0))
    pt.iterate()
    assert np.array_equal(first_hits, pt.target("Hit ID")), "first-hit ids differ from the oracle"
    for _ in range(spp - 1):
        pt.iterate()
    ref = pt.target("Radiance")
    assert np.array_equal(hid, pt.target("Hit ID")), "cumulative hit ids differ from the oracle"
    err = _rel_rmse(img, ref)
    assert err <= 1e-4, f"radiance relative RMSE {err}"
    return err


def test_bench_icosphere_1080p_16spp_matches_oracle(oracle):
    spec = scenes.displaced_icosphere(0, subdiv=8, width=1920, height=1080)
    assert spec.num_prims == 1_310_721  # 20 * 4^8 triangles + the ground quad
    _compare(oracle, spec, {"Max. path length": 10}, spp=16)


def test_bench_instanced_1080p_matches_oracle(oracle):
    spec = scenes.instanced_scene(0, width=1920, height=1080)
    assert len(spec.instance_lod) == 4096 + 1 and len(spec.lods[-1].spheres) == 20_000
    _compare(oracle, spec, {"Max. path length": 12, "RR start depth": 3}, spp=2)
