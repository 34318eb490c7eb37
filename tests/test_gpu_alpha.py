"""Alpha-tested surfaces (intersection.cu:181-316, any_intersection
intersection.cu:624-753): a material's alpha texture (MaterialParams.alpha)
cuts a triangle, quad or sphere where its first channel is below 0.5; a cut
quad or sphere falls back to its second root. The path tracer (both
schedules), the light tracer, the bidirectional path tracer and the shadow and
first-hit queries all test alpha; the wireframe renderer does not
(first_intersection<dev, false>, wireframe_common.hpp:108). Every GPU result is
compared with the oracle: hit ids and connection records bit for bit,
radiance within relative RMSE 1e-4 (path tracer) or 1e-5 (atomically summed
images)."""
import copy

import numpy as np
import pytest

from mufflon_b200 import bindings, scenes

pytestmark = pytest.mark.gpu

KERNELS = {"wavefront": 0, "megakernel": 1}


def rel_rmse(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.sqrt(np.mean((a - b) ** 2)) / max(np.sqrt(np.mean(b * b)), 1e-30))


def _opaque(spec):
    s = copy.deepcopy(spec)
    for m in s.materials:
        m.alpha_texture = -1
    return s


def _session(spec, renderer):
    d = bindings.DllInterface()
    bindings.load_scene_spec(d, spec)
    assert d.render_enable_renderer(renderer, 0)
    return d


@pytest.mark.parametrize("kernel", list(KERNELS))
def test_pt_alpha_matches_oracle(oracle, kernel):
    spec = scenes.alpha_cutouts(1, 96, 80)
    d = _session(spec, 0)
    try:
        for k, v in {"Seed": 3, "Max. path length": 7, "NEE count": 2, "Min. path length": 1,
                     "Megakernel": KERNELS[kernel]}.items():
            assert d.renderer_set_parameter_int(k, v)
        d.render_enable_render_target("Radiance", False)
        d.render_enable_render_target("Hit ID", False)
        pt = oracle.OraclePathTracer(oracle.OracleScene(spec), seed=3, min_path=1, max_path=7, nee_count=2)
        d.render_iterate()
        pt.iterate()
        hid, ohid = d.get_target_image("Hit ID").copy(), pt.target("Hit ID")
        for _ in range(2):
            d.render_iterate()
            pt.iterate()
        img, ref = d.get_target_image("Radiance").copy(), pt.target("Radiance")
        stats = d.render_stats()
    finally:
        d.close()
    assert np.array_equal(hid, ohid)
    assert rel_rmse(img, ref) <= 1e-4, rel_rmse(img, ref)
    assert stats["errors"] == 0
    # the cut-outs change what the camera sees
    sc = oracle.OracleScene(_opaque(spec))
    po = oracle.OraclePathTracer(sc, seed=3, min_path=1, max_path=7, nee_count=2)
    po.iterate()
    changed = np.any(po.target("Hit ID") != ohid, axis=-1)
    assert changed.mean() > 0.05, changed.mean()


def _rays_at(spec, sc, n, seed):
    """Rays from the camera and from random interior points towards the cut-out objects."""
    rng = np.random.default_rng(seed)
    a = sc.aabb()
    org = np.concatenate([np.tile(np.array(spec.cam_pos, np.float32), (n // 2, 1)),
                          rng.uniform(a[:3], a[3:], (n - n // 2, 3)).astype(np.float32)])
    tgt = rng.uniform((-0.95, -1.0, -0.95), (0.95, 0.95, 0.6), (n, 3)).astype(np.float32)
    d = tgt - org
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    return np.concatenate([org, d.astype(np.float32)], 1)


@pytest.mark.parametrize("kernel", list(KERNELS))
def test_first_hits_and_shadow_rays_with_alpha(dll, oracle, kernel):
    spec = scenes.alpha_cutouts(2, 64, 64)
    dll.world_clear_all()
    bindings.load_scene_spec(dll, spec)
    assert dll.render_enable_renderer(0, 0)
    assert dll.renderer_set_parameter_int("Megakernel", KERNELS[kernel])
    sc = oracle.OracleScene(spec)
    rays = _rays_at(spec, sc, 40000, 4)
    gt, gi, gp, gs = dll.trace_rays(rays)
    ot, oi, op, os_ = sc.trace_first(rays)
    assert np.array_equal(gi, oi) and np.array_equal(gp, op)
    assert np.array_equal(gt.view(np.uint32), ot.view(np.uint32))
    assert np.array_equal(gs.view(np.uint32), os_.view(np.uint32))
    # the same rays without the cut-outs hit something else often enough
    st, si, sp_, _ = oracle.OracleScene(_opaque(spec)).trace_first(rays)
    assert np.mean((si != oi) | (sp_ != op)) > 0.05
    rng = np.random.default_rng(8)
    box = sc.aabb()
    a = rng.uniform(box[:3], box[3:], (30000, 3)).astype(np.float32)
    b = rng.uniform(box[:3], box[3:], (30000, 3)).astype(np.float32)
    occ = dll.trace_occlusion(a, b)
    assert np.array_equal(occ, sc.trace_any(a, b))
    assert not np.array_equal(occ, oracle.OracleScene(_opaque(spec)).trace_any(a, b))


def test_lt_alpha_connections_match_oracle(oracle):
    spec = scenes.alpha_cutouts(3, 64, 64)
    lt = oracle.OracleLightTracer(oracle.OracleScene(spec), seed=5, min_path=0, max_path=6)
    d = _session(spec, 1)
    try:
        for k, v in {"Seed": 5, "Max. path length": 6, "Record connections": 1}.items():
            assert d.renderer_set_parameter_int(k, v)
        d.render_enable_render_target("Radiance", False)
        for it in range(2):
            d.render_iterate()
            lt.iterate()
            gp, gv = d.lt_records(6)
            op, ov = lt.records()
            assert np.array_equal(gp, op), f"iteration {it}: {np.sum(gp != op)} slots differ"
            assert np.array_equal(gv.view(np.uint32), ov.view(np.uint32))
            assert (gp >= 0).sum() > 50
        img = d.get_target_image("Radiance").copy()
    finally:
        d.close()
    assert rel_rmse(img, lt.target("Radiance")) <= 1e-5


def test_bpt_alpha_contributions_match_oracle(oracle):
    spec = scenes.alpha_cutouts(4, 48, 48)
    ob = oracle.OracleBidirPathTracer(oracle.OracleScene(spec), seed=7, min_path=0, max_path=5)
    d = _session(spec, 3)
    try:
        for k, v in {"Seed": 7, "Max. path length": 5, "Record connections": 1}.items():
            assert d.renderer_set_parameter_int(k, v)
        d.render_enable_render_target("Radiance", False)
        for it in range(2):
            d.render_iterate()
            ob.iterate()
            gp, gv = d.bpt_records(5)
            op, ov = ob.records()
            assert np.array_equal(gp, op), f"iteration {it}"
            assert np.array_equal(gv.view(np.uint32), ov.view(np.uint32)), f"iteration {it}"
        img = d.get_target_image("Radiance").copy()
    finally:
        d.close()
    assert rel_rmse(img, ob.target("Radiance")) <= 1e-5


def test_vcm_alpha_contributions_match_oracle(oracle):
    """Connections, hits and merges with cut-out surfaces: the light walk,
    the view walk and the connections' shadow rays all pass through the
    alpha test."""
    spec = scenes.alpha_cutouts(4, 48, 48)
    ov_ = oracle.OracleVcm(oracle.OracleScene(spec), seed=7, min_path=0, max_path=5, merge_radius=0.02)
    d = _session(spec, 4)
    try:
        for k, v in {"Seed": 7, "Max. path length": 5, "Record connections": 1}.items():
            assert d.renderer_set_parameter_int(k, v)
        assert d.renderer_set_parameter_float("Relative merge radius", 0.02)
        d.render_enable_render_target("Radiance", False)
        for it in range(2):
            d.render_iterate()
            ov_.iterate()
            gp, gv = d.vcm_records(5)
            op, ov = ov_.records()
            assert np.array_equal(gp, op), f"iteration {it}"
            assert np.array_equal(gv.view(np.uint32), ov.view(np.uint32)), f"iteration {it}"
        img = d.get_target_image("Radiance").copy()
    finally:
        d.close()
    assert rel_rmse(img, ov_.target("Radiance")) <= 1e-5


def test_wireframe_ignores_alpha(oracle):
    spec = scenes.alpha_cutouts(5, 64, 64, background=False)
    imgs = []
    for s in (spec, _opaque(spec)):
        d = _session(s, 2)
        try:
            d.render_enable_render_target("Border", False)
            d.render_iterate()
            imgs.append(d.get_target_image("Border").copy())
        finally:
            d.close()
    assert np.array_equal(imgs[0].view(np.uint32), imgs[1].view(np.uint32))
    ow = oracle.OracleWireframe(oracle.OracleScene(spec), 1.0, 1000)
    ow.iterate()
    ref = ow.target()
    differ = np.any(imgs[0].view(np.uint32) != ref.view(np.uint32), axis=-1)
    assert differ.sum() <= 2, np.argwhere(differ)
