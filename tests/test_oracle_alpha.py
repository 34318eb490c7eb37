"""CPU checks of the oracle's alpha test (intersection.cu:181-316) against
values computed here: a checkerboard quad lets rays through exactly where its
texel is below 0.5, a cut-out sphere shows its far side, and a fully cut
primitive is invisible to shadow rays too."""
import math

import numpy as np

from mufflon_b200 import scenes
from oracle import pyoracle


def _spec(lods, materials, textures, instance_lod=None):
    n = len(lods)
    il = np.arange(n, dtype=np.uint32) if instance_lod is None else np.asarray(instance_lod, np.uint32)
    return scenes.SceneSpec(lods, np.tile(scenes.identity34(), (len(il), 1)), il, materials,
                            np.zeros((0, 6), np.float32), None, (0.0, 0.0, 5.0), (0.0, 0.0, -1.0),
                            (0.0, 1.0, 0.0), math.radians(40.0), 16, 16, textures=textures, name="alpha_probe")


def _checker_quad(alpha):
    p, n = scenes._quad((-1, -1, 0), (1, -1, 0), (1, 1, 0), (-1, 1, 0))
    uv = np.array([(0, 0), (1, 0), (1, 1), (0, 1)], np.float32)
    quad = scenes._lod(p, n, uv, quads=np.arange(4, dtype=np.uint32).reshape(1, 4), mats=np.array([0], np.uint16))
    # a backstop behind it
    bp, bn = scenes._quad((-3, -3, -2), (3, -3, -2), (3, 3, -2), (-3, 3, -2))
    back = scenes._lod(bp, bn, uv, quads=np.arange(4, dtype=np.uint32).reshape(1, 4), mats=np.array([1], np.uint16))
    tex = np.zeros((4, 4, 4), np.float32)
    tex[..., 0] = (np.add.outer(np.arange(4), np.arange(4)) % 2).astype(np.float32)
    mats = [scenes.MaterialSpec(scenes.MAT_LAMBERT, alpha_texture=0 if alpha else -1), scenes.MaterialSpec(scenes.MAT_LAMBERT)]
    return _spec([quad, back], mats, [tex]), tex


def test_checkerboard_quad_cuts_where_the_texel_is_below_half():
    spec, tex = _checker_quad(True)
    sc = pyoracle.OracleScene(spec)
    # rays along -z through texel centres of the quad (u along x, v along y)
    c = (np.arange(4) + 0.5) / 4.0
    u, v = np.meshgrid(c, c, indexing="xy")
    org = np.stack([u.ravel() * 2 - 1, v.ravel() * 2 - 1, np.full(16, 3.0)], 1).astype(np.float32)
    rays = np.concatenate([org, np.tile(np.array([0, 0, -1], np.float32), (16, 1))], 1)
    t, inst, prim, _ = sc.trace_first(rays)
    texel = tex[(v.ravel() * 4).astype(int), (u.ravel() * 4).astype(int), 0]
    assert np.array_equal(inst == 0, texel >= 0.5)
    assert np.array_equal(inst == 1, texel < 0.5)
    assert np.allclose(t[inst == 0], 3.0) and np.allclose(t[inst == 1], 5.0)
    # without the alpha texture every ray stops at the quad
    _, inst2, _, _ = pyoracle.OracleScene(_checker_quad(False)[0]).trace_first(rays)
    assert (inst2 == 0).all()


def test_cut_sphere_shows_its_far_side_and_passes_shadow_rays():
    sph = np.array([(0.0, 0.0, 0.0, 1.0)], np.float32)
    lod = scenes._lod(np.zeros((0, 3), np.float32), np.zeros((0, 3), np.float32), np.zeros((0, 2), np.float32),
                      spheres=sph, sphere_mats=np.zeros(1, np.uint16))
    # u = atan2(n.z, n.x) / 2pi + 0.5: the half with n.z > 0 (u > 0.5) is cut
    tex = np.zeros((1, 2, 4), np.float32)
    tex[0, 0, 0] = 1.0
    spec = _spec([lod], [scenes.MaterialSpec(scenes.MAT_LAMBERT, alpha_texture=0)], [tex])
    sc = pyoracle.OracleScene(spec)
    # from +z the near side (n.z > 0) is cut, the far side (n.z < 0) is kept
    rays = np.array([[0.1, 0.2, 4.0, 0, 0, -1], [0.1, 0.2, -4.0, 0, 0, 1]], np.float32)
    t, inst, _, _ = sc.trace_first(rays)
    assert inst.tolist() == [0, 0]
    z = math.sqrt(1.0 - 0.1 ** 2 - 0.2 ** 2)
    assert abs(t[0] - (4.0 + z)) < 1e-5   # far root
    assert abs(t[1] - (4.0 - z)) < 1e-5   # near root, kept
    # a fully cut sphere stops neither closest-hit nor shadow rays
    tex0 = np.zeros((1, 1, 4), np.float32)
    sc0 = pyoracle.OracleScene(_spec([lod], [scenes.MaterialSpec(scenes.MAT_LAMBERT, alpha_texture=0)], [tex0]))
    assert (sc0.trace_first(rays)[1] == -1).all()
    a = np.array([[0, 0, 3]], np.float32)
    b = np.array([[0, 0, -3]], np.float32)
    assert not sc0.trace_any(a, b)[0]
    assert sc.trace_any(a, b)[0]


def test_alpha_scene_renders_differently_from_the_opaque_one():
    spec = scenes.alpha_cutouts(0, 32, 32)
    opaque = scenes.alpha_cutouts(0, 32, 32)
    for m in opaque.materials:
        m.alpha_texture = -1
    hits = []
    for s in (spec, opaque):
        pt = pyoracle.OraclePathTracer(pyoracle.OracleScene(s), seed=0, max_path=4)
        pt.iterate()
        hits.append(pt.target("Hit ID"))
    assert np.any(hits[0] != hits[1])
