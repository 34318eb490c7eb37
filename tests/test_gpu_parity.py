"""GPU-vs-oracle parity through the C ABI.

Integer and index results (sorted keys, BVH topology and nodes, first-hit
primitive ids) must be bit-exact. Radiance must be within relative RMSE 1e-4
of the CPU oracle at matched samples per pixel (the implementation aims for
bit equality; 1e-4 is the stated tolerance).
"""
import numpy as np
import pytest

from mufflon_b200 import bindings, scenes

pytestmark = pytest.mark.gpu

RMSE_TOL = 1e-4


def rel_rmse(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    den = np.sqrt(np.mean(b * b))
    return float(np.sqrt(np.mean((a - b) ** 2)) / max(den, 1e-30))


@pytest.mark.parametrize("n", [1, 2, 3, 255, 4095, 4096, 4097, 100_003, (1 << 20) + 7])
def test_sort_pairs_is_stable_radix_sort(dll, n):
    rng = np.random.default_rng(n)
    keys = rng.integers(0, 1 << 63, n, dtype=np.uint64)
    keys[rng.integers(0, n, n // 3)] = keys[0]  # duplicates
    keys[: n // 7] = rng.integers(0, 16, n // 7).astype(np.uint64)
    vals = np.arange(n, dtype=np.int32)
    k, v = bindings.sort_pairs(dll, keys, vals)
    order = np.argsort(keys, kind="stable")
    assert np.array_equal(k, keys[order])
    assert np.array_equal(v, vals[order])


def _compare_bvh(dll, oracle, lod):
    spec = scenes.SceneSpec([lod], np.array([scenes.identity34()]), np.array([0], np.uint32),
                            [scenes.MaterialSpec(0)], np.zeros((0, 6), np.float32), None,
                            (0, 0, 3), (0, 0, -1), (0, 1, 0), 0.8, 8, 8)
    sc = oracle.OracleScene(spec)
    om, op, onodes, oprim, oni = sc.bvh(0)
    gm, gp, gnodes, gprim, gni, _ = bindings.lbvh_build(dll, lod)
    n = lod.num_prims
    if n > 1:
        assert np.array_equal(gm, om), "Morton codes / sort order differ"
        assert np.array_equal(gp, op), "Karras parents differ"
    assert gni == oni, f"internal nodes after collapse: gpu {gni} oracle {oni}"
    assert np.array_equal(gprim, oprim), "primitive order differs"
    assert np.array_equal(gnodes.view(np.uint32), onodes.view(np.uint32)), "collapsed nodes differ"


def _random_tri_lod(n, seed):
    rng = np.random.default_rng(seed)
    c = rng.uniform(-5, 5, (n, 3))
    v = (c[:, None, :] + rng.normal(scale=0.2, size=(n, 3, 3))).reshape(-1, 3)
    f = np.arange(3 * n, dtype=np.uint32).reshape(n, 3)
    return scenes._lod(v, np.zeros_like(v), np.zeros((len(v), 2)), tris=f)


def _mixed_lod(seed):
    rng = np.random.default_rng(seed)
    nt, nq, ns = 300, 200, 150
    v = rng.uniform(-3, 3, (3 * nt + 4 * nq, 3))
    tris = np.arange(3 * nt, dtype=np.uint32).reshape(nt, 3)
    quads = (3 * nt + np.arange(4 * nq, dtype=np.uint32)).reshape(nq, 4)
    sph = np.concatenate([rng.uniform(-3, 3, (ns, 3)), rng.uniform(0.01, 0.3, (ns, 1))], 1)
    return scenes._lod(v, np.zeros_like(v), np.zeros((len(v), 2)), tris=tris, quads=quads,
                       mats=np.zeros(nt + nq, np.uint16), spheres=sph.astype(np.float32),
                       sphere_mats=np.zeros(ns, np.uint16))


def _single_lod_spec(lod):
    """One instance of `lod`, a Lambert material, a camera looking down -z."""
    return scenes.SceneSpec(lods=[lod], world_to_instance=scenes.identity34().reshape(1, 12),
                            instance_lod=np.zeros(1, np.uint32), materials=[scenes.MaterialSpec(type=0)],
                            point_lights=np.zeros((0, 6), np.float32), background=None, cam_pos=(0.5, 0.5, 8.0),
                            cam_dir=(0.0, 0.0, -1.0), cam_up=(0.0, 1.0, 0.0), vfov=0.8, width=64, height=64,
                            name="mixed")


@pytest.mark.parametrize("which", ["walls", "box", "light", "random_2", "random_5000", "mixed", "ico5", "ico7"])
def test_lbvh_bit_exact(dll, oracle, which):
    if which in ("walls", "box", "light"):
        spec = scenes.cornell_box(0)
        lod = spec.lods[{"walls": 0, "box": 1, "light": 3}[which]]
    elif which.startswith("random"):
        lod = _random_tri_lod(int(which.split("_")[1]), 11)
    elif which == "mixed":
        lod = _mixed_lod(5)
    else:
        v, f = scenes.displaced_sphere_mesh(int(which[3:]), 2)
        lod = scenes._lod(v, scenes.vertex_normals(v, f), scenes.spherical_uv(v), tris=f)
    _compare_bvh(dll, oracle, lod)


@pytest.mark.parametrize("which", ["walls", "random_5000", "mixed", "ico7", "ico8"])
def test_lbvh_30bit_morton_bit_exact(dll, oracle, which):
    """The reference's alternative 30-bit Morton code (build_lbvh.cu:59-69),
    mufflon_lbvh_build_ex(mortonBits = 30): sorted codes, Karras parents,
    collapsed nodes and primitive order equal to the oracle's build on 32-bit
    keys, though the GPU keeps the codes in 64-bit keys and sorts 4 bytes."""
    if which == "walls":
        lod = scenes.cornell_box(0).lods[0]
    elif which.startswith("random"):
        lod = _random_tri_lod(int(which.split("_")[1]), 12)
    elif which == "mixed":
        lod = _mixed_lod(6)
    else:
        v, f = scenes.displaced_sphere_mesh(int(which[3:]), 2)
        lod = scenes._lod(v, scenes.vertex_normals(v, f), scenes.spherical_uv(v), tris=f)
    spec = scenes.SceneSpec([lod], np.array([scenes.identity34()]), np.array([0], np.uint32),
                            [scenes.MaterialSpec(0)], np.zeros((0, 6), np.float32), None,
                            (0, 0, 3), (0, 0, -1), (0, 1, 0), 0.8, 8, 8)
    sc = oracle.OracleScene(spec)
    sc.rebuild_lod_bvhs(30)
    om, op, onodes, oprim, oni = sc.bvh(0)
    gm, gp, gnodes, gprim, gni, _ = bindings.lbvh_build(dll, lod, morton_bits=30)
    assert gm.max() < (1 << 30)
    assert np.array_equal(gm, om) and np.array_equal(gp, op)
    assert gni == oni and np.array_equal(gprim, oprim)
    assert np.array_equal(gnodes.view(np.uint32), onodes.view(np.uint32))


def test_lbvh_bit_exact_full_icosphere(dll, oracle):
    """The 1 310 720-triangle mesh of the 1080p workload."""
    spec = scenes.displaced_icosphere(0, subdiv=8, width=16, height=16)
    _compare_bvh(dll, oracle, spec.lods[0])


# "wavefront": stage kernels over the 8-wide hierarchies; "megakernel": one
# kernel over the binary (reference-layout) hierarchies.
KERNELS = {"wavefront": 0, "megakernel": 1}
DEFAULT_PARAMS = {"Seed": 0, "Min. path length": 0, "Max. path length": 16, "NEE count": 1,
                  "RR start depth": 0, "Megakernel": 0, "Wavefront bounces": 2, "Tail paths": 98304, "Iteration graph": 1,
                  "Planned tail": 1, "Ray sort bits": 12, "Ray sort direction bits": 3}


def _load(dll, spec):
    dll.world_clear_all()
    bindings.load_scene_spec(dll, spec)
    assert dll.render_enable_renderer(0, 0)
    for name, value in DEFAULT_PARAMS.items():  # the library instance is shared by all tests
        assert dll.renderer_set_parameter_int(name, value)


def _camera_rays(spec, n, seed):
    rng = np.random.default_rng(seed)
    d = np.array(spec.cam_dir, np.float64)
    d /= np.linalg.norm(d)
    dirs = d + rng.normal(scale=0.35, size=(n, 3))
    dirs /= np.linalg.norm(dirs, axis=1, keepdims=True)
    org = np.tile(np.array(spec.cam_pos, np.float64), (n, 1))
    return np.concatenate([org, dirs], 1).astype(np.float32)


def _interior_rays(spec, oracle_scene, n, seed):
    rng = np.random.default_rng(seed)
    a = oracle_scene.aabb()
    org = rng.uniform(a[:3], a[3:], (n, 3))
    dirs = rng.normal(size=(n, 3))
    dirs /= np.linalg.norm(dirs, axis=1, keepdims=True)
    return np.concatenate([org, dirs], 1).astype(np.float32)


def _small_instanced(seed=0):
    return scenes.instanced_scene(seed, num_meshes=4, num_instances=64, num_spheres=300,
                                  tri_range=(2000, 8000), width=64, height=48)


@pytest.mark.parametrize("kernel", list(KERNELS))
@pytest.mark.parametrize("scene", ["cornell", "icosphere6", "instanced", "mixed"])
def test_first_hit_bit_exact(dll, oracle, scene, kernel):
    """Closest hits over the 8-wide hierarchies ("wavefront") and the binary ones ("megakernel")."""
    if scene == "cornell":
        spec = scenes.cornell_box(3)
    elif scene == "icosphere6":
        spec = scenes.displaced_icosphere(1, subdiv=6, width=64, height=36)
    elif scene == "mixed":
        spec = _single_lod_spec(_mixed_lod(7))
    else:
        spec = _small_instanced(2)
    _load(dll, spec)
    assert dll.renderer_set_parameter_int("Megakernel", KERNELS[kernel])
    sc = oracle.OracleScene(spec)
    rays = np.concatenate([_camera_rays(spec, 20000, 1), _interior_rays(spec, sc, 20000, 2)])
    if scene == "instanced":
        # aim half of the interior rays at instance origins (the scene is sparse)
        w2i = spec.world_to_instance.reshape(-1, 3, 4).astype(np.float64)
        centers = np.stack([-np.linalg.solve(m[:, :3], m[:, 3]) for m in w2i])
        tgt = centers[np.random.default_rng(5).integers(0, len(centers), 10000)]
        d = tgt - rays[20000:30000, :3]
        rays[20000:30000, 3:] = d / np.linalg.norm(d, axis=1, keepdims=True)
    gt, gi, gp, gs = dll.trace_rays(rays)
    ot, oi, op, os_ = sc.trace_first(rays)
    assert np.array_equal(gi, oi)
    assert np.array_equal(gp, op)
    assert np.array_equal(gt.view(np.uint32), ot.view(np.uint32))
    assert np.array_equal(gs.view(np.uint32), os_.view(np.uint32))
    assert (gi >= 0).mean() > (0.12 if scene in ("instanced", "mixed") else 0.3)


@pytest.mark.parametrize("kernel", list(KERNELS))
@pytest.mark.parametrize("scene", ["icosphere6", "instanced", "mixed"])
def test_axis_aligned_rays_bit_exact(dll, oracle, scene, kernel):
    """Rays along the coordinate axes, with +0 and -0 in the other components
    (a point light's photon drawn at cos = -1 leaves as (-0, 0, -1)): their
    slab tests use finite reciprocals, and the hits stay the oracle's. Half
    of the rays pass through triangle interiors. (A ray exactly through a
    vertex along an axis is left out: there the reference's NaN slab results
    decide whether the box holding the hit is culled, which no other
    hierarchy can reproduce.)"""
    if scene == "icosphere6":
        spec = scenes.displaced_icosphere(1, subdiv=6, width=64, height=36)
    elif scene == "mixed":
        spec = _single_lod_spec(_mixed_lod(7))
    else:
        spec = _small_instanced(2)
    _load(dll, spec)
    assert dll.renderer_set_parameter_int("Megakernel", KERNELS[kernel])
    sc = oracle.OracleScene(spec)
    rng = np.random.default_rng(11)
    a = sc.aabb()
    n = 6000
    org = rng.uniform(a[:3], a[3:], (n, 3)).astype(np.float32)
    # half of the rays through points inside triangles of the first object
    lod = spec.lods[0]
    if scene != "instanced" and len(lod.triangles):
        k = rng.integers(0, len(lod.triangles), n // 2)
        b = rng.uniform(0.1, 0.8, (n // 2, 2))
        b[b.sum(1) > 0.9] *= 0.5
        v = lod.vertices[lod.triangles[k]].astype(np.float64)
        org[: n // 2] = (v[:, 0] + b[:, :1] * (v[:, 1] - v[:, 0]) + b[:, 1:] * (v[:, 2] - v[:, 0])).astype(np.float32)
    axis = rng.integers(0, 3, n)
    sign = np.where(rng.uniform(size=n) < 0.5, -1.0, 1.0).astype(np.float32)
    dirs = np.zeros((n, 3), np.float32)
    dirs[np.arange(n), axis] = sign
    zsign = rng.uniform(size=(n, 3)) < 0.5
    dirs[(dirs == 0) & zsign] = np.float32(-0.0)
    if scene != "instanced":
        org[np.arange(n // 2), axis[: n // 2]] -= 3.0 * sign[: n // 2]
    rays = np.concatenate([org, dirs], 1)
    gt, gi, gp, gs = dll.trace_rays(rays)
    ot, oi, op, os_ = sc.trace_first(rays)
    assert np.array_equal(gi, oi) and np.array_equal(gp, op)
    assert np.array_equal(gt.view(np.uint32), ot.view(np.uint32))
    assert np.array_equal(gs.view(np.uint32), os_.view(np.uint32))
    assert (gi >= 0).mean() > (0.02 if scene == "instanced" else 0.3)


@pytest.mark.parametrize("kernel", list(KERNELS))
@pytest.mark.parametrize("scene", ["cornell", "instanced"])
def test_occlusion_matches_oracle(dll, oracle, scene, kernel):
    spec = scenes.cornell_box(4) if scene == "cornell" else _small_instanced(3)
    _load(dll, spec)
    assert dll.renderer_set_parameter_int("Megakernel", KERNELS[kernel])
    sc = oracle.OracleScene(spec)
    rng = np.random.default_rng(9)
    box = sc.aabb()
    a = rng.uniform(box[:3], box[3:], (20000, 3)).astype(np.float32)
    b = rng.uniform(box[:3], box[3:], (20000, 3)).astype(np.float32)
    assert np.array_equal(dll.trace_occlusion(a, b), sc.trace_any(a, b))


def _render_pair(dll, oracle, spec, spp, max_path, seed=0, rr_start=0, kernel="wavefront", nee=1, min_path=0):
    _load(dll, spec)
    dll.render_enable_render_target("Radiance", False)
    dll.render_enable_render_target("Hit ID", False)
    assert dll.renderer_set_parameter_int("Megakernel", KERNELS[kernel])
    assert dll.renderer_set_parameter_int("Seed", seed)
    assert dll.renderer_set_parameter_int("Max. path length", max_path)
    assert dll.renderer_set_parameter_int("Min. path length", min_path)
    assert dll.renderer_set_parameter_int("NEE count", nee)
    assert dll.renderer_set_parameter_int("RR start depth", rr_start)
    sc = oracle.OracleScene(spec)
    pt = oracle.OraclePathTracer(sc, seed=seed, min_path=min_path, max_path=max_path, nee_count=nee,
                                 rr_start=rr_start)
    dll.render_iterate()
    pt.iterate()
    first_hits = (dll.get_target_image("Hit ID"), pt.target("Hit ID"))
    for _ in range(spp - 1):
        dll.render_iterate()
        pt.iterate()
    assert dll.render_get_current_iteration() == spp
    return first_hits, (dll.get_target_image("Radiance"), pt.target("Radiance"))


@pytest.mark.parametrize("kernel", list(KERNELS))
def test_pt_cornell_parity(dll, oracle, kernel):
    """Config 0: Cornell box 256x256, 4 spp, path length 8."""
    spec = scenes.cornell_box(0)
    (gh, oh), (gr, orad) = _render_pair(dll, oracle, spec, 4, 8, kernel=kernel)
    assert np.array_equal(gh, oh), "first-hit ids differ"
    err = rel_rmse(gr, orad)
    assert err <= RMSE_TOL, err
    assert orad.mean() > 0.05


@pytest.mark.parametrize("kernel", list(KERNELS))
def test_pt_icosphere_parity(dll, oracle, kernel):
    spec = scenes.displaced_icosphere(0, subdiv=6, width=160, height=90)
    (gh, oh), (gr, orad) = _render_pair(dll, oracle, spec, 2, 10, kernel=kernel)
    assert np.array_equal(gh, oh)
    assert rel_rmse(gr, orad) <= RMSE_TOL


@pytest.mark.parametrize("kernel", list(KERNELS))
def test_pt_instanced_parity(dll, oracle, kernel):
    spec = _small_instanced(1)
    (gh, oh), (gr, orad) = _render_pair(dll, oracle, spec, 2, 12, rr_start=3, kernel=kernel)
    assert np.array_equal(gh, oh)
    assert rel_rmse(gr, orad) <= RMSE_TOL


@pytest.mark.parametrize("kernel", list(KERNELS))
def test_pt_multi_nee_min_path_parity(dll, oracle, kernel):
    """Several next-event samples per vertex (shadow-ray groups) and a minimum path length."""
    spec = scenes.cornell_box(2, 96, 96)
    (gh, oh), (gr, orad) = _render_pair(dll, oracle, spec, 2, 6, nee=3, min_path=2, rr_start=2, kernel=kernel)
    assert np.array_equal(gh, oh)
    assert rel_rmse(gr, orad) <= RMSE_TOL
    assert orad.mean() > 0.01


@pytest.mark.parametrize("wavefront_bounces,tail_paths", [(0, 98304), (1, 98304), (3, 98304), (100, 98304),
                                                           (1, 0), (1, 2500)])
def test_pt_schedule_parity(dll, oracle, wavefront_bounces, tail_paths):
    """Any split between per-bounce stage launches and the path-finishing launch gives the oracle's bits
    (tail_paths 2500 hands over in the middle of the paths, 0 never before the queues are empty)."""
    spec = scenes.cornell_box(5, 80, 80)
    _load(dll, spec)
    dll.render_enable_render_target("Radiance", False)
    dll.render_enable_render_target("Hit ID", False)
    for name, value in {"Wavefront bounces": wavefront_bounces, "Tail paths": tail_paths, "NEE count": 2,
                        "Max. path length": 9, "RR start depth": 2, "Min. path length": 1}.items():
        assert dll.renderer_set_parameter_int(name, value)
    pt = oracle.OraclePathTracer(oracle.OracleScene(spec), seed=0, min_path=1, max_path=9, nee_count=2, rr_start=2)
    for _ in range(2):
        dll.render_iterate()
        pt.iterate()
    assert np.array_equal(dll.get_target_image("Hit ID"), pt.target("Hit ID"))
    assert rel_rmse(dll.get_target_image("Radiance"), pt.target("Radiance")) <= RMSE_TOL


@pytest.mark.parametrize("bits,dir_bits", [(3, 3), (12, 6), (16, 3), (16, 0), (6, 6)])
@pytest.mark.parametrize("scene", ["cornell_nee2", "instanced"])
def test_pt_ray_binning_parity(dll, oracle, scene, bits, dir_bits):
    """Rays traced in coherence-binned order (extension rays and shadow-ray groups of every bounce >= 1)
    give the oracle's bits: only the order of the trace launch's work changes."""
    if scene == "cornell_nee2":
        spec, kw = scenes.cornell_box(5, 80, 80), dict(nee=2, max_path=9, rr_start=2, min_path=1)
    else:
        spec, kw = _small_instanced(2), dict(nee=1, max_path=12, rr_start=3, min_path=0)
    _load(dll, spec)
    dll.render_enable_render_target("Radiance", False)
    dll.render_enable_render_target("Hit ID", False)
    for name, value in {"Ray sort bits": bits, "Ray sort direction bits": dir_bits, "NEE count": kw["nee"],
                        "Max. path length": kw["max_path"], "RR start depth": kw["rr_start"],
                        "Min. path length": kw["min_path"]}.items():
        assert dll.renderer_set_parameter_int(name, value)
    pt = oracle.OraclePathTracer(oracle.OracleScene(spec), seed=0, min_path=kw["min_path"], max_path=kw["max_path"],
                                 nee_count=kw["nee"], rr_start=kw["rr_start"])
    for _ in range(2):
        dll.render_iterate()
        pt.iterate()
    assert dll.stage_stats()["launches"] > 0
    assert np.array_equal(dll.get_target_image("Hit ID"), pt.target("Hit ID"))
    assert np.array_equal(dll.get_target_image("Radiance").view(np.uint32), pt.target("Radiance").view(np.uint32))


def test_ray_binning_parameters_are_checked(dll):
    _load(dll, scenes.cornell_box(0, 16, 16))
    assert not dll.renderer_set_parameter_int("Ray sort bits", 17)
    assert not dll.renderer_set_parameter_int("Ray sort direction bits", 4)
    assert dll.renderer_set_parameter_int("Ray sort bits", 0)


def test_graph_replay_equals_plain_launches(dll):
    """An iteration replayed from its captured CUDA graph gives the same bits as plain launches,
    also across a parameter change that forces a new capture."""
    spec = scenes.cornell_box(7, 96, 64)
    out = []
    for graph in (1, 0):
        _load(dll, spec)
        dll.render_enable_render_target("Radiance", False)
        dll.render_enable_render_target("Hit ID", False)
        assert dll.renderer_set_parameter_int("Iteration graph", graph)
        assert dll.renderer_set_parameter_int("Max. path length", 9)
        for _ in range(3):
            dll.render_iterate()
        assert dll.renderer_set_parameter_int("Max. path length", 5)  # resets and re-captures
        for _ in range(2):
            dll.render_iterate()
        out.append((dll.get_target_image("Radiance").copy(), dll.get_target_image("Hit ID").copy()))
    assert np.array_equal(out[0][0], out[1][0]) and np.array_equal(out[0][1], out[1][1])


def test_pt_long_paths_parity(dll, oracle):
    """Path length beyond the usual limit keeps the wavefront stages in step with the sequential loop."""
    spec = scenes.cornell_box(3, 48, 48)
    (gh, oh), (gr, orad) = _render_pair(dll, oracle, spec, 1, 40, rr_start=30)
    assert np.array_equal(gh, oh)
    assert rel_rmse(gr, orad) <= RMSE_TOL


def test_wavefront_equals_megakernel(dll):
    """The two kernel schedules produce the same bits."""
    spec = scenes.cornell_box(4, 128, 128)
    out = []
    for kernel in KERNELS.values():
        _load(dll, spec)
        dll.render_enable_render_target("Radiance", False)
        dll.render_enable_render_target("Hit ID", False)
        assert dll.renderer_set_parameter_int("Megakernel", kernel)
        assert dll.renderer_set_parameter_int("NEE count", 2)
        assert dll.renderer_set_parameter_int("Max. path length", 12)
        for _ in range(3):
            dll.render_iterate()
        out.append((dll.get_target_image("Radiance").copy(), dll.get_target_image("Hit ID").copy()))
    assert np.array_equal(out[0][0], out[1][0])
    assert np.array_equal(out[0][1], out[1][1])


def test_gpu_matches_golden_fixture(dll):
    import os
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "cornell_64.npz"))
    spec = scenes.cornell_box(0, 64, 64)
    _load(dll, spec)
    dll.render_enable_render_target("Hit ID", False)
    assert dll.renderer_set_parameter_int("Max. path length", 8)
    assert dll.renderer_set_parameter_int("Seed", 0)
    assert dll.renderer_set_parameter_int("RR start depth", 0)
    dll.render_iterate()
    assert np.array_equal(dll.get_target_image("Hit ID").astype(np.int16), g["hit_id"])
    for _ in range(3):
        dll.render_iterate()
    assert rel_rmse(dll.get_target_image("Radiance"), g["radiance"]) <= RMSE_TOL
