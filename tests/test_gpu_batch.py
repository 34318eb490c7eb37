"""Batched rendering (mufflon_render_batch): many jobs, several scenes, one set
of wavefront queues. Every job must come out exactly as the oracle renders it
alone, with and without capturing the batch as a CUDA graph."""
import dataclasses

import numpy as np
import pytest

from mufflon_b200 import bindings, scenes

pytestmark = pytest.mark.gpu


def _instanced():
    return scenes.instanced_scene(4, num_meshes=3, num_instances=24, num_spheres=120,
                                  tri_range=(1000, 3000), width=48, height=36)


@pytest.fixture(scope="module")
def worlds():
    specs = {"cornell": scenes.cornell_box(6, 64, 64),
             "ico": scenes.displaced_icosphere(2, subdiv=5, width=80, height=45),
             "inst": _instanced()}
    out = {}
    for k, spec in specs.items():
        d = bindings.DllInterface()
        bindings.load_scene_spec(d, spec)
        assert d.render_enable_renderer(0, 0)
        out[k] = (d, spec)
    yield out
    for d, _ in out.values():
        d.close()


def _jobs(worlds):
    return [
        dict(name="cornell", spp=3, max_path=6, seed=1),
        dict(name="ico", spp=2, max_path=8, seed=0, min_path=1),
        dict(name="inst", spp=1, max_path=12, seed=5, rr_start=3),
        dict(name="cornell", width=40, height=40, spp=2, max_path=4, seed=9),  # same scene, other resolution
        dict(name="ico", width=32, height=24, spp=4, max_path=5, seed=3, rr_start=2),
    ]


def _oracle_images(oracle, spec, job):
    spec = dataclasses.replace(spec, width=job.get("width") or spec.width, height=job.get("height") or spec.height)
    pt = oracle.OraclePathTracer(oracle.OracleScene(spec), seed=job.get("seed", 0), min_path=job.get("min_path", 0),
                                 max_path=job["max_path"], nee_count=1, rr_start=job.get("rr_start", 0))
    for _ in range(job["spp"]):
        pt.iterate()
    return pt.target("Radiance"), pt.target("Hit ID")


def test_batch_matches_oracle_per_job(worlds, oracle):
    jobs = _jobs(worlds)
    req = [dict(j, instance=worlds[j["name"]][0]) for j in jobs]
    imgs, hits, done, st = bindings.render_batch(req, use_graph=False, hit_ids=True)
    imgs_g, hits_g, done_g, st_g = bindings.render_batch(req, use_graph=True, hit_ids=True)
    assert st["usedGraph"] == 0 and st_g["usedGraph"] == 1
    assert st["pixels"] == sum((j.get("width") or worlds[j["name"]][1].width) *
                               (j.get("height") or worlds[j["name"]][1].height) for j in jobs)
    for k, job in enumerate(jobs):
        assert np.array_equal(imgs[k], imgs_g[k]), f"job {k}: graph and plain launches differ"
        assert np.array_equal(hits[k], hits_g[k])
        orad, ohit = _oracle_images(oracle, worlds[job["name"]][1], job)
        assert np.array_equal(hits[k], ohit), f"job {k}: hit ids differ"
        err = np.sqrt(np.mean((imgs[k] - orad) ** 2)) / max(np.sqrt(np.mean(orad ** 2)), 1e-12)
        assert err <= 1e-4, (k, err)
    # a job's completion time is the end of its last sample
    spp = [j["spp"] for j in jobs]
    assert done[int(np.argmax(spp))] == pytest.approx(max(done), rel=1e-6)
    assert all(d > 0 for d in done)


def test_batch_equals_single_job_render(worlds):
    """A one-job batch equals render_iterate on the same instance, bit for bit."""
    d, spec = worlds["cornell"]
    for name, v in {"Seed": 2, "Max. path length": 7, "Min. path length": 0, "NEE count": 1,
                    "RR start depth": 0}.items():
        assert d.renderer_set_parameter_int(name, v)
    d.render_enable_render_target("Radiance", False)
    d.render_reset()
    for _ in range(3):
        d.render_iterate()
    ref = d.get_target_image("Radiance").copy()
    imgs, _, _, _ = bindings.render_batch([dict(instance=d, spp=3, max_path=7, seed=2)], use_graph=True)
    assert np.array_equal(imgs[0], ref)


def test_batch_rejects_bad_jobs(worlds):
    d, _ = worlds["cornell"]
    with pytest.raises(bindings.MufflonError):
        bindings.render_batch([dict(instance=d, spp=0, max_path=4)])
    with pytest.raises(bindings.MufflonError):
        bindings.render_batch([dict(instance=d, spp=1, max_path=4, nee=1), dict(instance=d, spp=1, max_path=4, nee=2)])


def test_autotune_keeps_the_image(worlds):
    """Tuning picks one of the candidates and does not change the rendered bits."""
    from mufflon_b200 import autotune
    d, _ = worlds["ico"]
    d.render_enable_render_target("Radiance", False)
    for name, v in {"Seed": 0, "Max. path length": 8, "Min. path length": 0, "NEE count": 1, "RR start depth": 0,
                    "Megakernel": 0, "Wavefront bounces": 2, "Trace blocks per SM": 6, "Trace refill lanes": 32}.items():
        assert d.renderer_set_parameter_int(name, v)
    d.render_reset()
    for _ in range(2):
        d.render_iterate()
    before = d.get_target_image("Radiance").copy()
    cands = [dict(megakernel=0, trace_blocks=4, wavefront_bounces=1, refill_lanes=16),
             dict(megakernel=0, trace_blocks=6, wavefront_bounces=3, refill_lanes=32), dict(megakernel=1)]
    res = autotune.autotune(d, iterations=1, warmup=0, candidates=cands)
    assert res["best"] in cands and len(res["table"]) == 3
    for k, v in res["best"].items():
        assert d.renderer_get_parameter_int(autotune.PARAMS[k]) == v
    for _ in range(2):
        d.render_iterate()
    assert np.array_equal(d.get_target_image("Radiance"), before)
