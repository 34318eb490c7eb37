"""Path-tracer benchmark: Mrays/s (and spp/s) at 1920x1080 on the displaced
icosphere (1 310 720 triangles, 16 spp per frame, path length 10), next to the
CPU oracle timed on this host's cores.

One step = one 16-spp frame (16 render_iterate calls of the CUDA path tracer).

value  -- rays (extension + shadow) of the K timed frames / the summed device
          time of the path-tracing kernel (CUDA events on the library's stream);
          the scene stays resident in HBM.
e2e    -- the same metric through the public C API from host buffers: every step
          re-uploads the scene from host memory (world_load_scenario: geometry
          upload + GPU LBVH build), renders 16 iterations and copies the
          radiance image back to host memory (wall clock around the calls).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Under torchrun (N > 1) every rank renders the frame with its own seed (the
samples split across GPUs, per-GPU work fixed -> weak scaling); the e2e step
averages the images with one NCCL all-reduce.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

SPP_PER_FRAME = 16
MAX_PATH = 10
WIDTH, HEIGHT = 1920, 1080
METRIC = "Mrays/s & spp/s at 1080p vs CPU PT"
WORKLOAD = "displaced_icosphere_1310720tri_1920x1080_16spp_depth10"


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="b200", choices=["b200", "reference"])
    p.add_argument("--subdiv", type=int, default=8)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--cpu-seconds", type=float, default=15.0)
    p.add_argument("--workload", default="frame", choices=["frame", "batch", "adjoint", "load", "lights", "lt", "bpt", "vcm", "instanced"],
                   help="frame: the 1080p headline; batch: 64 mixed jobs in one batched launch vs one by one; "
                        "adjoint: albedo gradient vs forward time; load: scene-file import of the headline scene; "
                        "lights: GPU light-tree build of 262 145 lights; lt: the light tracer at 1080p; bpt: the bidirectional path tracer at 1080p; vcm: vertex connection and merging at 1080p; instanced: config 2 (4 096 instances) at 1080p")
    p.add_argument("--jobs", type=int, default=64)
    p.add_argument("--resolution", type=lambda v: tuple(int(x) for x in v.split("x")), default=(WIDTH, HEIGHT),
                   help="frame / lt / bpt / vcm: image size WxH (default 1920x1080; smaller for profiler captures)")
    p.add_argument("--merge-radius", type=float, default=0.001,
                   help="vcm: \"Relative merge radius\" (of the scene's diagonal; the reference's default 0.001)")
    p.add_argument("--megakernel", action="store_true",
                   help="lt / bpt: the single persistent kernel instead of the stages per path length")
    return p.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        try:
            return json.load(open(path)), "measured"
        except Exception:
            pass
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


class ClockSampler:
    """nvidia-smi sampling during the timed region (SM clock, reasons)."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-i", str(self.gpu), "-lms", "200"], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def scene_bytes(spec):
    """Host->device bytes of one scene upload (geometry, instances, materials, lights)."""
    b = 0
    for l in spec.lods:
        nv, nt, nq, ns = len(l.vertices), len(l.triangles), len(l.quads), len(l.spheres)
        b += nv * (12 + 12 + 8) + nt * 12 + nq * 16 + (nt + nq) * 2 + ns * (16 + 2)
    ni = len(spec.instance_lod)
    b += ni * (48 + 4 + 24 + 12)
    return b


def cpu_baseline(spec, seconds):
    """CPU oracle (restatement of the reference CPU path tracer) on all host cores."""
    from oracle import pyoracle
    threads = os.cpu_count() or 1
    sc = pyoracle.OracleScene(spec)
    pt = pyoracle.OraclePathTracer(sc, seed=0, max_path=MAX_PATH)
    rows_per_chunk = max(1, spec.height // 8)
    rays, elapsed, rows_done, passes = 0, 0.0, 0, 0
    t_start = time.perf_counter()
    y = 0
    while elapsed < seconds or rows_done == 0:
        y1 = min(spec.height, y + rows_per_chunk)
        before = pt.stats()["rays"]
        t0 = time.perf_counter()
        pt.iterate_rows(y, y1, threads)
        elapsed += time.perf_counter() - t0
        rays += pt.stats()["rays"] - before
        rows_done += y1 - y
        y = 0 if y1 >= spec.height else y1
        if y == 0:
            passes += 1
        if time.perf_counter() - t_start > 4 * seconds:
            break
    mrays = rays / elapsed / 1e6
    pixels = rows_done * spec.width
    return {"value": round(mrays, 3), "unit": "Mrays/s", "cores": threads, "kind": "port",
            "sample": f"{rows_done} rows x {spec.width} px x 1 spp ({pixels} paths, {rays} rays, {elapsed:.1f} s)",
            "spp_per_s_1080p": round(pixels / elapsed / (spec.width * spec.height), 4)}


def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    from mufflon_b200 import scenes
    spec = scenes.displaced_icosphere(0, subdiv=args.subdiv, width=WIDTH, height=HEIGHT)
    from oracle import pyoracle
    threads = os.cpu_count() or 1
    sc = pyoracle.OracleScene(spec)
    pt = pyoracle.OraclePathTracer(sc, seed=0, max_path=MAX_PATH)
    # one step: 1 spp over the whole 1080p frame (about 0.3 s on 16 host
    # cores), so the default 10 timed steps sample several seconds
    tot_rays, tot_time = 0, 0.0
    for i in range(args.warmup + args.steps):
        before = pt.stats()["rays"]
        t0 = time.perf_counter()
        pt.iterate_rows(0, HEIGHT, threads)
        dt = time.perf_counter() - t0
        r = pt.stats()["rays"] - before
        if i >= args.warmup:
            tot_rays += r
            tot_time += dt
    v = tot_rays / tot_time / 1e6
    line = {"impl": "reference", "metric": METRIC, "value": round(v, 3), "unit": "Mrays/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(1000 * tot_time / args.steps, 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": WORKLOAD, "step": "1 spp over the whole frame (CPU oracle port, all host threads)"},
            "cpu_baseline": {"value": round(v, 3), "unit": "Mrays/s", "cores": threads, "kind": "port",
                             "sample": f"{args.steps} frames of {WIDTH} x {HEIGHT} px at 1 spp, {tot_time:.1f} s"},
            "e2e": {"value": round(v, 3), "unit": "Mrays/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# DRAM bytes per algorithmic byte of the traversal launches, from an ncu
# capture of the bounce-1 k_trace launch of this workload.
TRACE_DRAM_PER_ALG_BYTE = 0.33  # 395.2 MB of DRAM traffic for 1.194 GB of algorithmic bytes
LBVH_STAGES = ["morton", "sort", "emit", "merge", "mark", "scan", "compact", "soup", "wide"]
# Algorithmic bytes per triangle of the reference's build stages (Morton 60,
# sort 200, emit 32, merge 148, mark 32, scan 8, compact 68, soup 96), and of
# the 8-wide conversion (binary boxes 32 B read, primitive ids 8 B, soup 36 B
# read + 48 B written).
LBVH_BYTES_PER_PRIM = 644
WIDE_BYTES_PER_PRIM = 124


def lbvh_build_measurement(dll, lod, torch, reps=10):
    """Device-resident LBVH build of the workload's mesh (CUDA events)."""
    import ctypes as C
    v = torch.from_numpy(np.ascontiguousarray(lod.vertices, np.float32)).cuda()
    idx = torch.from_numpy(np.ascontiguousarray(lod.triangles.reshape(-1).astype(np.int32))).cuda()
    aabb = np.concatenate([lod.vertices.min(0), lod.vertices.max(0)]).astype(np.float32)
    n = len(lod.triangles)
    ni = C.c_int32(0)
    ms = C.c_float(0.0)
    stages = np.zeros(9, np.float32)
    tot = np.zeros(9)
    total = 0.0
    for it in range(3 + reps):
        ok = dll.core.mufflon_lbvh_build_device(C.c_void_p(v.data_ptr()), C.c_void_p(idx.data_ptr()), n, 0, None, 0,
                                                aabb.ctypes.data, C.byref(ni), C.byref(ms), stages.ctypes.data)
        if not ok:
            raise RuntimeError(dll.core.core_get_dll_error())
        if it >= 3:
            tot += stages
            total += ms.value
    tot /= reps
    ref_ms = float(tot[:8].sum())
    gbs = n * LBVH_BYTES_PER_PRIM / (ref_ms * 1e-3) / 1e9
    peaks, kind = measured_peaks()
    return {"prims": n, "build_ms": round(total / reps, 4),
            "stage_ms": {k: round(float(t), 4) for k, t in zip(LBVH_STAGES, tot)},
            "reference_stages_ms": round(ref_ms, 4), "alg_bytes_per_prim": LBVH_BYTES_PER_PRIM,
            "achieved_gbs": round(gbs, 1), "frac_of_hbm": round(gbs / peaks["hbm_gbs"], 4),
            "wide_alg_bytes_per_prim": WIDE_BYTES_PER_PRIM,
            "wide_gbs": round(n * WIDE_BYTES_PER_PRIM / (float(tot[8]) * 1e-3) / 1e9, 1),
            "num_internal_after_collapse": int(ni.value)}


def run_b200(args):
    rank, world, local = dist_env()
    import torch
    torch.cuda.set_device(local)
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))
    from mufflon_b200 import bindings, build, distributed, scenes
    build.build()
    W, H = args.resolution
    spec = scenes.displaced_icosphere(0, subdiv=args.subdiv, width=W, height=H)
    dll = bindings.DllInterface()
    bindings.load_scene_spec(dll, spec)
    assert dll.render_enable_renderer(0, 0)
    assert dll.renderer_set_parameter_int("Max. path length", MAX_PATH)
    assert dll.renderer_set_parameter_int("Seed", distributed.rank_seed(0, rank))

    def frame():
        rays = shadow = nodes = prims = inst = 0
        ms = 0.0
        launches = 1  # the generator seeding after render_reset
        for _ in range(SPP_PER_FRAME):
            dll.render_iterate()
            s = dll.render_stats()
            rays += s["rays"]; shadow += s["shadowRays"]; nodes += s["nodeVisits"]
            prims += s["primTests"]; inst += s["instanceVisits"]; ms += s["kernelMs"]
            launches += dll.stage_stats()["launches"]
            if s["errors"]:
                raise RuntimeError(f"traversal errors reported: {s['errors']}")
        return rays, shadow, nodes, prims, inst, ms, launches

    def stage_frame(statistics=False):
        """One untimed frame with events around every stage launch, or (statistics=True) with the
        counting kernel variants that record node visits, primitive tests and instance entries. Both
        trace the same rays; only the non-counting frame's stage times are the product's."""
        param = "Traversal statistics" if statistics else "Stage timing"
        assert dll.renderer_set_parameter_int(param, 1)
        dll.render_reset()
        acc = {}
        for _ in range(SPP_PER_FRAME):
            dll.render_iterate()
            for k, v in dll.stage_stats().items():
                acc[k] = acc.get(k, 0) + v
        assert dll.renderer_set_parameter_int(param, 0)
        return acc

    def barrier():
        torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()

    for _ in range(args.warmup):
        dll.render_reset()
        frame()
    clocks = ClockSampler(local)
    clocks.start()
    barrier()
    tot = np.zeros(7)
    for _ in range(args.steps):
        dll.render_reset()
        tot += np.array(frame(), dtype=np.float64)
    barrier()
    clk = clocks.stop()
    rays, shadow, nodes, prims, inst, kernel_ms, gpu_launches = tot
    # max over ranks of the device time, sum of rays
    if world > 1:
        t = torch.tensor([kernel_ms], device="cuda")
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        kernel_ms_max = float(t.item())
        r = torch.tensor([rays], device="cuda", dtype=torch.float64)
        torch.distributed.all_reduce(r)
        rays_all = float(r.item())
    else:
        kernel_ms_max, rays_all = kernel_ms, rays
    mrays = rays_all / (kernel_ms_max * 1e-3) / 1e6
    spp_s = SPP_PER_FRAME * args.steps * world / (kernel_ms_max * 1e-3)

    # e2e: scene upload + BVH build + 16 iterations + image readback per step
    d2h = W * H * 3 * 4
    h2d = scene_bytes(spec)
    dll.get_target_image("Radiance", copy=False)  # warm-up: allocates the page-locked read-back buffer once
    barrier()
    e2e_rays, t_e2e = 0.0, 0.0
    load_ms = {}
    for _ in range(args.steps):
        t0 = time.perf_counter()
        dll.core.world_load_scenario(dll.muffInst, dll.core.world_get_current_scenario(dll.muffInst))
        for k, v in dll.load_stats().items():
            load_ms[k] = load_ms.get(k, 0.0) + v / args.steps
        for _ in range(SPP_PER_FRAME):
            dll.render_iterate()
            e2e_rays += dll.render_stats()["rays"]
        img = dll.get_target_image("Radiance", copy=False)  # the library's page-locked read-back buffer
        if world > 1:
            ti, _ = distributed.combine_images(torch.from_numpy(img).cuda(), SPP_PER_FRAME)
            img = ti.cpu().numpy()
        t_e2e += time.perf_counter() - t0
    if world > 1:
        t = torch.tensor([t_e2e], device="cuda")
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        t_e2e = float(t.item())
        r = torch.tensor([e2e_rays], device="cuda", dtype=torch.float64)
        torch.distributed.all_reduce(r)
        e2e_rays = float(r.item())
    e2e_mrays = e2e_rays / t_e2e / 1e6

    # roofline of the dominant kernel (k_trace: closest-hit and shadow-ray
    # traversal of one bounce): algorithmic bytes per launch / its average
    # launch time (events on the library's stream). Per unit: an 8-wide node
    # 80 B, a primitive-soup slot 48 B, an instance entry 56 B (world-to-instance
    # rows 48 B + LoD index 4 B + the LoD's hierarchy pointers); per extension
    # ray its queue entry 32 B in and 20 B out, per shadow ray 48 B in.
    st = stage_frame()
    counts = stage_frame(statistics=True)
    for k in ("extendNodeVisits", "shadowNodeVisits", "extendPrimTests", "shadowPrimTests", "extendInstanceVisits",
              "shadowInstanceVisits"):
        st[k] = counts[k]
    assert counts["extensionRays"] == st["extensionRays"] and counts["shadowRays"] == st["shadowRays"]
    wf_bounces = dll.renderer_get_parameter_int("Wavefront bounces")
    trace_launches = SPP_PER_FRAME * min(wf_bounces + 1, MAX_PATH)
    ext_rays, shd_rays = st["extensionRays"], st["shadowRays"]
    alg_bytes = ((st["extendNodeVisits"] + st["shadowNodeVisits"]) * 80
                 + (st["extendPrimTests"] + st["shadowPrimTests"]) * 48
                 + (st["extendInstanceVisits"] + st["shadowInstanceVisits"]) * 56
                 + ext_rays * (32 + 20) + shd_rays * 48)
    # the counters include the rays of the path-finishing launch; the trace
    # launches carry the rays of bounces 0..wf_bounces (their share measured
    # below from the stage times is not needed: bytes and time both cover
    # trace + tail)
    trace_ms = st["extendMs"] + st["tailMs"]
    achieved_gbs = alg_bytes / (trace_ms * 1e-3) / 1e9
    peaks, peak_kind = measured_peaks()
    l2 = bindings.c_float(0.0)
    dll.core.mufflon_measure_l2_bandwidth(32 << 20, 100, bindings.byref(l2))
    # Traversal reads nodes, soups and instance data that stay in L2 (the
    # hierarchies and soups of this scene, ~95 MB, fit in the 126 MB L2; the
    # ncu capture shows DRAM traffic at ~0.18 of these bytes), so its roof is
    # L2: "frac_of_l2" is the fraction of the L2 read bandwidth measured here
    # with mufflon_measure_l2_bandwidth (a 32 MiB buffer read 100 times, CUDA
    # events). "peak"/"frac" keep the measured HBM copy bandwidth for
    # comparison with the other kernels' lines.
    roofline = {"bound": "l2", "achieved": round(achieved_gbs, 1), "peak": peaks["hbm_gbs"], "unit": "GB/s",
                "frac": round(achieved_gbs / peaks["hbm_gbs"], 4),
                "traffic": round(TRACE_DRAM_PER_ALG_BYTE * alg_bytes / (trace_launches + SPP_PER_FRAME)),
                "traffic_note": ("DRAM bytes per launch: ncu dram__bytes_read+write of the bounce-1 k_trace launch "
                                 f"per algorithmic byte ({TRACE_DRAM_PER_ALG_BYTE}) x algorithmic bytes per launch"),
                "peak_source": f"{peak_kind} HBM copy bandwidth",
                "l2_read_peak_gbs": round(float(l2.value), 1),
                "l2_peak_source": "mufflon_measure_l2_bandwidth: 32 MiB L2-resident buffer read 100x, CUDA events",
                "frac_of_l2": round(achieved_gbs / max(float(l2.value), 1e-9), 4),
                "bytes_per_ray": round(alg_bytes / max(ext_rays + shd_rays, 1), 1),
                "kernel": "k_trace + k_tail", "launches": trace_launches + SPP_PER_FRAME,
                "avg_launch_ms": round(trace_ms / (trace_launches + SPP_PER_FRAME), 4)}
    stage_ms = {"camera": round(st["cameraMs"], 3), "trace": round(st["extendMs"], 3),
                "tail": round(st["tailMs"], 3), "shade": round(st["shadeMs"], 3),
                "finalize": round(st["finalizeMs"], 3), "bin": round(st["binMs"], 3)}
    per_ray = {"extend_nodes": round(st["extendNodeVisits"] / max(st["extensionRays"], 1), 2),
               "extend_prims": round(st["extendPrimTests"] / max(st["extensionRays"], 1), 2),
               "shadow_nodes": round(st["shadowNodeVisits"] / max(st["shadowRays"], 1), 2),
               "shadow_prims": round(st["shadowPrimTests"] / max(st["shadowRays"], 1), 2)}
    lbvh = lbvh_build_measurement(dll, spec.lods[0], torch) if rank == 0 else None
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(spec, args.cpu_seconds)
    if rank == 0:
        line = {"metric": METRIC, "value": round(mrays, 2), "unit": "Mrays/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": round(kernel_ms_max / args.steps, 3), "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": {"workload": WORKLOAD.replace("1920x1080", f"{W}x{H}"), "triangles": int(spec.num_prims), "resolution": [W, H],
                           "spp_per_step": SPP_PER_FRAME, "max_path_length": MAX_PATH,
                           "l2": "inputs larger than L2 (BVH + triangle soup + image > 126 MB)",
                           "parallelism": f"replicas x{world} (samples split by seed)"},
                "spp_per_s": round(spp_s, 3),
                "rays_per_step": int(rays / args.steps),
                "e2e": {"value": round(e2e_mrays, 2), "unit": "Mrays/s", "h2d_bytes_per_step": int(h2d),
                        "d2h_bytes_per_step": int(d2h),
                        "note": "scene upload + GPU LBVH build + 16 iterations + radiance readback per step (wall clock)",
                        "load_ms": {k: round(v, 3) for k, v in load_ms.items() if k.endswith("Ms")}},
                "gpu_launches": int(gpu_launches),
                "roofline": roofline,
                "stage_ms_per_frame": stage_ms,
                "lbvh": lbvh,
                "traversal_per_ray": per_ray,
                "cpu_baseline": cpu,
                "clocks": clk}
        print(json.dumps(line), flush=True)
    dll.close()
    if world > 1:
        torch.distributed.destroy_process_group()


def batch_jobs(n_jobs, seed=7):
    """The mixed-job workload: scene in {Cornell box, 1.3 M-triangle icosphere,
    4096 instances of 10 meshes + 20 000 spheres, 100 K-triangle displaced
    plane}, square side log-uniform in [128, 1024], spp uniform in 1..64, max
    path length uniform in 4..12 (seeded)."""
    rng = np.random.default_rng(seed)
    jobs = []
    for j in range(n_jobs):
        side = int(round(math.exp(rng.uniform(math.log(128), math.log(1024)))))
        jobs.append(dict(scene=int(rng.integers(0, 4)), width=side, height=side, spp=int(rng.integers(1, 65)),
                         max_path=int(rng.integers(4, 13)), seed=j))
    return jobs


def run_batch(args):
    import torch
    torch.cuda.set_device(0)
    from mufflon_b200 import autotune, bindings, build, scenes
    build.build()
    specs = [scenes.cornell_box(0), scenes.displaced_icosphere(0, subdiv=8, width=512, height=512),
             scenes.instanced_scene(0), scenes.displaced_plane(0)]
    worlds = []
    for spec in specs:
        d = bindings.DllInterface()
        bindings.load_scene_spec(d, spec)
        assert d.render_enable_renderer(0, 0)
        worlds.append(d)
    # The batch runs with the first job's schedule settings (the defaults here). Tuning them on one
    # scene does not carry over: the icosphere's best (4 trace blocks per SM) makes this mixed batch
    # slower (16.9 vs 18.6 jobs/s), the instanced scene's best is the default.
    schedule = {k: worlds[0].renderer_get_parameter_int(v) for k, v in autotune.PARAMS.items()}
    jobs = batch_jobs(args.jobs)
    req = [dict(instance=worlds[j["scene"]], width=j["width"], height=j["height"], spp=j["spp"],
                max_path=j["max_path"], seed=j["seed"]) for j in jobs]
    bindings.render_batch(req[:4], use_graph=False)  # warm-up of the batch buffers and kernels
    res = {}
    for graph in (True, False):
        t0 = time.perf_counter()
        _, _, done, st = bindings.render_batch(req, use_graph=graph)
        wall = time.perf_counter() - t0
        res[graph] = (done, st, wall)
    seq_done, seq_total, seq_wall = [], 0.0, 0.0
    per_scene = {}
    for j, r in zip(jobs, req):
        t0 = time.perf_counter()
        _, _, done, st = bindings.render_batch([r], use_graph=False)
        seq_wall += time.perf_counter() - t0
        seq_total += st["deviceMs"]
        seq_done.append(seq_total)
        ps = per_scene.setdefault(j["scene"], [0, 0.0, 0])
        ps[0] += j["width"] * j["height"] * j["spp"]
        ps[1] += st["deviceMs"]
        ps[2] += 1
    done_g, st_g, wall_g = res[True]
    pct = lambda v, q: float(np.percentile(np.asarray(v), q))
    samples = sum(j["width"] * j["height"] * j["spp"] for j in jobs)
    line = {"metric": "batched jobs/s (64 mixed jobs: 4 scenes, 128-1024 px, 1-64 spp, depth 4-12)",
            "value": round(len(jobs) / (st_g["deviceMs"] * 1e-3), 3), "unit": "jobs/s", "n_gpus": 1,
            "higher_is_better": True, "data": "synthetic", "dtype": "f32",
            "config": {"workload": "batch_64_mixed_jobs", "jobs": len(jobs), "pixels": st_g["pixels"],
                       "samples": int(samples), "scenes": ["cornell_box", "displaced_icosphere_1310720tri",
                                                           "instanced_4096x10meshes_20000spheres",
                                                           "displaced_plane_100k"]},
            "batched": {"device_ms": round(st_g["deviceMs"], 3), "wall_ms": round(wall_g * 1e3, 3),
                        "launches": st_g["launches"], "graph": True,
                        "p50_ms": round(pct(done_g, 50), 3), "p99_ms": round(pct(done_g, 99), 3),
                        "msamples_per_s": round(samples / (st_g["deviceMs"] * 1e-3) / 1e6, 1)},
            "batched_no_graph": {"device_ms": round(res[False][1]["deviceMs"], 3),
                                 "wall_ms": round(res[False][2] * 1e3, 3),
                                 "p50_ms": round(pct(res[False][0], 50), 3), "p99_ms": round(pct(res[False][0], 99), 3)},
            "sequential": {"device_ms": round(seq_total, 3), "wall_ms": round(seq_wall * 1e3, 3),
                           "jobs_per_s": round(len(jobs) / (seq_total * 1e-3), 3),
                           "p50_ms": round(pct(seq_done, 50), 3), "p99_ms": round(pct(seq_done, 99), 3)},
            "speedup_vs_sequential": round(seq_total / st_g["deviceMs"], 3),
            "sequential_per_scene": {["cornell", "icosphere", "instanced", "plane"][k]:
                                     {"jobs": v[2], "device_ms": round(v[1], 1),
                                      "msamples_per_s": round(v[0] / (v[1] * 1e-3) / 1e6, 1)}
                                     for k, v in sorted(per_scene.items())},
            "schedule": schedule}
    print(json.dumps(line), flush=True)
    for d in worlds:
        d.close()


def run_adjoint(args):
    """Config 4: gradient of an L2 image loss with respect to a 512^2 RGB albedo
    texture on the Cornell box's back wall (init 0.5), 512^2 image, 16 spp,
    depth 6; target rendered with a seeded smoothed-noise texture in
    [0.1, 0.9]. Reports forward time (16 iterations), adjoint time (replay of
    the 16 samples) and their ratio, and checks the gradient against the
    oracle's double-precision gradient and against central differences of GPU
    renders on 64 texel channels."""
    import torch
    torch.cuda.set_device(0)
    from mufflon_b200 import bindings, build, scenes
    from mufflon_b200.adjoint import AlbedoRenderer
    build.build()
    spp, depth, res, tsz = 16, 6, 512, 512
    spec = scenes.cornell_box_textured(0, res, res, texture_size=tsz)
    d = bindings.DllInterface()
    bindings.load_scene_spec(d, spec)
    assert d.render_enable_renderer(0, 0)
    r = AlbedoRenderer(d, d.textures[0], (tsz, tsz), spp=spp, seed=0, max_path=depth)
    target_tex = scenes.smooth_noise_texture(1, tsz)[..., :3]
    target = r.render(target_tex)
    tex = np.full((tsz, tsz, 3), 0.5, np.float32)
    fwd, adj = [], []
    for _ in range(3 + args.steps):
        img = r.render(tex)
        dldi = 2.0 * (img - target)
        g = r.gradient(dldi)
        fwd.append(r.last_forward_ms)
        adj.append(r.last_adjoint_ms)
    fwd_ms, adj_ms = float(np.median(fwd[3:])), float(np.median(adj[3:]))
    # FD on the 64 texel channels with the largest gradients (central, step 0.1: exact for the polynomial)
    loss = lambda t: float(np.sum((r.render(t).astype(np.float64) - target) ** 2))
    idx = np.argsort(-np.abs(g).reshape(-1))[:64]
    fd_err = []
    for k in idx:
        y, x, c = np.unravel_index(k, g.shape)
        tp, tm = tex.copy(), tex.copy()
        tp[y, x, c] += 0.1
        tm[y, x, c] -= 0.1
        fd = (loss(tp) - loss(tm)) / 0.2
        fd_err.append(abs(fd - g[y, x, c]) / max(abs(g[y, x, c]), 1e-12))
    ora = None
    if not args.no_cpu_baseline:
        sys.path.insert(0, ROOT)
        from oracle import pyoracle
        pt = pyoracle.OraclePathTracer(pyoracle.OracleScene(dataclasses_replace_texture(spec, tex)), seed=0,
                                       max_path=depth, rr_start=depth)
        t0 = time.perf_counter()
        ref = pt.albedo_gradient(0, spp, dldi)
        cpu_s = time.perf_counter() - t0
        scale = np.abs(ref).max()
        big = np.abs(ref) > 1e-2 * scale
        ora = {"max_abs_err_over_max": float(np.abs(g - ref).max() / scale),
               "max_rel_err_significant": float(np.max(np.abs(g[big] - ref[big]) / np.abs(ref[big]))),
               "cpu_seconds": round(cpu_s, 2), "cpu_cores": os.cpu_count()}
    # the emission adjoint of the ceiling light on the same scene (Russian
    # roulette on, as a plain render): its replay against its forward pass,
    # checked against the FP64 oracle gradient and central differences
    from mufflon_b200.adjoint import EmissionRenderer
    li = [i for i, m in enumerate(spec.materials) if m.type == scenes.MAT_EMISSIVE][0]
    d.texture_update(d.textures[0], tex)
    e = EmissionRenderer(d, d.materials[li], spp=spp, seed=0, max_path=depth, rr_start=0)
    L0 = np.array([15.0, 15.0, 15.0], np.float32)
    efwd, eadj = [], []
    for _ in range(3 + args.steps):
        eimg = e.render(L0)
        edldi = 2.0 * (eimg - target)
        eg = e.gradient(edldi)
        efwd.append(e.last_forward_ms)
        eadj.append(e.last_adjoint_ms)
    efwd_ms, eadj_ms = float(np.median(efwd[3:])), float(np.median(eadj[3:]))
    eloss = lambda L: float(np.sum((e.render(L).astype(np.float64) - target) ** 2))
    efd = []
    for c in range(3):
        lp, lm = L0.copy(), L0.copy()
        lp[c] += 1e-3
        lm[c] -= 1e-3
        efd.append(abs((eloss(lp) - eloss(lm)) / 2e-3 - eg[c]) / abs(eg[c]))
    eora = None
    if not args.no_cpu_baseline:
        import dataclasses
        mats = list(spec.materials)
        mats[li] = scenes.MaterialSpec(scenes.MAT_EMISSIVE, radiance=tuple(float(x) for x in L0), name="light")
        pte = pyoracle.OraclePathTracer(pyoracle.OracleScene(dataclasses.replace(dataclasses_replace_texture(spec, tex),
                                                                                 materials=mats)),
                                        seed=0, max_path=depth, rr_start=0)
        eref = pte.emission_gradient(li, spp, edldi)
        eora = {"max_rel_err": float(np.max(np.abs(eg - eref) / np.abs(eref)))}
    line = {"metric": "adjoint/forward time (512^2, 16 spp, depth 6, 512^2 albedo texture)",
            "value": round(adj_ms / fwd_ms, 3), "unit": "ratio", "higher_is_better": False, "n_gpus": 1,
            "data": "synthetic", "dtype": "f32",
            "config": {"workload": "cornell_textured_adjoint", "resolution": [res, res], "spp": spp, "depth": depth,
                       "texture": [tsz, tsz, 3], "russian_roulette": "off"},
            "forward_ms": round(fwd_ms, 3), "adjoint_ms": round(adj_ms, 3),
            "fd_check": {"texels": len(fd_err), "step": 0.1, "max_rel_err": float(np.max(fd_err))},
            "fp64_oracle_check": ora,
            "emission": {"ratio": round(eadj_ms / efwd_ms, 3), "forward_ms": round(efwd_ms, 3),
                         "adjoint_ms": round(eadj_ms, 3), "russian_roulette": "on",
                         "fd_check": {"step": 1e-3, "max_rel_err": float(np.max(efd))},
                         "fp64_oracle_check": eora}}
    print(json.dumps(line), flush=True)
    d.close()


def run_load(args):
    """Scene-file import of the headline scene (the 1.3 M-triangle displaced
    icosphere at 1080p) written as JSON + binary: loader_load_json wall time
    (JSON parse, binary header, LoD read through the core's LoD callback,
    geometry upload, LBVH + 8-wide build, lights and materials), for an
    uncompressed file and a DEFLATE file with packed normals, the file in the
    page cache. Each load is checked: one iteration's hit ids must equal the
    same scene built through the world API."""
    import tempfile
    import torch
    torch.cuda.set_device(0)
    from mufflon_b200 import bindings, build, scenefile, scenes
    build.build()
    spec = scenes.displaced_icosphere(0, subdiv=args.subdiv, width=WIDTH, height=HEIGHT)
    out = {}
    with tempfile.TemporaryDirectory() as tmp:
        d = bindings.DllInterface(useLoader=True)
        for name, kw in [("raw", dict()), ("deflate_packed_normals", dict(deflate=True, compressed_normals=True))]:
            jp = os.path.join(tmp, f"{name}.json")
            loaded = scenefile.write_scene(spec, jp, **kw)
            binp = os.path.join(tmp, json.load(open(jp))["binary"])
            times, stats = [], []
            for i in range(args.warmup + args.steps):
                t0 = time.perf_counter()
                bindings.load_scene_file(d, jp)
                dt = (time.perf_counter() - t0) * 1e3
                if i >= args.warmup:
                    times.append(dt)
                    stats.append(d.load_stats())
            assert d.render_enable_renderer(0, 0)
            d.render_enable_render_target("Hit ID", False)
            d.render_reset()
            d.render_iterate()
            hid = d.get_target_image("Hit ID").copy()
            ref = bindings.DllInterface()
            bindings.load_scene_spec(ref, loaded)
            assert ref.render_enable_renderer(0, 0)
            ref.render_enable_render_target("Hit ID", False)
            ref.render_iterate()
            same = bool(np.array_equal(hid, ref.get_target_image("Hit ID")))
            ref.close()
            ms = float(np.median(times))
            mb = os.path.getsize(binp) / 1e6
            core = {k: round(float(np.median([st[k] for st in stats])), 3) for k in ("totalMs", "uploadMs", "bvhMs")}
            out[name] = {"load_ms": round(ms, 2), "file_mb": round(mb, 1), "file_mb_per_s": round(mb / (ms / 1e3), 1),
                         "core_load_ms": core, "hit_ids_equal_api_scene": same}
        d.close()
    line = {"metric": "scene-file load time (JSON + binary, 1.3 M triangles)", "value": out["raw"]["load_ms"],
            "unit": "ms", "higher_is_better": False, "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "data": "synthetic", "dtype": "f32",
            "config": {"workload": "scene_file_load_" + WORKLOAD, "triangles": int(spec.num_prims)},
            "files": out}
    print(json.dumps(line), flush=True)


def run_lights(args):
    """Light list and light tree of 256 instances x 1024 emissive quads + 1
    point light (262 145 leaves), built on the GPU at every scene load
    (light_build.cu: quad corners, Hilbert keys, two stable radix sorts,
    128-sample quad fluxes, the tree level by level, the sorted code map),
    timed on the host around the lights stage of world_load_scenario, next to
    the oracle's single-threaded CPU build of the same tree; the two trees
    are compared byte for byte."""
    import torch
    torch.cuda.set_device(0)
    from mufflon_b200 import bindings, build, scenes
    build.build()
    spec = scenes.emissive_panels(0, 256, 1024, 1, width=WIDTH, height=HEIGHT)
    d = bindings.DllInterface()
    sc = bindings.load_scene_spec(d, spec)
    times = []
    for i in range(args.warmup + args.steps):
        assert d.world_load_scenario(sc)
        if i >= args.warmup:
            times.append(d.load_stats()["otherMs"])
    gpu_tree = d.light_tree()
    d.close()
    ms = float(np.median(times))
    n = len(gpu_tree[0])
    cpu = None
    if not args.no_cpu_baseline:
        from oracle import pyoracle
        osc = pyoracle.OracleScene(spec)
        ref = osc.light_tree()
        same = all(np.array_equal(a, b) for a, b in zip(gpu_tree[:4], ref[:4])) and \
            np.float32(gpu_tree[4]).view(np.uint32) == np.float32(ref[4]).view(np.uint32)
        cpu = {"value": round(osc.light_build_ms(), 2), "unit": "ms", "cores": 1, "kind": "port",
               "sample": "the same 262 145-light build (light_tree.cpp restated, one thread)", "tree_identical": bool(same)}
    line = {"metric": "light-tree build time (262 145 lights)", "value": round(ms, 3), "unit": "ms",
            "higher_is_better": False, "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "data": "synthetic",
            "dtype": "f32", "config": {"workload": "emissive_panels_256x1024_quads_1_point", "lights": n},
            "note": "host wall time of the lights stage of world_load_scenario (light build + materials + textures, one sync)",
            "cpu_baseline": cpu}
    print(json.dumps(line), flush=True)


def run_lt(args):
    """The light tracer ("Lighttracer", lt.cu) on the headline scene (the
    1080p icosphere, its point light and colored background): 16 iterations
    of 1920 x 1080 photons per step, path length up to 10. Device time per
    iteration from CUDA events around the launches; rays = extension rays +
    camera-connection shadow rays. The CPU baseline is one iteration of the
    oracle's light tracer on all host cores."""
    import torch
    W, H = args.resolution
    torch.cuda.set_device(0)
    from mufflon_b200 import bindings, build, scenes
    build.build()
    spec = scenes.displaced_icosphere(0, subdiv=args.subdiv, width=W, height=H)
    d = bindings.DllInterface()
    bindings.load_scene_spec(d, spec)
    assert d.render_enable_renderer(1, 0)
    assert d.renderer_set_parameter_int("Max. path length", MAX_PATH)
    assert d.renderer_set_parameter_int("Megakernel", int(args.megakernel))
    d.render_enable_render_target("Radiance", False)
    iters = SPP_PER_FRAME
    for _ in range(args.warmup * iters):
        d.render_iterate()
    torch.cuda.synchronize()
    ms = rays = shadow = 0.0
    t0 = time.perf_counter()
    for _ in range(args.steps * iters):
        d.render_iterate()
        st = d.render_stats()
        ms += st["kernelMs"]; rays += st["rays"]; shadow += st["shadowRays"]
        if st["errors"]:
            raise RuntimeError(f"traversal errors reported: {st['errors']}")
    wall = time.perf_counter() - t0
    img = d.get_target_image("Radiance")
    d.close()
    photons = args.steps * iters * W * H
    cpu = None
    if not args.no_cpu_baseline:
        from oracle import pyoracle
        threads = os.cpu_count() or 1
        lt = pyoracle.OracleLightTracer(pyoracle.OracleScene(spec), seed=0, max_path=MAX_PATH)
        t1 = time.perf_counter()
        lt.iterate(threads)
        el = time.perf_counter() - t1
        r = lt.stats()["rays"]
        cpu = {"value": round(r / el / 1e6, 3), "unit": "Mrays/s", "cores": threads, "kind": "port",
               "sample": f"one iteration: {W * H} photons, {r} rays, {el:.1f} s"}
    line = {"metric": "light tracer Mrays/s at 1080p", "value": round(rays / ms / 1e3, 2), "unit": "Mrays/s",
            "higher_is_better": True, "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "data": "synthetic",
            "dtype": "f32", "ms_per_step": round(ms / args.steps, 3),
            "config": {"workload": f"displaced_icosphere_{spec.num_prims - 1}tri_{W}x{H}_lt_16it_depth{MAX_PATH}",
                       "schedule": "single kernel" if args.megakernel else "stages per path length",
                       "photons_per_step": iters * W * H,
                       "l2": "inputs larger than L2 (BVH + triangle soup + image > 126 MB)"},
            "photons_per_s": round(photons / (ms / 1e3), 1), "rays_per_step": int(rays / args.steps),
            "shadow_rays_per_step": int(shadow / args.steps),
            "e2e": {"value": round(rays / wall / 1e6, 2), "unit": "Mrays/s", "note": "wall clock around render_iterate + stats"},
            "image_mean": [round(float(x), 5) for x in img.reshape(-1, 3).mean(0)],
            "cpu_baseline": cpu}
    print(json.dumps(line), flush=True)


def run_bpt(args, vcm=False):
    """The bidirectional path tracer ("Bidirectional Pathtracer", bpt.cu), or
    with vcm vertex connection and merging ("Vertex Connection and Merging",
    vcm.cu, merge radius --merge-radius of the scene's diagonal), on the
    headline scene (1080p icosphere, point light, colored background): 16
    iterations of one light and one view subpath per pixel per step, path
    length up to 10. Device time from CUDA events; rays = subpath segments +
    connection shadow rays. The CPU baseline is one iteration of the oracle's
    renderer on all host cores at 480 x 270 (the same scene and camera)."""
    import dataclasses
    import torch
    W, H = args.resolution
    torch.cuda.set_device(0)
    from mufflon_b200 import bindings, build, scenes
    build.build()
    spec = scenes.displaced_icosphere(0, subdiv=args.subdiv, width=W, height=H)
    d = bindings.DllInterface()
    bindings.load_scene_spec(d, spec)
    assert d.render_enable_renderer(4 if vcm else 3, 0)
    assert d.renderer_set_parameter_int("Max. path length", MAX_PATH)
    if vcm:
        assert d.renderer_set_parameter_float("Relative merge radius", args.merge_radius)
    else:
        assert d.renderer_set_parameter_int("Megakernel", int(args.megakernel))
    d.render_enable_render_target("Radiance", False)
    iters = SPP_PER_FRAME
    for _ in range(args.warmup * iters):
        d.render_iterate()
    torch.cuda.synchronize()
    ms = rays = shadow = 0.0
    t0 = time.perf_counter()
    for _ in range(args.steps * iters):
        d.render_iterate()
        st = d.render_stats()
        ms += st["kernelMs"]; rays += st["rays"]; shadow += st["shadowRays"]
        if st["errors"]:
            raise RuntimeError(f"traversal errors reported: {st['errors']}")
    wall = time.perf_counter() - t0
    img = d.get_target_image("Radiance")
    d.close()
    cpu = None
    if not args.no_cpu_baseline:
        from oracle import pyoracle
        threads = os.cpu_count() or 1
        small = dataclasses.replace(spec, width=W // 4, height=H // 4)
        if vcm:
            ob = pyoracle.OracleVcm(pyoracle.OracleScene(small), seed=0, max_path=MAX_PATH, merge_radius=args.merge_radius)
        else:
            ob = pyoracle.OracleBidirPathTracer(pyoracle.OracleScene(small), seed=0, max_path=MAX_PATH)
        t1 = time.perf_counter()
        ob.iterate(threads)
        el = time.perf_counter() - t1
        r = ob.stats()["rays"]
        cpu = {"value": round(r / el / 1e6, 3), "unit": "Mrays/s", "cores": threads, "kind": "port",
               "sample": f"one iteration at {small.width}x{small.height}: {r} rays, {el:.1f} s"}
    name = "vertex connection and merging" if vcm else "bidirectional path tracer"
    config = {"workload": f"displaced_icosphere_{spec.num_prims - 1}tri_{W}x{H}_{'vcm' if vcm else 'bpt'}_16it_depth{MAX_PATH}",
              "schedule": "single kernel" if args.megakernel and not vcm else "stages per path length",
              "samples_per_step": iters * W * H,
              "l2": "inputs larger than L2 (BVH + triangle soup + image > 126 MB)"}
    if vcm:
        config["relative_merge_radius"] = args.merge_radius
    line = {"metric": f"{name} Mrays/s at 1080p", "value": round(rays / ms / 1e3, 2), "unit": "Mrays/s",
            "higher_is_better": True, "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "data": "synthetic",
            "dtype": "f32", "ms_per_step": round(ms / args.steps, 3), "config": config,
            "samples_per_s": round(args.steps * iters * W * H / (ms / 1e3), 1),
            "rays_per_step": int(rays / args.steps), "shadow_rays_per_step": int(shadow / args.steps),
            "e2e": {"value": round(rays / wall / 1e6, 2), "unit": "Mrays/s", "note": "wall clock around render_iterate + stats"},
            "image_mean": [round(float(x), 5) for x in img.reshape(-1, 3).mean(0)],
            "cpu_baseline": cpu}
    print(json.dumps(line), flush=True)


def run_instanced(args):
    """Config 2: 4 096 rotated and scaled instances of 10 noise-displaced
    meshes (10 k - 200 k triangles) plus one object of 20 000 spheres, camera
    inside the box; 1920 x 1080, 64 spp per step, path length 12, Russian
    roulette from length 3. Device time from CUDA events; the load's object
    and instance hierarchy build times come from world_load_scenario."""
    import torch
    torch.cuda.set_device(0)
    from mufflon_b200 import bindings, build, scenes
    build.build()
    spec = scenes.instanced_scene(0, width=WIDTH, height=HEIGHT)
    d = bindings.DllInterface()
    sc = bindings.load_scene_spec(d, spec)
    assert d.render_enable_renderer(0, 0)
    for k, v in {"Max. path length": 12, "RR start depth": 3}.items():
        assert d.renderer_set_parameter_int(k, v)
    spp = 64
    for _ in range(args.warmup):
        d.render_iterate()
    torch.cuda.synchronize()
    ms = rays = 0.0
    for _ in range(args.steps * spp):
        d.render_iterate()
        st = d.render_stats()
        ms += st["kernelMs"]; rays += st["rays"]
        if st["errors"]:
            raise RuntimeError(f"traversal errors reported: {st['errors']}")
    loads = []
    for _ in range(3):
        assert d.world_load_scenario(sc)
        loads.append(d.load_stats())
    d.close()
    unique = sum(len(l.triangles) for l in spec.lods)
    inst_tris = int(sum(len(spec.lods[i].triangles) for i in spec.instance_lod))
    line = {"metric": "instanced scene Mrays/s at 1080p", "value": round(rays / ms / 1e3, 2), "unit": "Mrays/s",
            "higher_is_better": True, "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "data": "synthetic",
            "dtype": "f32", "ms_per_step": round(ms / args.steps, 3),
            "config": {"workload": "instanced_4096x10meshes_20000spheres_1920x1080_64spp_depth12_rr3",
                       "unique_triangles": unique, "instanced_triangles": inst_tris,
                       "instances": int(len(spec.instance_lod)), "spheres": int(len(spec.lods[-1].spheres))},
            "rays_per_step": int(rays / args.steps),
            "load_ms": {k: round(float(np.median([l[k] for l in loads])), 3)
                        for k in ("totalMs", "uploadMs", "bvhMs", "instanceBvhMs")}}
    print(json.dumps(line), flush=True)


def dataclasses_replace_texture(spec, tex3):
    import dataclasses
    t = np.ones(tex3.shape[:2] + (4,), np.float32)
    t[..., :3] = tex3
    return dataclasses.replace(spec, textures=[t])


def main():
    args = parse()
    if args.workload == "batch":
        run_batch(args)
        return
    if args.workload == "adjoint":
        run_adjoint(args)
        return
    if args.workload == "load":
        run_load(args)
        return
    if args.workload == "lights":
        run_lights(args)
        return
    if args.workload == "lt":
        run_lt(args)
        return
    if args.workload == "bpt":
        run_bpt(args)
        return
    if args.workload == "vcm":
        run_bpt(args, vcm=True)
        return
    if args.workload == "instanced":
        run_instanced(args)
        return
    if args.impl == "reference":
        run_reference(args)
    else:
        run_b200(args)


if __name__ == "__main__":
    main()
