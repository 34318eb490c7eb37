"""Autotuner of the path tracer's schedule for a loaded scene.

It times a few iterations of every candidate setting of the renderer's tuning
parameters and keeps the fastest:

* "Megakernel": the node width of the traversed hierarchy (0: the 8-wide one
  with the wavefront schedule, 1: the binary one with one kernel per path);
* "Trace blocks per SM": the trace kernel's register budget (block shape);
* "Wavefront bounces" and "Tail paths": how many bounces always run as
  separate launches, and the queue length at or below which one launch
  finishes the remaining paths;
* "Trace refill lanes": how many idle lanes of a warp are refilled together;
* "Ray sort bits": the resolution of the coherence binning of queued rays
  (0: traced in queue order).

Every candidate renders the same pixels with the same random numbers, so the
images are identical and only the time differs. Tuning resets the
accumulation. `mufflon_render_batch` takes these settings from the first
job's instance.
"""
from __future__ import annotations

import itertools
from typing import Dict, List, Optional

PARAMS = {"megakernel": "Megakernel", "trace_blocks": "Trace blocks per SM",
          "wavefront_bounces": "Wavefront bounces", "refill_lanes": "Trace refill lanes", "tail_paths": "Tail paths",
          "sort_bits": "Ray sort bits"}


def default_candidates() -> List[Dict[str, int]]:
    c = [dict(megakernel=0, trace_blocks=b, wavefront_bounces=k, refill_lanes=32, tail_paths=t)
         for b, k, t in itertools.product((4, 6), (1, 2), (32768, 98304, 262144))]
    c += [dict(megakernel=0, trace_blocks=6, wavefront_bounces=2, refill_lanes=32, tail_paths=98304, sort_bits=s)
          for s in (0, 16)]
    c.append(dict(megakernel=1))
    return c


def _apply(dll, cand: Dict[str, int]):
    for k, v in cand.items():
        if not dll.renderer_set_parameter_int(PARAMS[k], int(v)):
            raise ValueError(f"cannot set {PARAMS[k]}")


def autotune(dll, iterations: int = 3, warmup: int = 1, candidates: Optional[List[Dict[str, int]]] = None) -> dict:
    """Times each candidate on `dll`'s loaded scene (device time of
    `iterations` iterations after `warmup`), applies the fastest and returns
    {"best": candidate, "ms_per_iteration": t, "table": [(candidate, t), ...]}."""
    cands = candidates or default_candidates()
    saved = {k: dll.renderer_get_parameter_int(PARAMS[k]) for k in PARAMS}
    table = []
    try:
        for cand in cands:
            _apply(dll, dict(saved, **cand))
            dll.render_reset()
            for _ in range(warmup):
                dll.render_iterate()
            ms = 0.0
            for _ in range(iterations):
                dll.render_iterate()
                ms += dll.render_stats()["kernelMs"]
            table.append((dict(cand), ms / iterations))
    except Exception:
        _apply(dll, saved)
        raise
    best, t = min(table, key=lambda x: x[1])
    _apply(dll, dict(saved, **best))
    dll.render_reset()
    return {"best": best, "ms_per_iteration": t, "table": table}
