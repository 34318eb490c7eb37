"""Multi-GPU rendering helpers: one process per GPU, replicas of the scene.

Pixels and samples of the path tracer are independent, so the work shards
without any exchange inside an iteration. Two partitions are supported:

* sample split (default): every rank renders the whole frame with its own
  seed (`rank_seed`) and the ranks' running means are combined once per
  frame by an spp-weighted all-reduce (`combine_images`);
* row split: rank r renders the row band `row_band(height, world, r)` and
  the bands are gathered.

The reference's hybrid renderer splits by rows (src/core/renderer/pt/
hybrid_pt.cpp:28-48); its per-pixel generator seeding is
Rng(pixel + seed * (numPixels + 1)) (cpu_pt.cpp:40-45), so distinct seeds give
distinct streams for every pixel.

Everything here works with any torch.distributed backend: NCCL over NVLink
for the GPU runs, gloo for the CPU tests.
"""
from __future__ import annotations

from typing import Tuple

import numpy as np


def rank_seed(base_seed: int, rank: int) -> int:
    """Seed of `rank` for a sample-split render: base_seed for rank 0, then
    consecutive seeds (the "Seed" renderer parameter is a 32-bit int)."""
    s = (int(base_seed) + int(rank)) & 0xFFFFFFFF
    return s - (1 << 32) if s >= (1 << 31) else s


def row_band(height: int, world: int, rank: int) -> Tuple[int, int]:
    """Rows [begin, end) of `rank` when `height` rows are split into `world`
    contiguous bands whose sizes differ by at most one."""
    if world <= 0 or not (0 <= rank < world):
        raise ValueError("rank out of range")
    base, extra = divmod(int(height), int(world))
    begin = rank * base + min(rank, extra)
    return begin, begin + base + (1 if rank < extra else 0)


def combine_images(image, spp: int, group=None):
    """spp-weighted mean of the ranks' running-mean images.

    `image` is a torch tensor (on the rank's device for NCCL, on the CPU for
    gloo) holding this rank's mean over `spp` samples. Returns the combined
    mean over all ranks' samples (the same tensor on every rank) and the total
    spp. Two collectives: one all-reduce of the weighted image, one of the
    sample count."""
    import torch
    import torch.distributed as dist
    weighted = image.to(torch.float32) * float(spp)
    dist.all_reduce(weighted, op=dist.ReduceOp.SUM, group=group)
    total = torch.tensor([float(spp)], dtype=torch.float64, device=image.device)
    dist.all_reduce(total, op=dist.ReduceOp.SUM, group=group)
    n = float(total.item())
    if n <= 0:
        raise ValueError("no samples on any rank")
    return weighted / n, int(round(n))


def gather_rows(band, height: int, group=None):
    """Assembles the full image from the ranks' row bands (row split).
    `band` holds this rank's rows (rows, width, channels); returns the
    (height, width, channels) image on every rank."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    b, e = row_band(height, world, rank)
    if band.shape[0] != e - b:
        raise ValueError(f"rank {rank} holds {band.shape[0]} rows, expected {e - b}")
    full = torch.zeros((height,) + tuple(band.shape[1:]), dtype=band.dtype, device=band.device)
    full[b:e] = band
    dist.all_reduce(full, op=dist.ReduceOp.SUM, group=group)
    return full


def weighted_mean_reference(images, spps) -> np.ndarray:
    """The combination `combine_images` computes, on host arrays."""
    acc = np.zeros_like(np.asarray(images[0], np.float64))
    for im, s in zip(images, spps):
        acc += np.asarray(im, np.float64) * s
    return acc / float(sum(spps))
