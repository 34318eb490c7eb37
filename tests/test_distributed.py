"""Rank combination logic of multi-GPU rendering, run as two gloo ranks on CPU."""
import os
import socket

import numpy as np
import pytest

from mufflon_b200 import distributed as D


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import torch
    import torch.distributed as dist
    from datetime import timedelta
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        rng = np.random.default_rng(100 + rank)
        img = torch.from_numpy(rng.random((6, 5, 3)).astype(np.float32))
        spp = 3 + 5 * rank
        mean, total = D.combine_images(img, spp)
        rows = torch.full((D.row_band(7, world, rank)[1] - D.row_band(7, world, rank)[0], 4, 3), float(rank + 1))
        full = D.gather_rows(rows, 7)
        out.put((rank, mean.numpy(), total, full.numpy()))
    finally:
        dist.destroy_process_group()


def test_rank_seed_and_bands():
    assert D.rank_seed(0, 0) == 0 and D.rank_seed(0, 3) == 3
    assert D.rank_seed(2 ** 31 - 1, 1) == -(2 ** 31)
    for h in [1, 7, 1080]:
        for w in [1, 2, 3, 8]:
            bands = [D.row_band(h, w, r) for r in range(w)]
            assert bands[0][0] == 0 and bands[-1][1] == h
            assert all(bands[i][1] == bands[i + 1][0] for i in range(w - 1))
            sizes = [e - b for b, e in bands]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        D.row_band(10, 2, 2)


def test_two_gloo_ranks_combine():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted([q.get(timeout=120) for _ in procs], key=lambda x: x[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    imgs = [np.random.default_rng(100 + r).random((6, 5, 3)).astype(np.float32) for r in range(2)]
    want = D.weighted_mean_reference(imgs, [3, 8])
    for rank, mean, total, full in res:
        assert total == 11
        np.testing.assert_allclose(mean, want, rtol=1e-6, atol=1e-7)
        b0, e0 = D.row_band(7, 2, 0)
        assert np.all(full[b0:e0] == 1.0) and np.all(full[e0:] == 2.0)
