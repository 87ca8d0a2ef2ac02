"""Multi-GPU partitioning: pure host logic plus world_size-2 gloo runs on CPU
(the same code paths bench.py takes with NCCL on GPUs)."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from pedalsky_b200 import sharding


def test_partition_views_covers_all_once_and_balances():
    rng = np.random.default_rng(3)
    costs = [sharding.view_cost(int(w), int(h), int(s), int(l)) for w, h, s, l in
             zip(rng.integers(256, 3840, 64), rng.integers(256, 2160, 64),
                 rng.integers(48, 161, 64), rng.integers(1, 4, 64))]
    for ws in (1, 2, 3, 8):
        parts = sharding.partition_views(costs, ws)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(64))
        loads = [sum(costs[i] for i in p) for p in parts]
        # LPT bound: max load <= mean + largest item
        assert max(loads) <= sum(costs) / ws + max(costs) + 1e-6
    assert sharding.partition_views([5.0, 5.0], 2) == [[0], [1]]
    with pytest.raises(ValueError):
        sharding.partition_views([1.0], 0)


def test_row_bands_are_contiguous_and_weighted():
    bands = sharding.row_bands(1080, 4)
    assert bands[0].y0 == 0 and bands[-1].y1 == 1080
    assert all(a.y1 == b.y0 for a, b in zip(bands, bands[1:]))
    assert [b.y1 - b.y0 for b in bands] == [270] * 4
    w = np.concatenate([np.full(600, 10.0), np.full(480, 1.0)])  # sky rows cost more
    wb = sharding.row_bands(1080, 2, w)
    assert wb[0].y1 < 540  # the expensive upper rows are split earlier
    one = sharding.row_bands(7, 8)  # more ranks than rows: empty bands allowed
    assert sum(b.y1 - b.y0 for b in one) == 7
    with pytest.raises(ValueError):
        sharding.row_bands(10, 2, np.ones(9))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        H, W = 37, 11
        bands = sharding.row_bands(H, world, np.linspace(1, 3, H))
        band = bands[rank]
        # stand-in for the march: each pixel's value is a function of its
        # global coordinates, as the kernel's output depends only on them
        ys = torch.arange(band.y0, band.y1, dtype=torch.float32)[:, None, None]
        xs = torch.arange(W, dtype=torch.float32)[None, :, None]
        local = (ys * 100 + xs).expand(-1, -1, 4).contiguous()
        full = sharding.gather_rows(local, band, bands)
        t = sharding.max_over_ranks(1.5 + rank)
        parts = sharding.partition_views([3, 9, 4, 1, 7], world)
        q.put((rank, full.numpy(), t, parts))
    finally:
        dist.destroy_process_group()


def test_gloo_world_size_two_gather_and_timing():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    H, W = 37, 11
    want = (np.arange(H)[:, None] * 100 + np.arange(W)[None, :]).astype(np.float32)
    for rank, full, t, parts in res:
        assert full.shape == (H, W, 4)
        assert np.array_equal(full[..., 0], want)
        assert t == 2.5                       # max over ranks
        assert parts == res[0][3]             # every rank computes the same plan
        assert sorted(i for p in parts for i in p) == list(range(5))


def _march_worker(rank, world, port, q):
    """One gloo rank of the two forward partitions, with the FP64 CPU
    restatement standing in for the march kernel: a row band of one frame
    (psc_render's viewport offset does the same on a GPU), all-gathered into
    the frame, and this rank's share of a cost-partitioned set of views."""
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from oracle import pyoracle
        from pedalsky_b200 import scenes
        noise = pyoracle.bake_noise()
        s = scenes.precision_1080p(64, 37)
        luts = pyoracle.bake_luts(s.frame, s.world)
        bands = sharding.row_bands(s.height, world, (s.depth == 0).mean(axis=1) + 0.25)
        band = bands[rank]
        L, T = pyoracle.render(s, noise, luts, precision=pyoracle.FP64, threads=2,
                               rows=(band.y0, band.y1))
        local = torch.from_numpy(np.concatenate([L, T], axis=-1)[band.y0:band.y1].copy())
        full = sharding.gather_rows(local, band, bands).numpy()
        views = scenes.batch_views(5, seed=4, size_scale=0.03)
        costs = [sharding.view_cost(v.width, v.height, v.params.cloud_steps, v.n_layers)
                 for v in views]
        parts = sharding.partition_views(costs, world)
        mine = {}
        for i in parts[rank]:
            v = views[i]
            lv = pyoracle.bake_luts(v.frame, v.world)
            Lv, Tv = pyoracle.render(v, noise, lv, precision=pyoracle.FP64, threads=2)
            mine[i] = np.concatenate([Lv, Tv], axis=-1)
        gathered = [None] * world
        dist.all_gather_object(gathered, mine)
        q.put((rank, full, {k: v for d in gathered for k, v in d.items()}, parts))
    finally:
        dist.destroy_process_group()


def test_gloo_world_size_two_renders_bands_and_views_like_one_process(oracle, oracle_noise):
    """Row bands and view partitions over two gloo ranks reassemble the
    single-process FP64 renders bit for bit (the forward march has no
    exchange step: every pixel is a function of its own coordinates)."""
    from pedalsky_b200 import scenes
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_march_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=600) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    s = scenes.precision_1080p(64, 37)
    luts = oracle.bake_luts(s.frame, s.world)
    L, T = oracle.render(s, oracle_noise, luts, precision=oracle.FP64)
    want = np.concatenate([L, T], axis=-1)
    views = scenes.batch_views(5, seed=4, size_scale=0.03)
    for rank, full, rendered, parts in res:
        assert np.array_equal(full, want)
        assert sorted(rendered) == list(range(5))
        assert all(len(p) > 0 for p in parts)
        for i, img in rendered.items():
            v = views[i]
            lv = oracle.bake_luts(v.frame, v.world)
            Lv, Tv = oracle.render(v, oracle_noise, lv, precision=oracle.FP64)
            assert np.array_equal(img, np.concatenate([Lv, Tv], axis=-1)), i
