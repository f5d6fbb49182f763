"""Multi-process sharding on CPU: two gloo ranks over 127.0.0.1 (the GPU path uses nccl with
the same calls). The voxel fits have no exchange step, so what is tested is the host logic:
the shards cover every voxel once, a gather reassembles them in voxel order, and the slowest
rank's time is what every rank sees."""

from __future__ import annotations

import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from larmor_b200.sharding import gather_shards, max_over_ranks, shard_rows, shard_sizes, voxel_shard


@pytest.mark.parametrize("v", [0, 1, 7, 1000, 500040])
@pytest.mark.parametrize("world", [1, 2, 3, 8])
def test_shards_cover_every_voxel_once(v, world):
    covered = np.zeros(v, dtype=int)
    for r in range(world):
        covered[voxel_shard(v, r, world)] += 1
    assert (covered == 1).all()
    sizes = shard_sizes(v, world)
    assert sum(sizes) == v and max(sizes) - min(sizes) <= 1


def test_bad_rank_raises():
    with pytest.raises(ValueError):
        voxel_shard(10, 2, 2)
    with pytest.raises(ValueError):
        voxel_shard(-1, 0, 1)


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, v, results):
    import datetime

    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        full = np.arange(v * 3, dtype=np.float64).reshape(v, 3)
        local = torch.from_numpy(shard_rows(full, rank, world) * 2.0)
        out = gather_shards(local, v, root=0)
        slowest = max_over_ranks(10.0 + rank)
        results[rank] = (None if out is None else out.numpy(), slowest)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("v", [5, 1001])
def test_gather_and_max_over_two_gloo_ranks(v):
    ctx = mp.get_context("spawn")
    manager = ctx.Manager()
    results = manager.dict()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, v, results)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    full = np.arange(v * 3, dtype=np.float64).reshape(v, 3) * 2.0
    out0, slow0 = results[0]
    out1, slow1 = results[1]
    np.testing.assert_array_equal(out0, full)
    assert out1 is None
    assert slow0 == slow1 == 11.0
