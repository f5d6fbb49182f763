"""Multi-GPU sharding of the voxelwise fits: one process per GPU, voxels split across ranks.

The fits are independent per voxel (a voxel's result never depends on another's), so a volume
shards without any exchange on the data path: rank r fits the contiguous voxel range
voxel_shard(v, r, world), with the small design matrices replicated on every GPU, and keeps or
writes its own output shard. gather_shards brings the shards to one rank when a caller wants
the whole result there, with point-to-point sends of each shard (no collective computation);
max_over_ranks takes the slowest rank's time for benchmarks.

The process group is the caller's (torch.distributed, "nccl" between GPUs, "gloo" on CPU).
"""

from __future__ import annotations

import numpy as np


def voxel_shard(v: int, rank: int, world: int) -> slice:
    """The contiguous voxel range of one rank: the first v % world ranks take one voxel more."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} is not in a world of {world}")
    if v < 0:
        raise ValueError("v must be at least 0")
    base, extra = divmod(v, world)
    start = rank * base + min(rank, extra)
    return slice(start, start + base + (1 if rank < extra else 0))


def shard_sizes(v: int, world: int) -> list[int]:
    """The voxel count of every rank's shard."""
    return [voxel_shard(v, r, world).stop - voxel_shard(v, r, world).start for r in range(world)]


def gather_shards(local, v: int, root: int = 0, group=None):
    """The whole (v, ...) result on `root`, assembled in voxel order from every rank's shard
    (`local`: this rank's rows, a torch tensor on the process group's device); None elsewhere.
    Each non-root rank sends its shard to root; root receives them in rank order."""
    import torch
    import torch.distributed as dist

    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    sizes = shard_sizes(v, world)
    if local.shape[0] != sizes[rank]:
        raise ValueError(f"rank {rank} holds {local.shape[0]} rows, its shard has {sizes[rank]}")
    if rank != root:
        if sizes[rank]:
            dist.send(local.contiguous(), dst=root, group=group)
        return None
    out = torch.empty((v, *local.shape[1:]), dtype=local.dtype, device=local.device)
    for r in range(world):
        rows = voxel_shard(v, r, world)
        if r == root:
            out[rows] = local
        elif sizes[r]:
            buf = torch.empty((sizes[r], *local.shape[1:]), dtype=local.dtype, device=local.device)
            dist.recv(buf, src=r, group=group)
            out[rows] = buf
    return out


def max_over_ranks(value: float, device=None, group=None) -> float:
    """The largest value over the ranks (one all-reduce of a scalar; the value itself when no
    process group is initialised)."""
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()):
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())


def shard_rows(array: np.ndarray, rank: int, world: int) -> np.ndarray:
    """This rank's rows of a (v, ...) host array."""
    return array[voxel_shard(len(array), rank, world)]
