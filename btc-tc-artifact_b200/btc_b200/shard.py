"""One graph counted by several ranks (one process per GPU, torch.distributed).

Every rank builds the same Bit-BSR from the same input, so the sample tiles and their
order agree on all ranks.  ``BitBSR.partition(world)`` cuts [0, num_tiles) into ranges
of about equal estimated count cost; rank r counts its range with
``BitBSR.count_tiles`` and one int64 all-reduce (NCCL over NVLink for CUDA tensors,
gloo for CPU tensors) adds the ranks' counts.  The count of any partition of the tiles
adds up to the single-GPU count, because every tile's term of the sum is independent
of the others.  The reference counts on one GPU; this is the engine's own extension.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import check, lib


def partition_from_costs(bucket_cost, bucket_tiles: int, num_tiles: int, parts: int) -> list[int]:
    """Host half of the partition (btc_partition_from_costs; needs no GPU): tile bounds
    from per-bucket cost estimates, bucket b holding tiles [b*bucket_tiles, (b+1)*bucket_tiles)."""
    cost = np.ascontiguousarray(bucket_cost, dtype=np.uint64)
    b = np.zeros(int(parts) + 1, np.uint32)
    check(lib().btc_partition_from_costs(cost.ctypes.data if len(cost) else None,
                                         C.c_uint64(len(cost)), int(bucket_tiles),
                                         int(num_tiles), int(parts), b.ctypes.data),
          "btc_partition_from_costs")
    return [int(x) for x in b]


def shard_sum(count_range, bounds, group=None, device=None) -> int:
    """Sum over the ranks of ``count_range(bounds[rank], bounds[rank + 1])``.

    ``count_range`` returns an int or a one-element int64 tensor (a CUDA tensor is
    all-reduced in place, on the device).  Every rank calls this once, in the same
    order as its other collectives."""
    import torch
    import torch.distributed as dist

    rank = dist.get_rank(group)
    local = count_range(bounds[rank], bounds[rank + 1])
    if not isinstance(local, torch.Tensor):
        local = torch.tensor([int(local)], dtype=torch.int64, device=device)
    dist.all_reduce(local, op=dist.ReduceOp.SUM, group=group)
    return int(local.item())


def count_sharded(g, group=None, tau: int = -1, bounds=None) -> int:
    """Whole-graph triangle count of BitBSR ``g`` with each rank of ``group`` counting
    one cost-balanced tile range; returns the total on every rank."""
    import torch.distributed as dist

    if bounds is None:
        bounds = g.partition(dist.get_world_size(group))
    return shard_sum(lambda a, b: g.count_tiles(a, b, tau=tau), bounds, group)
