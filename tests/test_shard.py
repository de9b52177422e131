"""Multi-GPU count plumbing on the CPU: the tile partition (host half of
btc_partition_tiles) and the rank sum, run as world_size 2 and 3 gloo process groups
whose ranks count their tile ranges with the oracle.  The GPU half (partition kernel,
tile-range count, NCCL) is in test_gpu_shard.py."""
from __future__ import annotations

import os
import socket

import numpy as np
import pytest

from conftest import golden_graph, load_golden

from btc_b200 import BtcError
from btc_b200 import shard


def _check_bounds(b, T, parts, bucket):
    assert len(b) == parts + 1 and b[0] == 0 and b[-1] == T
    assert all(b[i] <= b[i + 1] for i in range(parts))
    assert all(x % bucket == 0 or x == T for x in b)


@pytest.mark.parametrize("parts", [1, 2, 3, 7, 8, 64])
def test_partition_balances_costs(parts):
    rng = np.random.default_rng(parts)
    for trial in range(20):
        nb = int(rng.integers(1, 400))
        bucket = int(rng.choice([1, 16, 256]))
        T = (nb - 1) * bucket + int(rng.integers(1, bucket + 1))
        cost = rng.integers(0, 1000, nb).astype(np.uint64)
        if trial % 4 == 0:  # power-law: a few buckets hold most of the cost
            cost = (rng.pareto(0.8, nb) * 100).astype(np.uint64)
        b = shard.partition_from_costs(cost, bucket, T, parts)
        _check_bounds(b, T, parts, bucket)
        total = int(cost.sum())
        for r in range(parts):
            lo, hi = b[r] // bucket, (b[r + 1] + bucket - 1) // bucket
            part = int(cost[lo:hi].sum())
            # a part exceeds an even share by less than the largest bucket, twice over
            assert part <= total / parts + 2 * int(cost.max()) + 1


def test_partition_edge_cases():
    assert shard.partition_from_costs([], 256, 0, 3) == [0, 0, 0, 0]
    assert shard.partition_from_costs([0, 0, 0], 256, 700, 2)[-1] == 700
    b = shard.partition_from_costs([5], 256, 100, 4)  # more parts than buckets
    _check_bounds(b, 100, 4, 256)
    assert shard.partition_from_costs([1, 1, 1, 1], 1, 4, 4) == [0, 1, 2, 3, 4]
    with pytest.raises(BtcError):
        shard.partition_from_costs([1, 1], 256, 1000, 2)  # tiles beyond the buckets
    with pytest.raises(BtcError):
        shard.partition_from_costs([1], 256, 10, 0)


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


SHARD_CASES = [("rmat_12_16_s7_deg", 128), ("rmat_12_16_s7_deg", 32), ("stencil27_16", 128),
               ("K130", 32), ("sbm_600_8_dense", 128), ("stencil7_16", 32)]


def _rank_main(rank, world, port, out_dir):
    import torch.distributed as dist

    from oracle import oracle as O

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world)
    results = []
    try:
        for name, C_ in SHARD_CASES:
            src, dst, n = golden_graph(name)
            rp, col, _ = O.lower_csr(src, dst, n)
            bsr = O.bitbsr_build(rp, col, n, C_)
            T = bsr["num_blocks"]
            # bucket costs: bits of the tiles (any cost gives a valid partition)
            bits = np.unpackbits(bsr["blocks"].view(np.uint8)).reshape(max(T, 1), -1).sum(1)[:T]
            bucket = 16
            nb = (T + bucket - 1) // bucket
            cost = np.zeros(nb, np.uint64)
            np.add.at(cost, np.arange(T) // bucket, bits.astype(np.uint64) + 16)
            bounds = shard.partition_from_costs(cost, bucket, T, world)
            total = shard.shard_sum(lambda a, b: O.bitbsr_count_range(bsr, a, b, 1), bounds)
            # an arbitrary partition (rank 0's random cuts, broadcast) adds up too
            cuts = sorted(np.random.default_rng(7).integers(0, T + 1, world - 1).tolist())
            rb = [0] + cuts + [T]
            total2 = shard.shard_sum(lambda a, b: O.bitbsr_count_range(bsr, a, b, 1), rb)
            results.append((name, C_, total, total2))
    finally:
        dist.destroy_process_group()
    with open(os.path.join(out_dir, f"rank{rank}.txt"), "w") as f:
        for name, C_, total, total2 in results:
            f.write(f"{name} {C_} {total} {total2}\n")


@pytest.mark.parametrize("world", [2, 3])
def test_gloo_shard_sum_matches_whole_count(world, tmp_path):
    import torch.multiprocessing as mp

    mp.start_processes(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world,
                       join=True, start_method="spawn")
    golden = load_golden()
    for r in range(world):
        lines = (tmp_path / f"rank{r}.txt").read_text().split("\n")
        rows = [ln.split() for ln in lines if ln]
        assert len(rows) == len(SHARD_CASES)
        for (name, C_, total, total2) in rows:
            assert int(total) == golden[name]["count"], (name, C_, r)
            assert int(total2) == golden[name]["count"], (name, C_, r)
