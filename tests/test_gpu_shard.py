"""Multi-GPU count pieces on one B200: the cost partition (btc_partition_tiles), the
tile-range count (btc_count_tiles_async) against the oracle's count of the same range,
and the NCCL path of count_sharded at world size 1."""
from __future__ import annotations

import socket

import numpy as np
import pytest

from conftest import golden_graph, load_golden

pytestmark = pytest.mark.gpu

CASES = [("rmat_12_16_s7_deg", 128), ("rmat_12_16_s7_deg", 32), ("rmat_15_16_s7_deg", 128),
         ("stencil27_16", 128), ("stencil27_16", 32), ("er_5000_32_s5", 32), ("K130", 128),
         ("sbm_600_8_dense", 32), ("stencil7_16", 128)]


def _engine(name, C_):
    import torch

    from btc_b200 import BitBSR
    src, dst, n = golden_graph(name)
    return BitBSR(torch.from_numpy(np.asarray(src, np.int32)).cuda(),
                  torch.from_numpy(np.asarray(dst, np.int32)).cuda(), n, C_)


@pytest.mark.parametrize("name,C_", CASES)
def test_partition_ranges_add_up(name, C_):
    from oracle import oracle as O
    g = _engine(name, C_)
    want = load_golden()[name]["count"]
    assert g.count() == want
    src, dst, n = golden_graph(name)
    rp, col, _ = O.lower_csr(src, dst, n)
    bsr = O.bitbsr_build(rp, col, n, C_)
    T = g.num_tiles
    assert T == bsr["num_blocks"]
    for parts in (1, 2, 3, 5, 8, 64):
        b = g.partition(parts)
        assert len(b) == parts + 1 and b[0] == 0 and b[-1] == T
        assert all(b[i] <= b[i + 1] for i in range(parts))
        total = 0
        for r in range(parts):
            c = int(g.count_tiles(b[r], b[r + 1]).item())
            assert c == O.bitbsr_count_range(bsr, b[r], b[r + 1]), (parts, r)
            total += c
        assert total == want, parts
    rng = np.random.default_rng(3)
    for _ in range(5):  # arbitrary cuts, single tiles and empty ranges included
        cuts = sorted(rng.integers(0, T + 1, 4).tolist())
        rb = [0] + cuts + [T]
        assert sum(int(g.count_tiles(rb[i], rb[i + 1]).item()) for i in range(5)) == want
    t = int(rng.integers(0, T))
    assert int(g.count_tiles(t, t + 1).item()) == O.bitbsr_count_range(bsr, t, t + 1)
    assert g.count() == want  # the whole count after range counts (queue word reset)
    g.free()


def test_count_tiles_rejects_bad_ranges():
    from btc_b200 import BtcError
    g = _engine("K130", 128)
    T = g.num_tiles
    for a, b in ((1, 0), (0, T + 1), (T + 1, T + 1)):
        with pytest.raises(BtcError):
            g.count_tiles(a, b)
    with pytest.raises(BtcError):
        g.partition(0)
    g.free()


def test_count_sharded_nccl_world1():
    import torch
    import torch.distributed as dist

    from btc_b200.shard import count_sharded
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    torch.cuda.set_device(0)
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1)
    try:
        for name, C_ in (("rmat_15_16_s7_deg", 128), ("stencil27_16", 32)):
            g = _engine(name, C_)
            assert count_sharded(g) == load_golden()[name]["count"]
            g.free()
    finally:
        dist.destroy_process_group()
