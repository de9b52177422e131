"""GPU tests of the batched path (btc_batch_*): one build and one count launch over many
graphs must give every graph the count it gets alone, and the union Bit-BSR must equal
the oracle's Bit-BSR of the block-diagonal union graph byte for byte."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import golden_graph, load_golden

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

from btc_b200 import Batch, BitBSR, BtcError, graphs as G, _lib  # noqa: E402
from oracle import oracle as O  # noqa: E402

NAMES = ["K4", "K33", "K130", "stencil7_8", "stencil27_4", "stencil27_10", "er_1000_8_s3",
         "rmat_10_8_s11", "rmat_12_16_s7_deg", "sbm_600_8_dense", "sbm_2000_8_s2", "K5"]


@pytest.mark.parametrize("tile_cols", [32, 128])
@pytest.mark.parametrize("device_input", [False, True])
def test_batch_counts_and_union_layout(tile_cols, device_input):
    gs = [golden_graph(nm) for nm in NAMES]
    want = [load_golden()[nm]["count"] for nm in NAMES]
    if device_input:
        src, dst, off, nv = Batch.concat(gs)
        b = Batch(src=torch.from_numpy(src).cuda(), dst=torch.from_numpy(dst).cuda(), offsets=off,
                  num_vertices=nv, tile_cols=tile_cols)
    else:
        b = Batch(gs, tile_cols=tile_cols)
    assert b.count().tolist() == want
    assert b.count(tau=0).tolist() == want
    assert b.count(tau=_lib.BTC_TAU_ALL_SPARSE).tolist() == want
    us, ud, un = G.union_graph(gs)
    rp, col, _ = O.lower_csr(us, ud, un)
    ref = O.bitbsr_build(rp, col, un, tile_cols)
    h = b.to_host()
    for k in ("indptr", "indices", "row_indices", "blocks"):
        assert np.array_equal(h[k], ref[k]), k
    assert b.info().num_edges == len(col)
    ro = b.row_offsets()
    assert ro[0] == 0 and ro[-1] == (un + 15) // 16
    b.free()


def test_batch_with_empty_graphs_and_raw_duplicates():
    gs = [(np.zeros(0, np.int32), np.zeros(0, np.int32), 0),
          golden_graph("K33"),
          (np.zeros(0, np.int32), np.zeros(0, np.int32), 50),
          (np.array([3, 3, 1, 0, 2, 0, 1], np.int32), np.array([3, 1, 3, 1, 0, 2, 2], np.int32), 4),
          (np.zeros(0, np.int32), np.zeros(0, np.int32), 0),
          golden_graph("stencil27_4")]
    b = Batch(gs, tile_cols=128)
    assert b.count().tolist() == [0, 5456, 0, 1, 0, 1296]


def test_batch_matches_single_graph_path_on_mixed_workload():
    graphs = G.batch_mix(48, n_min=256, n_max=4096, seed=3)
    b = Batch([(s, d, n) for s, d, n, _ in graphs], tile_cols=32)
    got = b.count()
    for (s, d, n, kind), c in zip(graphs, got):
        single = BitBSR(torch.from_numpy(s).cuda(), torch.from_numpy(d).cuda(), n, 32).count()
        rp, col, _ = O.lower_csr(s, d, n)
        assert int(c) == single == O.tc_merge(rp, col), kind
    b.rebuild([(s, d, n) for s, d, n, _ in graphs[::-1]], tile_cols=128)
    assert b.count().tolist() == got[::-1].tolist()


def test_batch_rejects_bad_input():
    with pytest.raises(BtcError) as e:
        Batch([(np.array([0], np.int32), np.array([9], np.int32), 5)], tile_cols=128)
    assert e.value.status == _lib.BTC_E_RANGE
    with pytest.raises(BtcError):
        Batch([(np.array([0], np.int32), np.array([1], np.int32), 5)], tile_cols=64)
