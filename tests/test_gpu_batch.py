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


def test_enqueued_rebuild_and_cuda_graph():
    """btc_batch_rebuild with BTC_BUILD_ASYNC (same graphs' sizes, device edges) enqueues
    the build without a wait, so rebuild + count can be captured in a CUDA graph; replays
    count whatever edges the buffers hold then."""
    gs = [golden_graph(nm) for nm in NAMES]
    want = [load_golden()[nm]["count"] for nm in NAMES]
    src, dst, off, nv = Batch.concat(gs)
    d_src, d_dst = torch.from_numpy(src).cuda(), torch.from_numpy(dst).cuda()
    args = dict(src=d_src, dst=d_dst, offsets=off, num_vertices=nv, tile_cols=32)
    b = Batch(**args)
    assert b.count().tolist() == want
    out = torch.zeros(len(gs), dtype=torch.int64, device="cuda")
    b.rebuild(**args, asynchronous=True)
    b.count_async(out.data_ptr())
    assert out.cpu().tolist() == want
    assert b.count().tolist() == want  # the waiting call reports the enqueued build's status

    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        b.rebuild(**args, stream=s, asynchronous=True)
        b.count_async(out.data_ptr(), stream=s)
    s.synchronize()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph, stream=s):
        b.rebuild(**args, stream=s, asynchronous=True)
        b.count_async(out.data_ptr(), stream=s)
    for _ in range(3):
        out.zero_()
        graph.replay()
        torch.cuda.synchronize()
        assert out.cpu().tolist() == want
    # other edges in the same buffers (src and dst swapped: the same undirected graphs in
    # another orientation); the replay builds from what the buffers hold now
    tmp = d_src.clone()
    d_src.copy_(d_dst)
    d_dst.copy_(tmp)
    out.zero_()
    graph.replay()
    torch.cuda.synchronize()
    assert out.cpu().tolist() == want
    b.free()


def test_enqueued_rebuild_failures_surface_at_the_next_wait():
    gs = [golden_graph("K33"), golden_graph("stencil27_4")]
    src, dst, off, nv = Batch.concat(gs)
    d_src, d_dst = torch.from_numpy(src).cuda(), torch.from_numpy(dst).cuda()
    b = Batch(src=d_src, dst=d_dst, offsets=off, num_vertices=nv, tile_cols=128)
    want = b.count().tolist()
    # an out-of-range id: nothing counted, BTC_E_RANGE at the waiting count
    bad = d_src.clone()
    bad[3] = 1 << 20
    b.rebuild(src=bad, dst=d_dst, offsets=off, num_vertices=nv, tile_cols=128, asynchronous=True)
    with pytest.raises(BtcError) as e:
        b.count()
    assert e.value.status == _lib.BTC_E_RANGE
    # the batch refuses to count until a rebuild succeeds
    with pytest.raises(BtcError):
        b.count()
    b.rebuild(src=d_src, dst=d_dst, offsets=off, num_vertices=nv, tile_cols=128)
    assert b.count().tolist() == want
    b.free()


def test_enqueued_rebuild_needing_more_tiles_reports_capacity():
    """A batch first built with graph 1's edges all on one vertex pair holds arrays for a
    few tiles; an enqueued rebuild with the real edges (the same sizes) needs more: it
    builds nothing and reports BTC_E_CAPACITY at the next wait; a waiting rebuild grows
    the arrays."""
    gs = [golden_graph("K33"), golden_graph("stencil27_10")]
    want = [load_golden()[nm]["count"] for nm in ("K33", "stencil27_10")]
    src, dst, off, nv = Batch.concat(gs)
    d_src, d_dst = torch.from_numpy(src).cuda(), torch.from_numpy(dst).cuda()
    few_s, few_d = d_src.clone(), d_dst.clone()
    a, z = int(off[1]), int(off[2])
    few_s[a:z], few_d[a:z] = 1, 0
    b = Batch(src=few_s, dst=few_d, offsets=off, num_vertices=nv, tile_cols=128)
    assert b.count().tolist() == [want[0], 0]
    tiles_few = b.info().bcsr.num_blocks
    b.rebuild(src=d_src, dst=d_dst, offsets=off, num_vertices=nv, tile_cols=128, asynchronous=True)
    out = torch.full((2,), 7, dtype=torch.int64, device="cuda")
    b.count_async(out.data_ptr())
    torch.cuda.synchronize()
    assert out.cpu().tolist() == [0, 0]  # nothing built, nothing counted
    with pytest.raises(BtcError) as e:
        b.info()
    assert e.value.status == _lib.BTC_E_CAPACITY
    b.rebuild(src=d_src, dst=d_dst, offsets=off, num_vertices=nv, tile_cols=128)
    assert b.count().tolist() == want
    assert b.info().bcsr.num_blocks > tiles_few
    b.free()
