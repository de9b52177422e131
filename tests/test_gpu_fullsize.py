"""Full-size GPU parity: the largest single graph (R-MAT scale 22, descending-degree order)
and a 256-graph subset of the batched mix, each count checked against the reference's own
CPU path (cpu_tc_intersection_lower_triangular, btc/operations/triangle_count_cpu.h:59-101).

* R-MAT scale 22: the golden count, edge count and tile counts were computed once on the
  CPU from the numpy twin of the GPU generator (tests/golden/make_golden.py --large); the
  test generates the same draws on the GPU, builds both tile widths and counts at the
  default tau, tau = 0 (every tile on the binary tensor core) and all-sparse.
* Batched mix: 256 graphs of the 4096-graph mix (the bench's seed), chosen by a seeded
  draw plus the mix's largest SBM, R-MAT and Erdos-Renyi graphs, generated on the GPU;
  each graph's count from one batch launch (both tile widths) must equal the reference's
  CPU count of that graph, computed here on the host.
Counts are integers: the tolerance is zero.
"""
from __future__ import annotations

import json
import os

import numpy as np
import pytest

from conftest import GOLDEN_DIR

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

from btc_b200 import Batch, BitBSR, graphs as G, _lib  # noqa: E402
from oracle import oracle as O  # noqa: E402


def _large(name):
    with open(os.path.join(GOLDEN_DIR, "golden_large.json")) as f:
        return json.load(f)["fixtures"][name]


@pytest.fixture(scope="module")
def rmat22():
    fx = _large("rmat_raw_22_16_s7")
    src, dst, n = G.rmat_raw_torch(**fx["kwargs"], device="cuda")
    assert n == fx["n"] and src.numel() == fx["m_input"]
    yield src, dst, n, fx
    del src, dst
    torch.cuda.empty_cache()


@pytest.mark.parametrize("tile_cols", [128, 32])
def test_rmat22_degree_order_every_tau(rmat22, tile_cols):
    src, dst, n, fx = rmat22
    g = BitBSR(src, dst, n, tile_cols, orient_degree=True)
    try:
        assert g.num_edges == fx["m_lower"]
        assert g.num_tiles == fx[f"tiles_{tile_cols}_degree"]
        for tau in (_lib.BTC_TAU_DEFAULT, 0, _lib.BTC_TAU_ALL_SPARSE):
            assert g.count(tau=tau) == fx["count"], tau
        # an asynchronous rebuild into the same arrays counts the same
        g.rebuild(src, dst, n, tile_cols, orient_degree=True, asynchronous=True)
        out = torch.zeros(1, dtype=torch.int64, device="cuda")
        g.count_async(d_out=out.data_ptr())
        assert int(out.item()) == fx["count"]
    finally:
        g.free()


def test_rmat22_natural_order_same_count(rmat22):
    """The count does not depend on the vertex order (natural ids, 16x128)."""
    src, dst, n, fx = rmat22
    g = BitBSR(src, dst, n, 128)
    try:
        assert g.num_edges == fx["m_lower"]
        assert g.count() == fx["count"]
    finally:
        g.free()


MIX_GRAPHS, MIX_SEED = 4096, 11   # the bench's batched workload (rank 0)
SUBSET = 256
SUBSET_MAX_EDGES = 2_000_000      # the seeded draw's graphs; the largest ones come on top


def _subset():
    plan = G.batch_mix_plan(MIX_GRAPHS, 256, 65536, seed=MIX_SEED)
    sizes = np.array([sum(sg[-1] for sg in segs) for _, _, segs in plan])
    kinds = np.array([k for k, _, _ in plan])
    top = [int(np.flatnonzero(kinds == k)[np.argmax(sizes[kinds == k])]) for k in ("sbm", "rmat", "er")]
    rng = np.random.default_rng(2024)
    pool = [i for i in rng.permutation(MIX_GRAPHS) if sizes[i] <= SUBSET_MAX_EDGES and i not in top]
    pick = sorted(pool[: SUBSET - len(top)])
    # the largest graphs sit in the middle of the batch, among the small ones
    return pick[: len(pick) // 2] + top + pick[len(pick) // 2:], kinds


def test_batch_mix_subset_against_reference_cpu():
    sel, kinds = _subset()
    assert len(sel) == SUBSET
    d_src, d_dst, off, nv, kl = G.batch_mix_device(MIX_GRAPHS, 256, 65536, seed=MIX_SEED, select=sel)
    assert set(kl) == {"er", "sbm", "rmat"}
    h_src, h_dst = d_src.cpu().numpy(), d_dst.cpu().numpy()
    threads = os.cpu_count() or 1
    count_fn = O.ref_cpu_count if O.ref_cpu_available() else O.tc_merge
    want = np.zeros(len(sel), np.uint64)
    for i in range(len(sel)):
        a, z = int(off[i]), int(off[i + 1])
        rp, col, _ = O.lower_csr(h_src[a:z], h_dst[a:z], int(nv[i]))
        want[i] = count_fn(rp, col, threads)
    assert int(want.max()) > 0
    for tile_cols in (32, 128):
        b = Batch(src=d_src, dst=d_dst, offsets=off, num_vertices=nv, tile_cols=tile_cols)
        try:
            got = b.count()
            bad = np.flatnonzero(got != want)
            assert bad.size == 0, [(sel[i], kl[i], int(got[i]), int(want[i])) for i in bad[:5]]
            out = torch.zeros(len(sel), dtype=torch.int64, device="cuda")
            b.count_async(out.data_ptr())
            assert np.array_equal(out.cpu().numpy().astype(np.uint64), want)
        finally:
            b.free()
