"""CPU tests: the oracle against the golden fixtures, closed forms and the reference's
own CPU path (oracle/_ref/libref_cpu.so) -- the pin that makes the oracle trustworthy."""
from __future__ import annotations

import hashlib
from math import comb

import numpy as np
import pytest

from conftest import golden_graph, load_golden
from oracle import oracle as O

FIXTURES = sorted(load_golden().keys())
FAST = [f for f in FIXTURES if load_golden()[f]["m_lower"] <= 500_000]


def _digest(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()[:16]


@pytest.mark.parametrize("name", FIXTURES)
def test_generator_matches_fixture(name):
    fx = load_golden()[name]
    src, dst, n = golden_graph(name)
    assert n == fx["n"] and len(src) == fx["m_input"]
    assert _digest(np.stack([src, dst]).astype(np.int32)) == fx["edges_digest"]


@pytest.mark.parametrize("name", FIXTURES)
def test_merge_count_matches_golden(name):
    fx = load_golden()[name]
    src, dst, n = golden_graph(name)
    rp, col, _ = O.lower_csr(src, dst, n)
    assert len(col) == fx["m_lower"]
    assert O.tc_merge(rp, col) == fx["count"]


@pytest.mark.parametrize("name", FAST)
@pytest.mark.parametrize("tile_cols", [32, 128])
def test_bitbsr_count_matches_golden(name, tile_cols):
    fx = load_golden()[name]
    src, dst, n = golden_graph(name)
    rp, col, _ = O.lower_csr(src, dst, n)
    b = O.bitbsr_build(rp, col, n, tile_cols)
    assert b["num_blocks"] == fx[f"tiles_{tile_cols}"]
    assert {k: _digest(b[k]) for k in ("indptr", "indices", "row_indices", "blocks")} == \
        fx[f"digest_{tile_cols}"]
    assert O.bitbsr_count(b) == fx["count"]
    # invariants of the layout: sorted unique column blocks per row block, popcount = edges
    ip = b["indptr"]
    for I in range(b["n_row_blocks"]):
        seg = b["indices"][ip[I]:ip[I + 1]]
        assert np.all(np.diff(seg.astype(np.int64)) > 0)
        assert np.all(b["row_indices"][ip[I]:ip[I + 1]] == I)
    assert int(np.unpackbits(b["blocks"].view(np.uint8)).sum()) == fx["m_lower"]


@pytest.mark.parametrize("name", FAST)
def test_degree_order_keeps_count(name):
    fx = load_golden()[name]
    src, dst, n = golden_graph(name)
    rp, col, rank = O.lower_csr(src, dst, n, "degree")
    assert sorted(rank.tolist()) == list(range(n))
    assert O.tc_merge(rp, col) == fx["count"]
    b = O.bitbsr_build(rp, col, n, 128)
    assert b["num_blocks"] == fx["tiles_128_degree"]
    assert O.bitbsr_count(b) == fx["count"]


@pytest.mark.parametrize("n", [3, 4, 7, 16, 17, 33, 64])
def test_complete_graph_closed_form(n):
    from btc_b200 import graphs as G
    src, dst, _ = G.complete(n)
    rp, col, _ = O.lower_csr(src, dst, n)
    assert O.tc_merge(rp, col) == comb(n, 3)
    for C in (32, 128):
        assert O.bitbsr_count(O.bitbsr_build(rp, col, n, C)) == comb(n, 3)


def test_bipartite_stencil_has_no_triangles():
    from btc_b200 import graphs as G
    src, dst, n = G.stencil7(12)
    rp, col, _ = O.lower_csr(src, dst, n)
    assert O.tc_merge(rp, col) == 0


def test_duplicates_selfloops_both_directions():
    # K4 given as both directions, with duplicates and self-loops: still 4 triangles
    src = np.array([0, 1, 0, 2, 0, 3, 1, 2, 1, 3, 2, 3, 3, 3, 2, 0], np.int32)
    dst = np.array([1, 0, 2, 0, 3, 0, 2, 1, 3, 1, 3, 2, 3, 1, 0, 0], np.int32)
    rp, col, _ = O.lower_csr(src, dst, 4)
    assert len(col) == 6
    assert O.tc_merge(rp, col) == 4


def test_empty_and_out_of_range():
    rp, col, _ = O.lower_csr(np.zeros(0, np.int32), np.zeros(0, np.int32), 10)
    assert len(col) == 0 and O.tc_merge(rp, col) == 0
    b = O.bitbsr_build(rp, col, 10, 128)
    assert b["num_blocks"] == 0 and O.bitbsr_count(b) == 0
    with pytest.raises(ValueError):
        O.lower_csr(np.array([0], np.int32), np.array([10], np.int32), 10)


@pytest.mark.skipif(not O.ref_cpu_available(), reason="oracle/_ref not built")
@pytest.mark.parametrize("name", FIXTURES)
def test_reference_cpu_pins_oracle(name):
    """The reference's own cpu_tc_intersection_lower_triangular agrees with the oracle."""
    src, dst, n = golden_graph(name)
    rp, col, _ = O.lower_csr(src, dst, n)
    assert O.ref_cpu_count(rp, col) == O.tc_merge(rp, col) == load_golden()[name]["count"]


def test_planted_mistake_is_caught():
    """A corrupted Bit-BSR (one bit flipped in the oracle's copy) changes the count,
    so the parity tests can detect a wrong tile."""
    src, dst, n = golden_graph("K33")
    rp, col, _ = O.lower_csr(src, dst, n)
    b = O.bitbsr_build(rp, col, n, 32)
    good = O.bitbsr_count(b)
    b["blocks"] = b["blocks"].copy()
    b["blocks"][5] ^= np.uint32(1 << 3)
    assert O.bitbsr_count(b) != good


# ---------------------------------------------------------------------------
# HashOrder (reorder.h:411-587)
# ---------------------------------------------------------------------------
def test_hashorder_params_match_engine():
    """The oracle draws (a_j, b_j) with its own C++ <random> helper; the engine's host
    code must draw the same values (both follow reorder.h:495-506)."""
    from btc_b200 import hashorder_params
    for H in (1, 4, 16, 64):
        oa, ob = O.hashorder_params(H)
        ea, eb = hashorder_params(H)
        assert np.array_equal(oa, ea) and np.array_equal(ob, eb)
        assert oa.min() >= 1 and ob.max() <= 4294967290


@pytest.mark.parametrize("name", ["stencil27_10", "rmat_12_16_s7", "K33", "er_1000_8_s3"])
@pytest.mark.parametrize("hops", [0, 1, 2])
def test_oracle_hashorder_keeps_the_graph(name, hops):
    """HashOrder is a relabelling: a permutation of [0, n), oriented output, same count."""
    src, dst, n = golden_graph(name)
    rp, col, _ = O.lower_csr(src, dst, n)
    rows = np.repeat(np.arange(n, dtype=np.int32), np.diff(rp))
    r2, c2, perm = O.hashorder(rows, col, n, num_hashes=8, num_hops=hops)
    assert np.array_equal(np.sort(perm), np.arange(n))
    assert np.all(r2 >= c2)
    rp2, col2, _ = O.lower_csr(r2, c2, n)
    assert O.tc_merge(rp2, col2) == load_golden()[name]["count"]


def test_oracle_hashorder_groups_twins():
    """Two vertices with the same closed neighbourhood get the same signature, so the
    order places them next to each other."""
    # 0 and 1 are twins (both adjacent to each other and to 2, 3); 4..9 hang off 5
    rows = np.array([1, 2, 2, 3, 3, 5, 6, 7, 8, 9, 4], np.int32)
    cols = np.array([0, 0, 1, 0, 1, 4, 5, 5, 5, 5, 3], np.int32)
    _, _, perm = O.hashorder(rows, cols, 10)
    assert abs(int(perm[0]) - int(perm[1])) == 1


def test_should_reorder_follows_the_reference_rules():
    """btc_should_reorder against the decision trees of convert.h:443-575 (B200 is
    sm_100, which takes the Hopper/Ampere tree)."""
    from btc_b200 import should_reorder as sr
    # sm_100: N <= 5000 skip; avg degree <= 28.93 reorder; log E <= 6.03 skip;
    # log N <= 5.95 reorder, else skip
    assert not sr(5000, 20000, 100)
    assert sr(5001, 20000, 100)
    assert sr(16384, 130990, 100) and sr(262144, 3298428, 100)
    assert not sr(20000, 1000000, 100)            # avg 100, E = 10^6
    assert sr(500000, 10000000, 100)              # avg 40, log N 5.70
    assert not sr(4194304, 64153542, 100)         # config 3: log N 6.62
    assert sr(800000, 12000000, 90) and not sr(800000, 12000000, 80)  # 5.95 vs 5.80
    # structured names with E > 10^2.04 are skipped on every device
    assert not sr(100000, 300000, 100, "roadNet-CA")
    assert not sr(100000, 300000, 120, "delaunay_n17")
    # sm_120: log N <= 3.65 skip; log avg <= 1.84 reorder unless avg > 35 and N > 500000;
    # log N <= 4.96 skip; else reorder
    assert not sr(4000, 40000, 120)
    assert sr(10000, 100000, 120)
    assert not sr(600000, 12000000, 120)          # avg 40 > 35, N > 500000
    assert not sr(50000, 2000000, 120)            # avg 80, log N 4.70
    assert sr(200000, 8000000, 120)               # avg 80, log N 5.30
    assert not sr(0, 0, 100) and not sr(10, 0, 100)
