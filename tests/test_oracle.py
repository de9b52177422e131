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
