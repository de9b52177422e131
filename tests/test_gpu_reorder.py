"""GPU tests of btc_reorder_hashorder: the relabelled COO against the oracle's numpy
restatement and against the reference's own reorder_hashorder_gpu (oracle/_ref), element
for element; the count is unchanged."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import golden_graph, load_golden

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

import btc_b200  # noqa: E402
from btc_b200 import BitBSR, BtcError, CooMatrix, graphs as G  # noqa: E402
from btc_b200 import _lib  # noqa: E402
from oracle import oracle as O  # noqa: E402


def _lower_coo(src, dst, n):
    rp, col, _ = O.lower_csr(src, dst, n)
    rows = np.repeat(np.arange(n, dtype=np.int32), np.diff(rp)).astype(np.int32)
    return rows, np.asarray(col, np.int32)


def _coo(rows, cols, n):
    coo = CooMatrix(torch.from_numpy(rows).cuda(), torch.from_numpy(cols).cuda(), n)
    return coo


@pytest.mark.parametrize("name", ["stencil27_10", "rmat_12_16_s7", "er_5000_32_s5", "K33",
                                  "sbm_2000_8_s2"])
@pytest.mark.parametrize("hashes,hops", [(16, 1), (4, 0), (8, 2)])
def test_hashorder_matches_oracle(name, hashes, hops):
    src, dst, n = golden_graph(name)
    rows, cols = _lower_coo(src, dst, n)
    coo = _coo(rows, cols, n)
    perm = btc_b200.reorder_hashorder_gpu(coo, num_hashes=hashes, num_hops=hops)
    r2, c2, p2 = O.hashorder(rows, cols, n, num_hashes=hashes, num_hops=hops)
    assert np.array_equal(perm.cpu().numpy(), p2)
    assert np.array_equal(coo.row_indices.cpu().numpy(), r2)
    assert np.array_equal(coo.column_indices.cpu().numpy(), c2)
    g = BitBSR(coo.row_indices, coo.column_indices, n, 32)
    assert g.count() == load_golden()[name]["count"]


@pytest.mark.skipif(not O.ref_gpu_available(), reason="oracle/_ref/libref_gpu.so not built")
@pytest.mark.parametrize("name", ["stencil27_16", "rmat_12_16_s7", "er_5000_32_s5"])
def test_hashorder_matches_the_reference(name):
    """The reference's reorder_hashorder_gpu (reorder.h:443-587, compiled unchanged) on the
    same COO leaves exactly the same arrays."""
    src, dst, n = golden_graph(name)
    rows, cols = _lower_coo(src, dst, n)
    coo = _coo(rows, cols, n)
    btc_b200.reorder_hashorder_gpu(coo)
    rr, rc = O.ref_hashorder(rows, cols, n)
    assert np.array_equal(coo.row_indices.cpu().numpy(), rr)
    assert np.array_equal(coo.column_indices.cpu().numpy(), rc)


def test_hashorder_edge_cases():
    # no edges: identity order of isolated vertices, nothing to relabel
    coo = _coo(np.zeros(0, np.int32), np.zeros(0, np.int32), 5)
    perm = btc_b200.reorder_hashorder_gpu(coo)
    assert np.array_equal(perm.cpu().numpy(), O.hashorder([], [], 5)[2])
    # an id outside [0, n): BTC_E_RANGE and the COO is left as it was
    rows = np.array([1, 2, 7], np.int32)
    cols = np.array([0, 1, 2], np.int32)
    coo = _coo(rows, cols, 5)
    with pytest.raises(BtcError) as e:
        btc_b200.reorder_hashorder_gpu(coo)
    assert e.value.status == _lib.BTC_E_RANGE
    assert np.array_equal(coo.row_indices.cpu().numpy(), rows)
    # unsupported parameters
    coo = _coo(np.array([1], np.int32), np.array([0], np.int32), 2)
    with pytest.raises(BtcError):
        btc_b200.reorder_hashorder_gpu(coo, num_hashes=0)
    with pytest.raises(BtcError):
        btc_b200.reorder_hashorder_gpu(coo, num_hashes=65)


def test_preprocess_reorder_modes():
    """preprocess_for_triangle_counting with reorder=8 is the plain preprocess followed by
    HashOrder; reorder=9 applies the reference's rule (ER n = 8192, mean degree 8,
    qualifies on B200); an unknown mode is refused."""
    src, dst, n = G.erdos_renyi(8192, 8, seed=2)
    src, dst = src.astype(np.int32), dst.astype(np.int32)
    rp, col, _ = O.lower_csr(src, dst, n)
    want = O.tc_merge(rp, col)
    plain = _coo(src, dst, n)
    btc_b200.preprocess_for_triangle_counting(plain, reorder=0)
    assert btc_b200.should_reorder_gpu(plain)
    r2, c2, _ = O.hashorder(plain.row_indices.cpu().numpy(), plain.column_indices.cpu().numpy(),
                            plain.num_rows)
    for mode in (8, 9):
        coo = _coo(src, dst, n)
        btc_b200.preprocess_for_triangle_counting(coo, reorder=mode)
        assert np.array_equal(coo.row_indices.cpu().numpy(), r2)
        assert np.array_equal(coo.column_indices.cpu().numpy(), c2)
        assert BitBSR(coo.row_indices, coo.column_indices, coo.num_rows, 32).count() == want
    with pytest.raises(BtcError):
        btc_b200.preprocess_for_triangle_counting(_coo(src, dst, n), reorder=3)


def test_hashorder_packs_low_degree_graphs_into_fewer_tiles():
    """The point of the reorder: on Erdos-Renyi n=16384 (mean degree 16) the 16x32
    Bit-BSR gets fewer tiles, and the count is unchanged."""
    src, dst, n = G.erdos_renyi(16384, 16, seed=1)
    rows, cols = _lower_coo(src, dst, n)
    before = BitBSR(torch.from_numpy(rows).cuda(), torch.from_numpy(cols).cuda(), n, 32)
    coo = _coo(rows, cols, n)
    btc_b200.reorder_hashorder_gpu(coo)
    after = BitBSR(coo.row_indices, coo.column_indices, n, 32)
    assert after.count() == before.count()
    assert after.num_tiles < before.num_tiles


@pytest.mark.parametrize("mode", ["8", "9"])
def test_compat_cli_reorder_modes(mode, tmp_path):
    """apps/btc_tc_lite.cu honours BTC_REORDER like the reference's preprocess (8: GPU
    HashOrder; 9: when the automatic rule says so, which it does for this ER graph on
    B200); the count is unchanged."""
    import os
    import re
    import subprocess
    src, dst, n = G.erdos_renyi(8192, 8, seed=2)
    rp, col, _ = O.lower_csr(src, dst, n)
    want = O.tc_merge(rp, col)
    path = tmp_path / "er_8192_8.mtx"
    G.write_mtx(str(path), src, dst, n)
    app = os.path.join(os.path.dirname(_lib.LIB_PATH), "btc_tc_lite")
    env = dict(os.environ, BTC_REORDER=mode)
    out = subprocess.run([app, "-i", str(path), "-w", "1", "-r", "2"], capture_output=True,
                         text=True, timeout=120, env=env)
    assert out.returncode == 0, out.stdout + out.stderr
    assert int(re.search(r"Triangles \(GPU\): (\d+)", out.stdout).group(1)) == want
