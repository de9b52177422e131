"""GPU parity tests: the sm_100a engine against the oracle and the golden fixtures,
called through the C ABI (libbtc_b200.so).  Counts are integers: the bar is bit-exact
equality, and the Bit-BSR arrays must equal the oracle's byte for byte."""
from __future__ import annotations

import hashlib
from math import comb

import numpy as np
import pytest

from conftest import golden_graph, load_golden

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

import btc_b200  # noqa: E402
from btc_b200 import BitBSR, BtcError, graphs as G  # noqa: E402
from btc_b200 import _lib  # noqa: E402
from oracle import oracle as O  # noqa: E402

FIXTURES = sorted(load_golden().keys())
TAUS = [_lib.BTC_TAU_DEFAULT, 0, _lib.BTC_TAU_ALL_SPARSE]


def _digest(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()[:16]


def _dev(a):
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.int32)).cuda()


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    torch.cuda.init()
    yield
    torch.cuda.synchronize()


@pytest.mark.parametrize("radix", [False, True], ids=["bitmap", "radix"])
@pytest.mark.parametrize("tile_cols", [32, 128])
@pytest.mark.parametrize("name", FIXTURES)
def test_build_is_bitexact_and_count_matches(name, tile_cols, radix):
    fx = load_golden()[name]
    src, dst, n = golden_graph(name)
    g = BitBSR(_dev(src), _dev(dst), n, tile_cols, radix=radix)
    h = g.to_host()
    assert h["num_blocks"] == fx[f"tiles_{tile_cols}"]
    assert {k: _digest(h[k]) for k in ("indptr", "indices", "row_indices", "blocks")} == \
        fx[f"digest_{tile_cols}"]
    assert g.num_edges == fx["m_lower"]
    for tau in TAUS:
        assert g.count(tau=tau) == fx["count"], (name, tile_cols, tau)
    g.free()


@pytest.mark.parametrize("tile_cols", [32, 128])
@pytest.mark.parametrize("name", ["K130", "rmat_12_16_s7_deg", "sbm_600_8_dense", "stencil27_10",
                                  "er_1000_8_s3"])
def test_tau_sweep_is_invariant(name, tile_cols):
    """apps/tau_sweep.cu:529-537 checks every tau against the default; here every tau
    must also equal the reference's CPU count."""
    fx = load_golden()[name]
    src, dst, n = golden_graph(name)
    g = BitBSR(_dev(src), _dev(dst), n, tile_cols)
    for tau in [0, 1, 8, 32, 64, 100, 256, 512, 1024, 2048]:
        assert g.count(tau=tau) == fx["count"], tau


@pytest.mark.parametrize("radix", [False, True], ids=["bitmap", "radix"])
@pytest.mark.parametrize("name", ["rmat_12_16_s7", "rmat_15_16_s7_deg", "sbm_2000_8_s2",
                                  "stencil27_16", "K33"])
@pytest.mark.parametrize("tile_cols", [32, 128])
def test_degree_orientation(name, tile_cols, radix):
    fx = load_golden()[name]
    src, dst, n = golden_graph(name)
    g = BitBSR(_dev(src), _dev(dst), n, tile_cols, orient_degree=True, radix=radix)
    assert g.num_tiles == fx[f"tiles_{tile_cols}_degree"]
    rp, col, _ = O.lower_csr(src, dst, n, "degree")
    ref = O.bitbsr_build(rp, col, n, tile_cols)
    h = g.to_host()
    for k in ("indptr", "indices", "row_indices", "blocks"):
        assert np.array_equal(h[k], ref[k]), k
    assert g.count() == fx["count"]


def test_host_input_matches_device_input():
    src, dst, n = golden_graph("er_5000_32_s5")
    fx = load_golden()["er_5000_32_s5"]
    gh = BitBSR(np.ascontiguousarray(src), np.ascontiguousarray(dst), n, 128)
    gd = BitBSR(_dev(src), _dev(dst), n, 128)
    assert gh.count() == gd.count() == fx["count"]
    hh, hd = gh.to_host(), gd.to_host()
    for k in ("indptr", "indices", "row_indices", "blocks"):
        assert np.array_equal(hh[k], hd[k])


def test_policy_tile_width():
    src, dst, n = golden_graph("er_5000_32_s5")
    g = BitBSR(_dev(src), _dev(dst), n, 0)
    assert g.tile_cols == btc_b200.lite_select_tile_cols(len(src), n)


def test_duplicates_both_directions_and_selfloops():
    src, dst, n = golden_graph("stencil27_10")
    fx = load_golden()["stencil27_10"]
    s2 = np.concatenate([src, dst, src, np.arange(n, dtype=np.int32)])
    d2 = np.concatenate([dst, src, dst, np.arange(n, dtype=np.int32)])
    perm = np.random.default_rng(0).permutation(len(s2))
    g = BitBSR(_dev(s2[perm]), _dev(d2[perm]), n, 128)
    assert g.num_edges == fx["m_lower"]
    assert g.info().input_edges == len(s2)
    assert g.count() == fx["count"]
    assert {k: _digest(v) for k, v in g.to_host().items() if k in fx["digest_128"]} == fx["digest_128"]


@pytest.mark.parametrize("radix", [False, True], ids=["bitmap", "radix"])
@pytest.mark.parametrize("tile_cols", [32, 128])
def test_edge_cases(tile_cols, radix):
    B = lambda s, d, n, tc: BitBSR(s, d, n, tc, radix=radix)
    # empty graph
    g = B(_dev(np.zeros(0)), _dev(np.zeros(0)), 100, tile_cols)
    assert g.num_tiles == 0 and g.count() == 0
    h = g.to_host()
    assert np.all(h["indptr"] == 0) and len(h["indptr"]) == (100 + 15) // 16 + 1
    # only self-loops
    v = np.arange(50, dtype=np.int32)
    g = B(_dev(v), _dev(v), 50, tile_cols)
    assert g.num_tiles == 0 and g.count() == 0
    # zero vertices
    g = B(_dev(np.zeros(0)), _dev(np.zeros(0)), 0, tile_cols)
    assert g.count() == 0
    # one triangle at the last ids of a ragged n
    n = 1000
    g = B(_dev([999, 998, 999]), _dev([998, 997, 997]), n, tile_cols)
    assert g.count() == 1 and g.num_edges == 3
    # one full 16 x C tile (all-ones under the diagonal) and K_n closed forms
    for k in (16, 17, 31, 32, 33, 129, 200):
        s, d, _ = G.complete(k)
        assert B(_dev(s), _dev(d), k, tile_cols).count() == comb(k, 3)


def test_out_of_range_ids_are_rejected():
    with pytest.raises(BtcError) as e:
        BitBSR(_dev([0, 1, 5]), _dev([1, 2, 3]), 5, 128)
    assert e.value.status == _lib.BTC_E_RANGE
    with pytest.raises(BtcError):
        BitBSR(_dev([-1]), _dev([0]), 5, 128)
    with pytest.raises(BtcError) as e:
        BitBSR(_dev([0]), _dev([1]), 5, 64)
    assert e.value.status == _lib.BTC_E_INVAL


def test_rebuild_reuses_handle():
    a = load_golden()["stencil27_16"]
    b = load_golden()["rmat_12_16_s7"]
    s1, d1, n1 = golden_graph("stencil27_16")
    s2, d2, n2 = golden_graph("rmat_12_16_s7")
    g = BitBSR(_dev(s1), _dev(d1), n1, 128)
    assert g.count() == a["count"]
    g.rebuild(_dev(s2), _dev(d2), n2, 32)
    assert g.tile_cols == 32 and g.num_tiles == b["tiles_32"]
    assert g.count() == b["count"]
    g.rebuild(_dev(s1), _dev(d1), n1, 128)
    assert g.count() == a["count"]


def _arrays_match_oracle(g, name, C_):
    src, dst, n = golden_graph(name)
    rp, col, _ = O.lower_csr(src, dst, n)
    ref = O.bitbsr_build(rp, col, n, C_)
    h = g.to_host()
    for k in ("indptr", "indices", "row_indices", "blocks"):
        assert np.array_equal(np.asarray(h[k]), ref[k]), (name, C_, k)


def test_rebuild_sequences_enqueued_against_capacity():
    """Rebuilds run the whole build against the tile capacity of the previous build and
    wait once; a graph with more tiles than that capacity redoes the post-count steps.
    Every step of a sequence that grows, shrinks, switches tile width and hits a bad id
    must give the oracle's arrays and the golden count."""
    gold = load_golden()
    seq = [("stencil27_16", 128), ("stencil27_16", 128), ("K33", 128), ("rmat_12_16_s7", 128),
           ("rmat_15_16_s7_deg", 128), ("stencil27_4", 32), ("rmat_15_16_s7_deg", 32),
           ("sbm_600_8_dense", 128), ("rmat_15_16_s7_deg", 128), ("stencil7_16", 32),
           ("er_5000_32_s5", 128), ("K130", 32)]
    s0, d0, n0 = golden_graph(seq[0][0])
    g = BitBSR(_dev(s0), _dev(d0), n0, seq[0][1])
    for i, (name, C_) in enumerate(seq):
        s, d, n = golden_graph(name)
        if i:
            g.rebuild(_dev(s), _dev(d), n, C_)
        assert g.num_tiles == gold[name][f"tiles_{C_}"], (i, name, C_)
        _arrays_match_oracle(g, name, C_)
        assert g.count() == gold[name]["count"], (i, name, C_)
        if i == 4:  # a bad id after a good build, then the same graph again
            bad = np.asarray(s, np.int32).copy()
            bad[len(bad) // 2] = n + 3
            with pytest.raises(BtcError) as e:
                g.rebuild(_dev(bad), _dev(d), n, C_)
            assert e.value.status == _lib.BTC_E_RANGE
            g.rebuild(_dev(s), _dev(d), n, C_)
            assert g.count() == gold[name]["count"]
    g.free()


def test_async_rebuild_pipeline():
    """BTC_BUILD_ASYNC: rebuilds enqueued without a wait, counted on the device, give the
    golden counts; the tile count is right once a waiting call resolves the build."""
    gold = load_golden()
    s0, d0, n0 = golden_graph("rmat_15_16_s7_deg")  # large first build: room for the rest
    g = BitBSR(_dev(s0), _dev(d0), n0, 128)
    out = torch.zeros(1, dtype=torch.int64, device="cuda")
    for name in ["stencil27_16", "rmat_12_16_s7", "K130", "stencil7_16", "sbm_600_8_dense",
                 "er_5000_32_s5", "rmat_15_16_s7_deg"]:
        s, d, n = golden_graph(name)
        for deg, on_host in ((False, False), (True, True)):
            src = np.ascontiguousarray(s, np.int32) if on_host else _dev(s)
            dst = np.ascontiguousarray(d, np.int32) if on_host else _dev(d)
            g.rebuild(src, dst, n, 128, orient_degree=deg, asynchronous=True)
            g.count_async(d_out=out.data_ptr())
            assert int(out.item()) == gold[name]["count"], (name, deg)
            assert g.count() == gold[name]["count"], (name, deg)
            if not deg:
                assert g.num_tiles == gold[name]["tiles_128"]
                _arrays_match_oracle(g, name, 128)
    g.free()


def test_async_rebuild_graph_replay_follows_buffer_contents():
    """Identical asynchronous rebuilds (same buffers, sizes, flags) replay a captured
    CUDA graph from the second repeat on; the graph reads the buffers when it runs, so
    new contents in the same buffers give their own count."""
    gold = load_golden()
    s, d, n = golden_graph("rmat_12_16_s7")
    want = gold["rmat_12_16_s7"]["count"]
    ds, dd = _dev(s), _dev(d)
    g = BitBSR(ds, dd, n, 128)
    out = torch.zeros(1, dtype=torch.int64, device="cuda")
    rng = np.random.default_rng(11)
    for i in range(6):
        if i >= 3:  # same edges, new order and orientation, written into the same buffers
            perm = rng.permutation(len(s))
            flip = rng.random(len(s)) < 0.5
            ss, dd_ = np.asarray(s)[perm], np.asarray(d)[perm]
            ds.copy_(torch.from_numpy(np.where(flip, dd_, ss).astype(np.int32)))
            dd.copy_(torch.from_numpy(np.where(flip, ss, dd_).astype(np.int32)))
        g.rebuild(ds, dd, n, 128, asynchronous=True)
        g.count_async(d_out=out.data_ptr())
        assert int(out.item()) == want, i
    # a bad id in the replayed buffers surfaces at the next wait, then a fix replays again
    keep = int(ds[5].item())
    ds[5] = n + 1
    g.rebuild(ds, dd, n, 128, asynchronous=True)
    g.count_async(d_out=out.data_ptr())
    assert int(out.item()) == -1
    with pytest.raises(BtcError) as e:
        g.count()
    assert e.value.status == _lib.BTC_E_RANGE
    ds[5] = keep
    for _ in range(2):
        g.rebuild(ds, dd, n, 128, asynchronous=True)
        assert g.count() == want
    _arrays_match_oracle(g, "rmat_12_16_s7", 128)
    g.free()


def test_async_rebuild_failures_surface_at_next_wait():
    gold = load_golden()
    s, d, n = golden_graph("stencil27_16")
    g = BitBSR(_dev(s), _dev(d), n, 128)
    out = torch.zeros(1, dtype=torch.int64, device="cuda")
    # an out-of-range id: the enqueued count writes all ones, the next wait reports it
    bad = np.asarray(s, np.int32).copy()
    bad[7] = n
    g.rebuild(_dev(bad), _dev(d), n, 128, asynchronous=True)
    g.count_async(d_out=out.data_ptr())
    assert int(out.item()) == -1
    with pytest.raises(BtcError) as e:
        g.count()
    assert e.value.status == _lib.BTC_E_RANGE
    with pytest.raises(BtcError):
        g.count()  # the handle stays failed until a good rebuild
    g.rebuild(_dev(s), _dev(d), n, 128, asynchronous=True)
    assert g.count() == gold["stencil27_16"]["count"]
    # more tiles than the arrays hold: nothing built, BTC_E_CAPACITY, then a waiting
    # rebuild of the same graph succeeds
    s2, d2, n2 = golden_graph("rmat_15_16_s7_deg")
    g.rebuild(_dev(s2), _dev(d2), n2, 128, asynchronous=True)
    g.count_async(d_out=out.data_ptr())
    assert int(out.item()) == -1
    with pytest.raises(BtcError) as e:
        g.info()
    assert e.value.status == _lib.BTC_E_CAPACITY
    g.rebuild(_dev(s2), _dev(d2), n2, 128)
    assert g.count() == gold["rmat_15_16_s7_deg"]["count"]
    g.free()


def test_count_async_device_output():
    s, d, n = golden_graph("rmat_10_8_s11")
    fx = load_golden()["rmat_10_8_s11"]
    g = BitBSR(_dev(s), _dev(d), n, 128)
    out = torch.zeros(4, dtype=torch.int64, device="cuda")
    stream = torch.cuda.current_stream()
    for i in range(4):
        g.count_async(stream=stream, d_out=out.data_ptr() + 8 * i)
    torch.cuda.synchronize()
    assert out.tolist() == [fx["count"]] * 4


def test_density_hist_matches_oracle():
    s, d, n = golden_graph("rmat_12_16_s7_deg")
    rp, col, _ = O.lower_csr(s, d, n)
    for C in (32, 128):
        g = BitBSR(_dev(s), _dev(d), n, C)
        want = O.density_hist(O.bitbsr_build(rp, col, n, C))
        got = g.density_hist()
        assert np.array_equal(got.astype(np.int64), want)


# ---------------------------------------------------------------------------
# reference-shaped struct surface (include/btc_c.h "Reference-shaped surface")
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("tile_cols", [32, 128])
def test_reference_struct_api(tile_cols):
    name = "rmat_12_16_s7"
    fx = load_golden()[name]
    src, dst, n = golden_graph(name)
    r, c = G.lower_coo(src, dst, n)
    coo = btc_b200.CooMatrix(_dev(r), _dev(c), n)
    if tile_cols == 128:
        b = btc_b200.BCSR_16x128_Device()
        btc_b200.convert_coo_to_bcsr_16x128_gpu(b, coo)
        ms = []
        cnt = btc_b200.count_triangles_16x128_adaptive(b, 2048, ms)
    else:
        b = btc_b200.BCSR_16x32_Device()
        btc_b200.convert_coo_to_bcsr_16x32_gpu(b, coo)
        ms = []
        cnt = btc_b200.count_triangles_16x32_adaptive(b, 40000, ms)
    assert cnt == fx["count"] and len(ms) == 1 and ms[0] > 0
    assert b.get_result() == fx["count"]
    b.reset_result()
    assert b.get_result() == 0
    assert b.num_blocks == fx[f"tiles_{tile_cols}"]
    assert b.n == n and b.n_row_blocks == (n + 15) // 16
    h = b.to_host()
    assert {k: _digest(h[k]) for k in fx[f"digest_{tile_cols}"]} == fx[f"digest_{tile_cols}"]
    b.free()
    assert not b.indptr


@pytest.mark.parametrize("remap", [False, True])
def test_preprocess_matches_reference_semantics(remap):
    # ids spread out with gaps (isolated vertices) plus duplicates and self-loops
    rng = np.random.default_rng(5)
    n = 5000
    src = rng.integers(0, n, 20000).astype(np.int32) * 1
    dst = rng.integers(0, n, 20000).astype(np.int32)
    src[:10] = dst[:10]
    keep_ids = rng.permutation(n)[:3000]
    src = keep_ids[src % 3000].astype(np.int32)
    dst = keep_ids[dst % 3000].astype(np.int32)
    coo = btc_b200.CooMatrix(_dev(src), _dev(dst), n)
    btc_b200.preprocess_for_triangle_counting(coo, remap=remap)
    r, c = G.lower_coo(src, dst, n)
    if remap:
        used = np.unique(np.concatenate([r, c]))
        newid = np.full(n, -1, np.int64)
        newid[used] = np.arange(len(used))
        r, c = newid[r], newid[c]
        assert coo.num_rows == len(used)
    else:
        assert coo.num_rows == n
    assert np.array_equal(coo.row_indices.cpu().numpy(), r)
    assert np.array_equal(coo.column_indices.cpu().numpy(), c)
    # the preprocessed COO counts the same through the struct surface
    rp, col, _ = O.lower_csr(src, dst, n)
    want = O.tc_merge(rp, col)
    b = btc_b200.BCSR_16x32_Device()
    btc_b200.convert_coo_to_bcsr_16x32_gpu(b, coo)
    assert btc_b200.count_triangles_16x32_adaptive(b) == want


# ---------------------------------------------------------------------------
# full-size cases: size-independent properties
# ---------------------------------------------------------------------------
def test_config2_stencil_full_size():
    """27-point stencil on 64^3, 16x128 tiles: 11,049,696 triangles (closed form,
    also the reference CPU count)."""
    src, dst, n = G.stencil27(64)
    g = BitBSR(_dev(src), _dev(dst), n, 128)
    assert g.num_tiles == 56072 and g.num_edges == 3298428
    assert g.count() == 11049696
    assert g.count(tau=0) == 11049696


def test_host_input_full_size():
    """The 64^3 stencil from pageable and from pinned host memory: the arrays equal the
    device-input build's, asynchronous rebuilds from host memory keep the count, and an
    out-of-range id in the last edge is still reported."""
    src, dst, n = G.stencil27(64)
    ref = BitBSR(_dev(src), _dev(dst), n, 128)
    pinned = [torch.from_numpy(a).pin_memory().numpy() for a in (src, dst)]
    for hs, hd in ((src, dst), pinned):
        g = BitBSR(hs, hd, n, 128)
        h, r = g.to_host(), ref.to_host()
        for k in ("indptr", "indices", "row_indices", "blocks"):
            assert np.array_equal(h[k], r[k]), k
        for _ in range(3):
            g.rebuild(hs, hd, n, 128, asynchronous=True)
            assert g.count() == 11049696
        g.free()
    bad = src.copy()
    bad[-1] = n
    with pytest.raises(BtcError) as e:
        BitBSR(bad, dst, n, 128)
    assert e.value.status == _lib.BTC_E_RANGE


def test_rmat_scale18_orders_and_paths_agree():
    src, dst, n = G.rmat(18, 16, seed=7)
    rp, col, _ = O.lower_csr(src, dst, n)
    want = O.tc_merge(rp, col)
    counts = set()
    for C in (32, 128):
        for deg in (False, True):
            g = BitBSR(_dev(src), _dev(dst), n, C, orient_degree=deg, radix=deg and C == 32)
            counts.add(g.count())
            counts.add(g.count(tau=0))
            counts.add(g.count(tau=_lib.BTC_TAU_ALL_SPARSE))
            g.free()
    assert counts == {want}


@pytest.mark.parametrize("name", ["stencil27_16", "rmat_12_16_s7", "K130", "stencil7_8"])
def test_compat_cli_reads_matrix_market(name, tmp_path):
    """apps/btc_tc_lite.cu reads a Matrix Market coordinate file (graphs.write_mtx)."""
    import os
    import re
    import subprocess
    fx = load_golden()[name]
    src, dst, n = golden_graph(name)
    path = tmp_path / f"{name}.mtx"
    G.write_mtx(str(path), src, dst, n)
    app = os.path.join(os.path.dirname(_lib.LIB_PATH), "btc_tc_lite")
    out = subprocess.run([app, "-i", str(path), "-w", "1", "-r", "2"], capture_output=True,
                         text=True, timeout=120)
    assert out.returncode == 0, out.stdout + out.stderr
    got = int(re.search(r"Triangles \(GPU\): (\d+)", out.stdout).group(1))
    assert got == fx["count"], out.stdout


@pytest.mark.parametrize("name", ["stencil27_16", "rmat_12_16_s7", "K130"])
def test_compat_cli_reads_reference_bin_format(name, tmp_path):
    """apps/btc_tc_lite.cu: the reference's CLI flow over btc_compat.hpp, fed the
    reference's binary CSR file, prints the reference's result line."""
    import os
    import re
    import subprocess
    fx = load_golden()[name]
    src, dst, n = golden_graph(name)
    rp, col, _ = O.lower_csr(src, dst, n)
    path = tmp_path / f"{name}.bin"
    G.write_bin_csr(str(path), rp, col, n)
    app = os.path.join(os.path.dirname(_lib.LIB_PATH), "btc_tc_lite")
    for mode in ("0", "1", "2"):
        out = subprocess.run([app, "-i", str(path), "-w", "1", "-r", "3"], capture_output=True,
                             text=True, env={**os.environ, "BTC_MODE": mode}, timeout=120)
        assert out.returncode == 0, out.stdout + out.stderr
        got = int(re.search(r"Triangles \(GPU\): (\d+)", out.stdout).group(1))
        assert got == fx["count"], (mode, out.stdout)


def test_row_index_follows_the_graph_class():
    """The row index (and with it the row-wise count) exists for graphs averaging 8 or more
    tiles per row block.  An enqueued rebuild predicts that from the handle's previous
    graph of the same geometry; alternating a mesh (a few tiles per row block) and a
    random graph (dozens) on one handle, waiting and enqueued, must count exactly either
    way -- a wrong prediction only changes which kernel counts."""
    n = 4096
    mesh = G.stencil27(16)                     # 16^3 = 4096 vertices, a few tiles per row block
    rand = G.erdos_renyi(n, 32, seed=3)        # ~30 tiles per row block at 16x128
    assert mesh[2] == n and rand[2] == n
    want = {}
    for key, (s, d, _) in (("mesh", mesh), ("rand", rand)):
        rp, col, _ = O.lower_csr(s, d, n)
        want[key] = O.tc_merge(rp, col)
    # the random graph first: its tile arrays have room for every later enqueued rebuild
    g = BitBSR(_dev(rand[0]), _dev(rand[1]), n, 128)
    assert g.count() == want["rand"]
    out = torch.zeros(1, dtype=torch.int64, device="cuda")
    seq = ["mesh", "mesh", "rand", "rand", "mesh", "rand", "mesh", "rand", "rand"]
    for i, key in enumerate(seq):
        s, d, _ = rand if key == "rand" else mesh
        asynchronous = i % 3 != 2
        g.rebuild(_dev(s), _dev(d), n, 128, asynchronous=asynchronous)
        g.count_async(d_out=out.data_ptr())
        assert int(out.item()) == want[key], (i, key, asynchronous)
        assert g.count() == want[key], (i, key, asynchronous)
        for tau in (0, _lib.BTC_TAU_ALL_SPARSE):
            assert g.count(tau=tau) == want[key], (i, key, tau)
    g.free()
