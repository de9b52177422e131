"""CPU tests of the seeded generators (inputs of every parity test and of the bench)."""
from __future__ import annotations

import numpy as np
import pytest

from btc_b200 import graphs as G


def _check_simple(src, dst, n):
    assert src.dtype == np.int32 and dst.dtype == np.int32
    assert np.all(src != dst)
    assert src.min() >= 0 and dst.min() >= 0 and max(src.max(), dst.max()) < n
    lo, hi = np.minimum(src, dst).astype(np.int64), np.maximum(src, dst).astype(np.int64)
    key = hi * n + lo
    assert len(np.unique(key)) == len(key)


@pytest.mark.parametrize("k,edges", [(2, 28), (4, 468), (64, 3_298_428)])
def test_stencil27_sizes(k, edges):
    src, dst, n = G.stencil27(k)
    assert n == k ** 3 and len(src) == edges
    _check_simple(src, dst, n)


def test_stencil7_size():
    src, dst, n = G.stencil7(8)
    assert len(src) == 3 * 8 * 8 * 7
    _check_simple(src, dst, n)


def test_er_is_seeded_and_simple():
    a = G.erdos_renyi(2000, 8, seed=3)
    b = G.erdos_renyi(2000, 8, seed=3)
    c = G.erdos_renyi(2000, 8, seed=4)
    assert np.array_equal(a[0], b[0]) and not np.array_equal(a[0], c[0])
    _check_simple(*a)


def test_rmat_degree_order_puts_hubs_first():
    src, dst, n = G.rmat(10, 8, seed=11, degree_order=True)
    _check_simple(src, dst, n)
    deg = np.bincount(src, minlength=n) + np.bincount(dst, minlength=n)
    assert np.all(np.diff(deg) <= 0)


def test_sbm_and_complete():
    _check_simple(*G.sbm(800, 8, 0.2, 0.01, seed=1))
    src, dst, n = G.complete(10)
    assert len(src) == 45


def test_lower_coo_and_bin_writer(tmp_path):
    src = np.array([1, 0, 2, 2, 3], np.int32)
    dst = np.array([0, 1, 1, 2, 0], np.int32)
    r, c = G.lower_coo(src, dst, 4)
    assert r.tolist() == [1, 2, 3] and c.tolist() == [0, 1, 0]
    rowptr = np.array([0, 0, 1, 2, 3], np.int32)
    p = tmp_path / "g.bin"
    G.write_bin_csr(str(p), rowptr, c, 4)
    raw = np.fromfile(p, np.int32)
    assert raw[:3].tolist() == [4, 4, 3]
    assert raw[3:8].tolist() == rowptr.tolist()
    assert raw[8:11].tolist() == c.tolist()


def test_write_mtx_is_lower_triangle_pattern(tmp_path):
    import numpy as np
    from btc_b200 import graphs as G
    s, d, n = G.stencil27(4)
    p = tmp_path / "g.mtx"
    G.write_mtx(str(p), s, d, n)
    lines = p.read_text().splitlines()
    assert lines[0] == "%%MatrixMarket matrix coordinate pattern symmetric"
    nr, nc, nnz = map(int, lines[1].split())
    assert nr == nc == n and nnz == len(lines) - 2
    e = np.array([list(map(int, ln.split())) for ln in lines[2:]])
    assert (e[:, 0] > e[:, 1]).all() and e.min() >= 1 and e.max() <= n
    r, c = G.lower_coo(s, d, n)
    assert nnz == len(r) and len({(a, b) for a, b in e}) == nnz


def test_batch_mix_plan_matches_batch_mix():
    """The plan behind the GPU-generated batch draws batch_mix's kinds, vertex counts and
    ER / R-MAT sizes from the same seeds."""
    host = G.batch_mix(48, 256, 65536, seed=3)
    plan = G.batch_mix_plan(48, 256, 65536, seed=3)
    for (s, d, n, kind), (pk, pn, segs) in zip(host, plan):
        assert (kind, n) == (pk, pn)
        if kind != "sbm":
            assert len(s) == sum(sg[-1] for sg in segs)
        else:
            assert all(0 <= a < b <= n and 0 <= c < e <= n for a, b, c, e, _ in segs)


def test_batch_mix_device_on_cpu_is_seeded_and_in_range():
    torch = pytest.importorskip("torch")
    a = G.batch_mix_device(24, 256, 4096, seed=5, device="cpu")
    b = G.batch_mix_device(24, 256, 4096, seed=5, device="cpu")
    src, dst, off, nv, kinds = a
    assert torch.equal(src, b[0]) and torch.equal(dst, b[1])
    assert off[0] == 0 and off[-1] == len(src) == len(dst) and len(nv) == len(kinds) == 24
    for i in range(24):
        s, d = src[off[i]:off[i + 1]], dst[off[i]:off[i + 1]]
        if len(s):
            assert int(s.min()) >= 0 and int(s.max()) < nv[i]
            assert int(d.min()) >= 0 and int(d.max()) < nv[i]


def test_batch_bench_groups_respect_the_launch_limit():
    """bench.py's batch workload cuts the graphs into consecutive launches of at most
    `limit` edges (a larger graph alone), covering every graph once, in order."""
    import importlib.util
    import os
    spec = importlib.util.spec_from_file_location(
        "bench_mod", os.path.join(os.path.dirname(os.path.dirname(__file__)), "bench.py"))
    bench = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(bench)
    rng = np.random.default_rng(4)
    sizes = rng.integers(0, 1000, 300)
    sizes[[7, 100]] = 5000  # larger than the limit
    off = np.zeros(len(sizes) + 1, np.int64)
    off[1:] = np.cumsum(sizes)
    groups = bench.batch_groups(off, 2000)
    assert groups[0][0] == 0 and groups[-1][1] == len(sizes)
    for (a, b), (c, _) in zip(groups, groups[1:]):
        assert b == c and b > a
    for a, b in groups:
        assert off[b] - off[a] <= 2000 or b == a + 1
