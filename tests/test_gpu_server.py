"""GPU tests of the continuous-batching server (btc_server_*): every request's count is
the reference CPU path's count of that graph (cpu_tc_intersection_lower_triangular,
btc/operations/triangle_count_cpu.h:59-101), the same alone (plain path, and the
single-graph BitBSR) and in the mix, whatever batch it lands in and however its arrival
overlaps others on the device.  Counts are integers, so the tolerance is zero."""
from __future__ import annotations

import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

import json  # noqa: E402
import os  # noqa: E402

from conftest import GOLDEN_DIR  # noqa: E402

from btc_b200 import BitBSR, Server, graphs as G, _lib  # noqa: E402
from oracle import oracle as O  # noqa: E402


def _pool():
    gs = [(s, d, n) for s, d, n, _ in G.batch_mix(40, 256, 4096, seed=5)]
    gs.append(G.stencil7(24))
    gs.append(G.stencil27(20))
    return gs


def _reference(gs):
    """The reference CPU path's count of each graph (the oracle restatement where the
    reference build is absent)."""
    fn = O.ref_cpu_count if O.ref_cpu_available() else O.tc_merge
    out = []
    for s, d, n in gs:
        rp, col, _ = O.lower_csr(s, d, n)
        out.append(int(fn(rp, col, os.cpu_count() or 1)))
    return out


def _alone(gs):
    want = _reference(gs)
    single = [BitBSR(torch.from_numpy(s).cuda(), torch.from_numpy(d).cuda(), n, 32).count()
              for s, d, n in gs]
    assert single == want
    return want


def _run(server, gs, order, gap_s=0.0, borrow=False):
    ids = {}
    for k in order:
        s, d, n = gs[k]
        ids[server.submit(s, d, n, borrow=borrow)] = k
        if gap_s:
            time.sleep(gap_s)
    got = {}
    deadline = time.time() + 120
    while len(got) < len(ids) and time.time() < deadline:
        for r in server.poll(wait_ms=100):
            assert r["status"] == 0
            assert r["done_s"] >= r["submit_s"]
            got[r["id"]] = r["count"]
    assert len(got) == len(ids)
    return [(ids[i], c) for i, c in got.items()]


@pytest.mark.parametrize("slots,max_graphs,borrow", [(2, 4096, False), (2, 7, True), (1, 1, False),
                                                     (3, 16, True)])
def test_counts_same_alone_and_in_the_mix(slots, max_graphs, borrow):
    gs = _pool()
    want = _alone(gs)
    rng = np.random.default_rng(slots * 100 + max_graphs)
    order = list(rng.permutation(len(gs))) * 3
    srv = Server(slots=slots, max_batch_graphs=max_graphs)
    try:
        for k, c in _run(srv, gs, order, gap_s=0.0005, borrow=borrow):
            assert c == want[k]
        st = srv.stats()
        assert st["graphs"] == len(order) and st["rejected"] == 0
        if max_graphs > 1:
            # a burst of submissions (no gaps) queues behind the running batches, so the
            # engine must put several requests in one batch
            for k, c in _run(srv, gs, order, gap_s=0.0, borrow=borrow):
                assert c == want[k]
            st2 = srv.stats()
            assert st2["graphs"] == 2 * len(order)
            assert st2["batches"] - st["batches"] < len(order)
    finally:
        srv.close()


def test_budget_rejects_a_request_too_large_alone():
    srv = Server(hbm_budget_bytes=1 << 20)  # 1 MiB: nothing but the smallest fits
    s, d, n = G.stencil27(32)
    rid = srv.submit(s, d, n)
    res = []
    while not res:
        res = srv.poll(wait_ms=200)
    assert res[0]["id"] == rid and res[0]["status"] == _lib.BTC_E_NOMEM
    assert srv.stats()["rejected"] == 1
    srv.close()


def test_close_drains_queue():
    gs = _pool()
    srv = Server()
    for s, d, n in gs:
        srv.submit(s, d, n)
    srv.close()  # returns after every queued request ran


def test_large_requests_in_the_mix():
    """The served workload's large requests (R-MAT scale 20 ef 16 and the 7-point stencil
    128^3) among small ones: each large count equals its golden count, each small one the
    reference CPU count, alone and in the mix."""
    with open(os.path.join(GOLDEN_DIR, "golden_large.json")) as f:
        fx = json.load(f)["fixtures"]
    r20 = G.rmat_raw_np(**fx["rmat_raw_20_16_s21"]["kwargs"])
    st7 = G.stencil7(128)
    small = _pool()[:20]
    gs = small + [r20, st7]
    want = _reference(small) + [fx["rmat_raw_20_16_s21"]["count"], 0]
    order = list(range(len(small))) + [len(small)] + list(range(len(small))) + [len(small) + 1] * 2
    for slots, max_graphs in ((2, 4096), (1, 1)):
        srv = Server(slots=slots, max_batch_graphs=max_graphs, tile_cols=32)
        try:
            for k, c in _run(srv, gs, order, gap_s=0.0002, borrow=True):
                assert c == want[k], k
        finally:
            srv.close()


def test_server_recovers_from_injected_allocation_failures(monkeypatch):
    """Reservations 2 and 9 report BTC_E_NOMEM.  Reservations are numbered as they are
    attempted (six per launched batch, none after a failure): request 0 fails at its
    second (#2), request 1 takes #3-#8, request 2 fails at its first (#9).  Those two
    complete with BTC_E_NOMEM and count 0; every other request, before and after, gets the
    reference CPU count."""
    gs = _pool()[:8]
    want = _reference(gs)
    monkeypatch.setenv("BTC_SERVER_FAIL_RESERVE", "2,9")
    srv = Server(slots=1, max_batch_graphs=1)
    monkeypatch.delenv("BTC_SERVER_FAIL_RESERVE")
    try:
        for k, (s, d, n) in enumerate(gs):  # one at a time: six reservations per request
            rid = srv.submit(s, d, n)
            res = []
            while not res:
                res = srv.poll(wait_ms=200)
            assert res[0]["id"] == rid
            if k in (0, 2):
                assert res[0]["status"] == _lib.BTC_E_NOMEM and res[0]["count"] == 0, res
            else:
                assert res[0]["status"] == 0 and res[0]["count"] == want[k], (k, res)
    finally:
        srv.close()


def test_sparse_graphs_on_large_vertex_ranges_in_the_mix():
    """A request's cell bitmap grows with its vertex range, not its edges: graphs of two
    million vertices and a few thousand edges, with the edge threshold for running alone
    raised so that only their vertex range sends them there, mixed with small graphs,
    still count exactly (a batch holding several of them would need more cell words than
    a batch may hold)."""
    rng = np.random.default_rng(17)
    gs = _pool()
    for k in range(4):
        n = 1 << 21
        hub = rng.integers(0, n, 64)
        s = np.concatenate([hub[rng.integers(0, 64, 3000)], rng.integers(0, n, 1000)]).astype(np.int32)
        d = np.concatenate([hub[rng.integers(0, 64, 3000)], rng.integers(0, n, 1000)]).astype(np.int32)
        gs.append((s, d, n))
    want = _reference(gs)
    order = list(rng.permutation(len(gs))) * 2
    srv = Server(slots=2, max_batch_graphs=4096, solo_edges=1 << 24)
    try:
        for k, c in _run(srv, gs, order):
            assert c == want[k], k
    finally:
        srv.close()
