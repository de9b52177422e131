"""GPU test of btc_count_bcsr_noalloc, the count entry point that allocates nothing.

It serves callers that cannot let the library call cudaMalloc (a process whose own pool
already holds the device memory, or a loop that must not risk cudaMalloc's device
synchronisation); its scratch is a fixed array in the library's device image.  The test
calls it through the C ABI, twice in a row on one stream, and requires exactly the count
of the existing entry point (btc_count / the reference-shaped struct count): counts are
integers, so the tolerance is zero.  This file sorts last so a run that stops at the
first failure has run every other test first; it also passes alone in a fresh process.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from conftest import golden_graph, load_golden

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

import btc_b200  # noqa: E402
from btc_b200 import BitBSR, _lib  # noqa: E402

CASES = [("stencil27_16", 128, -1), ("rmat_12_16_s7", 32, -1), ("er_5000_32_s5", 128, -1),
         ("K130", 128, 0), ("sbm_600_8_dense", 32, 0)]


def _noalloc(bcsr, tile_cols, tau, stream, d_out):
    return _lib.lib().btc_count_bcsr_noalloc(C.byref(bcsr), tile_cols, tau, stream, d_out)


@pytest.mark.parametrize("name,tile_cols,tau", CASES)
def test_noalloc_matches_existing_count_twice(name, tile_cols, tau):
    torch.cuda.init()
    fx = load_golden()[name]
    src, dst, n = golden_graph(name)
    g = BitBSR(torch.from_numpy(src).cuda(), torch.from_numpy(dst).cuda(), n, tile_cols)
    want = g.count(tau=tau)  # the existing entry point
    assert want == fx["count"]
    view = g.info()
    stream = torch.cuda.current_stream()
    out = torch.full((3,), -1, dtype=torch.int64, device="cuda")
    # first call performs the per-device set-up (symbol address lookup)
    assert _noalloc(view.bcsr, tile_cols, tau, stream.cuda_stream, out.data_ptr()) == 0
    torch.cuda.synchronize()
    free_before = torch.cuda.mem_get_info()[0]
    for i in (1, 2):  # two calls in a row, no host synchronisation between them
        assert _noalloc(view.bcsr, tile_cols, tau, stream.cuda_stream, out.data_ptr() + 8 * i) == 0
    torch.cuda.synchronize()
    assert out.tolist() == [want, want, want]
    assert torch.cuda.mem_get_info()[0] >= free_before  # nothing was allocated
    g.free()


@pytest.mark.parametrize("tile_cols", [32, 128])
def test_noalloc_on_reference_struct(tile_cols):
    """The reference-shaped struct from btc_convert_* counts the same without allocating;
    with d_out NULL the count lands in bcsr->result, as in the reference."""
    name = "rmat_12_16_s7"
    fx = load_golden()[name]
    src, dst, n = golden_graph(name)
    coo = btc_b200.CooMatrix(torch.from_numpy(src).cuda(), torch.from_numpy(dst).cuda(), n)
    if tile_cols == 128:
        b = btc_b200.BCSR_16x128_Device()
        btc_b200.convert_coo_to_bcsr_16x128_gpu(b, coo)
        want = btc_b200.count_triangles_16x128_adaptive(b)
    else:
        b = btc_b200.BCSR_16x32_Device()
        btc_b200.convert_coo_to_bcsr_16x32_gpu(b, coo)
        want = btc_b200.count_triangles_16x32_adaptive(b)
    assert want == fx["count"]
    for _ in range(2):
        b.reset_result()
        assert _noalloc(b._s, tile_cols, -1, None, None) == 0
        torch.cuda.synchronize()
        assert b.get_result() == want
    b.free()


def test_noalloc_rejects_bad_arguments():
    s = _lib.BtcBcsrDevice()
    assert _noalloc(s, 64, -1, None, None) == _lib.BTC_E_INVAL       # tile width
    assert _noalloc(s, 128, -1, None, None) == _lib.BTC_E_INVAL      # no output word
    assert _lib.lib().btc_count_bcsr_noalloc(None, 128, -1, None, None) == _lib.BTC_E_INVAL
    out = torch.zeros(1, dtype=torch.int64, device="cuda")
    s.num_blocks = 5                                                   # tiles but no arrays
    assert _noalloc(s, 128, -1, None, out.data_ptr()) == _lib.BTC_E_INVAL
    assert _noalloc(s, 128, -7, None, out.data_ptr()) == _lib.BTC_E_INVAL  # tau
