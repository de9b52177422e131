"""GPU A/B against the reference's own Bit-BSR build and count kernels, compiled from its
headers for sm_100a (oracle/_ref/libref_gpu.so): same tiles, byte for byte, and the
same count."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import golden_graph, load_golden

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

from btc_b200 import BitBSR, graphs as G  # noqa: E402
from oracle import oracle as O  # noqa: E402

NAMES = ["K130", "stencil27_16", "er_5000_32_s5", "rmat_12_16_s7", "rmat_15_16_s7_deg",
         "sbm_600_8_dense", "stencil7_16", "er_16384_16_s1"]


@pytest.mark.skipif(not O.ref_gpu_available(), reason="oracle/_ref/libref_gpu.so not built")
@pytest.mark.parametrize("tile_cols", [32, 128])
@pytest.mark.parametrize("name", NAMES)
def test_reference_gpu_tiles_and_count(name, tile_cols):
    fx = load_golden()[name]
    src, dst, n = golden_graph(name)
    r, c = G.lower_coo(src, dst, n)
    ref = O.ref_gpu_run(r, c, n, tile_cols, warmup=1, repeat=3, export=True)
    assert ref["count"] == fx["count"]
    g = BitBSR(torch.from_numpy(src).cuda(), torch.from_numpy(dst).cuda(), n, tile_cols)
    h = g.to_host()
    assert ref["num_blocks"] == h["num_blocks"]
    for k in ("indptr", "indices", "row_indices", "blocks"):
        assert np.array_equal(ref[k], h[k]), k
    assert g.count() == ref["count"]
