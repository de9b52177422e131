"""GPU tests of the measurement helpers: the tile-width autotuner (both widths built,
counts cross-checked) and the binary tensor-core peak microbenchmark."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from conftest import golden_graph, load_golden

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


@pytest.mark.parametrize("name,deg", [("stencil27_16", False), ("rmat_12_16_s7", True),
                                      ("er_5000_32_s5", False)])
def test_autotune_measures_both_widths(name, deg):
    from btc_b200 import tune
    from btc_b200._lib import lib
    s, d, n = golden_graph(name)
    r = tune.autotune(torch.from_numpy(np.asarray(s, np.int32)).cuda(),
                      torch.from_numpy(np.asarray(d, np.int32)).cuda(), n,
                      orient_degree=deg, reps=3)
    assert r["count"] == load_golden()[name]["count"]
    assert r["tile_cols"] in (32, 128) and set(r["table"]) == {32, 128}
    assert r["lite_policy"] == lib().btc_lite_select_tile_cols(len(s), n, 0)
    for t in r["table"].values():
        assert t["count_ms"] > 0 and t["build_ms"] > 0 and t["tiles"] > 0


def test_b1_mma_peak_is_measured():
    from btc_b200._lib import lib
    ops = C.c_double(0.0)
    assert lib().btc_b1_mma_peak(None, 200, C.byref(ops)) == 0
    assert 1e13 < ops.value < 1e17  # binary ops per second: tens to thousands of Tops
    assert lib().btc_b1_mma_peak(None, 0, C.byref(ops)) != 0
