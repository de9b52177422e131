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


@pytest.mark.parametrize("cfg", ["er_16384_16", "stencil27_64", "rmat22_deg"])
def test_policy_pick_is_the_measured_best(cfg):
    """On the single-graph configurations (Erdos-Renyi 16384 / 16, the 27-point stencil
    64^3, R-MAT scale 22 in descending-degree order) the engine's tile policy -- what
    tile_cols=0 applies -- picks the width that measures fastest (build + count, both
    widths built and counted, counts cross-checked)."""
    from btc_b200 import graphs as G, tile_policy, tune
    deg = cfg == "rmat22_deg"
    if cfg == "er_16384_16":
        s, d, n = G.erdos_renyi(16384, 16, seed=1)
    elif cfg == "stencil27_64":
        s, d, n = G.stencil27(64)
    else:
        s, d, n = G.rmat_raw_torch(22, 16, 7, device="cuda")
    if isinstance(s, np.ndarray):
        s, d = torch.from_numpy(s).cuda(), torch.from_numpy(d).cuda()
    pick = tile_policy(s, d, n, orient_degree=deg)[0]
    r = tune.autotune(s, d, n, orient_degree=deg, reps=3)
    t = {C: v["build_ms"] + v["count_ms"] for C, v in r["table"].items()}
    assert pick == r["tile_cols"], (cfg, pick, t)
