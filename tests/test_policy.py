"""The engine's tile policy (btc_tile_policy_from_features / btc_select_tile_policy) on
the CPU: its rules, the host-side locality sample, and -- against the committed sweep of
both tile widths on a B200 (profiles/autotune_sweep.json) -- that it beats the
reference's BTC-Lite rule (apps/btc_tc_lite.cu:45-65)."""
from __future__ import annotations

import json
import math
import os

import numpy as np
import pytest

from conftest import ROOT

from btc_b200 import graphs as G, lite_select_tile_cols, tile_policy, tile_policy_from_features


def test_rules():
    assert tile_policy_from_features(10 ** 6, 10 ** 5, orient_degree=True) == (128, 1024)
    assert tile_policy_from_features(10 ** 6, 10 ** 5, locality=1.0) == (32, 64)
    assert tile_policy_from_features(10 ** 6, 10 ** 5, locality=16.0) == (128, 1024)
    # average degree >= 512: 16x32 whatever the locality or the ordering
    assert tile_policy_from_features(300 * 1000, 1000, locality=100.0) == (32, 64)
    assert tile_policy_from_features(300 * 1000, 1000, orient_degree=True) == (32, 64)
    assert tile_policy_from_features(0, 0) == (32, 64)


@pytest.mark.parametrize("gen,want", [
    (lambda: G.erdos_renyi(16384, 16, seed=1), 32),   # random ids
    (lambda: G.stencil27(32), 128),                   # banded ids
    (lambda: G.stencil7(32), 128),
    (lambda: G.rmat(14, 16, seed=7), 32),             # natural-order R-MAT
    (lambda: G.complete(600), 32),                    # average degree >= 512
])
def test_host_sample(gen, want):
    s, d, n = gen()
    assert tile_policy(s, d, n)[0] == want
    assert tile_policy(s, d, n, orient_degree=True)[0] == (32 if 2 * len(s) >= 512 * n else 128)


def _sweep():
    with open(os.path.join(ROOT, "profiles", "autotune_sweep.json")) as f:
        return json.load(f)["graphs"]


def _regen(name):
    if name.startswith("er_"):
        _, n, d = name.split("_")
        return G.erdos_renyi(int(n), int(d), seed=5)
    if name.startswith("st27_"):
        return G.stencil27(int(name.split("_")[1]))
    if name.startswith("st7_"):
        return G.stencil7(int(name.split("_")[1]))
    if name.startswith("rmat"):
        return G.rmat_raw_np(int(name[4:6]), 16, 7)
    if name.startswith("sbm_"):
        _, n, p = name.split("_")
        return G.sbm(int(n), 8, float(p), 0.001, seed=3)
    return G.complete(int(name[1:]))


def test_policy_beats_btc_lite_on_the_sweep():
    """Slowdown of each rule's pick against the measured best width (build + count at the
    default tau): the engine's policy must do better than BTC-Lite in geometric mean and
    in the worst case."""
    slow = {"lite": [], "policy": []}
    for r in _sweep():
        if r["n"] > 300000:
            continue
        s, d, n = _regen(r["name"])
        t = {C: r[f"c{C}"]["build_ms"] + r[f"c{C}"]["count_ms"]["-1"] for C in (32, 128)}
        best = min(t.values())
        lite = lite_select_tile_cols(r["m_in"], r["n"])
        pol = tile_policy(np.asarray(s), np.asarray(d), n, orient_degree=r["degree_order"])[0]
        slow["lite"].append(t[lite] / best)
        slow["policy"].append(t[pol] / best)
    gm = {k: math.exp(np.mean(np.log(v))) for k, v in slow.items()}
    assert len(slow["policy"]) >= 30
    assert gm["policy"] < gm["lite"], gm
    assert max(slow["policy"]) < max(slow["lite"])
