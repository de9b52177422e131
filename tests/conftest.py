"""Shared test setup: the `gpu` marker, import paths and golden fixtures."""
from __future__ import annotations

import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "btc-tc-artifact_b200")
for p in (ROOT, PKG):
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN_DIR = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100a) GPU")
    config.addinivalue_line("markers", "slow: larger CPU cases")


def load_golden() -> dict:
    with open(os.path.join(GOLDEN_DIR, "golden.json")) as f:
        return json.load(f)["fixtures"]


_SMALL = None


def golden_graph(name: str):
    """(src, dst, n) of a golden fixture: stored arrays for small graphs, else the
    seeded generator (its output is checked against the stored digest)."""
    global _SMALL
    fx = load_golden()[name]
    if _SMALL is None:
        _SMALL = np.load(os.path.join(GOLDEN_DIR, "small_graphs.npz"))
    key = f"{name}__src"
    if key in _SMALL.files:
        return _SMALL[key], _SMALL[f"{name}__dst"], fx["n"]
    from btc_b200 import graphs as G
    return getattr(G, fx["generator"])(**fx["kwargs"])


@pytest.fixture(scope="session")
def golden():
    return load_golden()
