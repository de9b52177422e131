"""Host-side logic of the Python mirror that needs no GPU."""
from __future__ import annotations

import pytest

torch = pytest.importorskip("torch")

from btc_b200 import api  # noqa: E402


@pytest.mark.parametrize("env,want", [
    ({}, (16, 1)),
    ({"BTC_HASHORDER_HASHES": "8"}, (8, 1)),
    ({"BTC_HASHORDER_HOPS": "2"}, (16, 2)),
    ({"BTC_HASHORDER_HASHES": "4", "BTC_HASHORDER_HOPS": "0"}, (4, 0)),
    ({"BTC_HASHORDER_HASHES": "12abc"}, (12, 1)),   # atoi stops at the first non-digit
    ({"BTC_HASHORDER_HASHES": "x"}, (0, 1)),        # atoi of no digits is 0
])
def test_hashorder_env(monkeypatch, env, want):
    for k in ("BTC_HASHORDER_HASHES", "BTC_HASHORDER_HOPS"):
        monkeypatch.delenv(k, raising=False)
    for k, v in env.items():
        monkeypatch.setenv(k, v)
    assert api.hashorder_env() == want


def test_preprocess_forwards_hashorder_env(monkeypatch):
    """BTC_REORDER=8 runs HashOrder with the BTC_HASHORDER_* values (convert.h:668-674)."""
    seen = {}

    class FakeLib:
        @staticmethod
        def btc_preprocess_for_triangle_counting(rows, cols, nnz, num_rows, remap):
            return 0

    monkeypatch.setattr(api, "lib", lambda: FakeLib)
    monkeypatch.setattr(api, "reorder_hashorder_gpu",
                        lambda coo, num_hashes=16, num_hops=1: seen.update(h=num_hashes, k=num_hops))
    monkeypatch.setenv("BTC_HASHORDER_HASHES", "6")
    monkeypatch.setenv("BTC_HASHORDER_HOPS", "2")
    coo = object.__new__(api.CooMatrix)
    coo.row_indices = torch.tensor([1, 2, 2], dtype=torch.int32)
    coo.column_indices = torch.tensor([0, 0, 1], dtype=torch.int32)
    coo.num_rows = coo.num_cols = 3
    api.preprocess_for_triangle_counting(coo, reorder=8)
    assert seen == {"h": 6, "k": 2}
    seen.clear()
    api.preprocess_for_triangle_counting(coo, reorder=0)
    assert seen == {}
