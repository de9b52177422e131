"""Measurement side of the tile-width / tau policy.

``tau_sweep`` times the count kernel of one Bit-BSR at several dense/sparse switches
tau (a tile takes the binary tensor-core path when its popcount exceeds tau), the
experiment apps/tau_sweep.cu:410-566 runs for the reference, here checking every tau
against the first one.  ``python btc-tc-artifact_b200/btc_b200/tune.py`` runs the sweep
on the standard graphs and prints a markdown table (microseconds per launch).

``tune.py --count GRAPH --tile C [--reps K]`` builds one standard graph and counts it K
times (default tau), printing the counts: a fixed target for profilers.
"""
from __future__ import annotations

import statistics
import sys

TAUS = [0, 8, 16, 32, 64, 128, 256, 512, 1024, 0x7FFFFFFF]


def tau_sweep(g, taus=TAUS, reps: int = 30) -> dict:
    """{tau: median kernel ms} for BitBSR g; raises if any tau changes the count."""
    out = {}
    ref = None
    for tau in taus:
        times = []
        for _ in range(reps):
            c, ms = g.count(tau=tau, timing=True)
            if ref is None:
                ref = c
            if c != ref:
                raise AssertionError(f"tau={tau} counted {c}, tau={taus[0]} counted {ref}")
            times.append(ms)
        out[tau] = statistics.median(times)
    return out


def standard_graphs(names=None):
    from . import graphs as G
    makers = {"stencil27_64": lambda: G.stencil27(64),
              "er_16384_16": lambda: G.erdos_renyi(16384, 16, seed=1),
              "rmat18_deg": lambda: G.rmat(18, 16, seed=7),
              "rmat20_deg": lambda: G.rmat(20, 16, seed=7)}
    names = names or ["stencil27_64", "er_16384_16", "rmat18_deg"]
    return [(k, makers[k](), k.endswith("_deg")) for k in names]


def count_once(name: str, tile: int, reps: int) -> None:
    import torch

    from .api import BitBSR
    [(_, (s, d, n), deg)] = standard_graphs([name])
    g = BitBSR(torch.from_numpy(s).cuda(), torch.from_numpy(d).cuda(), n, tile,
               orient_degree=deg)
    print(name, f"16x{tile}", g.num_tiles, [g.count() for _ in range(reps)], flush=True)
    g.free()


def main() -> None:
    import argparse

    import torch

    from .api import BitBSR
    ap = argparse.ArgumentParser()
    ap.add_argument("--count", default=None, help="count one standard graph instead of the sweep")
    ap.add_argument("--tile", type=int, default=128)
    ap.add_argument("--reps", type=int, default=3)
    args = ap.parse_args()
    if args.count:
        count_once(args.count, args.tile, args.reps)
        return
    print("| graph | tile | tiles | " + " | ".join(
        "all-sparse" if t == 0x7FFFFFFF else f"tau={t}" for t in TAUS) + " |")
    print("|---|---|---|" + "---|" * len(TAUS))
    for name, (s, d, n), deg in standard_graphs():
        for C in (128, 32):
            g = BitBSR(torch.from_numpy(s).cuda(), torch.from_numpy(d).cuda(), n, C,
                       orient_degree=deg)
            row = tau_sweep(g)
            print(f"| {name} | 16x{C} | {g.num_tiles} | " +
                  " | ".join(f"{1e3 * row[t]:.1f}" for t in TAUS) + " |", flush=True)
            g.free()


if __name__ == "__main__":
    import os
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    from btc_b200 import tune as _t
    _t.main()
