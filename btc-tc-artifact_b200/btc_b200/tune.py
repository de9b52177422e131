"""Measurement side of the tile-width / tau policy.

``tau_sweep`` times the count kernel of one Bit-BSR at several dense/sparse switches
tau (a tile takes the binary tensor-core path when its popcount exceeds tau), the
experiment apps/tau_sweep.cu:410-566 runs for the reference, here checking every tau
against the first one.  ``python btc-tc-artifact_b200/btc_b200/tune.py`` runs the sweep
on the standard graphs and prints a markdown table (microseconds per launch).

``tune.py --count GRAPH --tile C [--reps K]`` builds one standard graph and counts it K
times (default tau), printing the counts: a fixed target for profilers.

``autotune(src, dst, n)`` measures the tile width for one graph (both widths built and
timed, counts cross-checked); ``tune.py --autotune`` prints it for the standard graphs
next to the reference's BTC-Lite choice.

``tune.py --sweep OUT.json`` measures the class sweep the engine's tile policy
(csrc/policy.cu) was set from: 37 graphs over five families (Erdos-Renyi, 27- and 7-point
stencils, R-MAT in natural and descending-degree order, 8-block SBMs, complete graphs),
both widths, three taus (default, all b1 MMA, all sparse), build and count with the L2
flushed before each; ``tune.py --table OUT.json`` prints the markdown table with the
measured best width, BTC-Lite's pick and the engine policy's pick.
"""
from __future__ import annotations

import json
import math
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


def autotune(src, dst, n: int, orient_degree: bool = False, tiles=(32, 128), reps: int = 5,
             stream=None) -> dict:
    """Measured tile-width choice for one graph (the reference's tile policy is the fixed
    BTC-Lite rule, apps/btc_tc_lite.cu:45-65).  Builds the Bit-BSR at every width in
    `tiles`, times rebuild and count (CUDA events, medians of `reps`), checks that all
    widths give the same count, and returns {"tile_cols": best by build + count,
    "count": c, "lite_policy": the BTC-Lite choice, "table": {C: {"build_ms", "count_ms",
    "tiles"}}}."""
    import torch

    from . import _lib
    from .api import BitBSR

    def ms_of(fn):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        st = torch.cuda.current_stream() if stream is None else stream
        e0.record(st)
        fn()
        e1.record(st)
        e1.synchronize()
        return e0.elapsed_time(e1)

    table, count = {}, None
    for C in tiles:
        g = BitBSR(src, dst, n, C, orient_degree=orient_degree, stream=stream)
        c = g.count(stream=stream)
        if count is None:
            count = c
        if c != count:
            raise AssertionError(f"16x{C} counted {c}, the first width {count}")
        builds = [ms_of(lambda: g.rebuild(src, dst, n, C, orient_degree=orient_degree,
                                          stream=stream)) for _ in range(reps)]
        counts = [g.count(stream=stream, timing=True)[1] for _ in range(reps)]
        table[C] = {"build_ms": statistics.median(builds), "count_ms": statistics.median(counts),
                    "tiles": g.num_tiles}
        g.free()
    m = int(src.numel()) if hasattr(src, "numel") else len(src)
    best = min(table, key=lambda C: table[C]["build_ms"] + table[C]["count_ms"])
    lite = int(_lib.lib().btc_lite_select_tile_cols(m, int(n), 0))
    return {"tile_cols": best, "count": count, "lite_policy": lite, "table": table}


def _mix_graph(index: int):
    from . import graphs as G
    s, d, _, nv, _ = G.batch_mix_device(4096, 256, 65536, seed=11, select=[index])
    return s, d, int(nv[0])


def standard_graphs(names=None):
    from . import graphs as G
    makers = {"stencil27_64": lambda: G.stencil27(64),
              "er_16384_16": lambda: G.erdos_renyi(16384, 16, seed=1),
              "rmat18_deg": lambda: G.rmat(18, 16, seed=7),
              "rmat20_deg": lambda: G.rmat(20, 16, seed=7),
              # the counter-based draws of the bench's R-MAT workloads (raw: the builder
              # dedups), generated on the GPU
              "rmat_raw18_deg": lambda: G.rmat_raw_torch(18, 16, 7),
              "rmat_raw20_deg": lambda: G.rmat_raw_torch(20, 16, 21),
              "rmat_raw22_deg": lambda: G.rmat_raw_torch(22, 16, 7),
              # the largest graph of the bench's 4096-graph batched mix (seed 11, graph 1742:
              # an 8-community SBM, n = 60,747, 68.3M raw pairs), generated on the GPU
              "sbm_mix1742": lambda: _mix_graph(1742)}
    names = names or ["stencil27_64", "er_16384_16", "rmat18_deg"]
    return [(k, makers[k](), k.endswith("_deg")) for k in names]


def count_once(name: str, tile: int, reps: int) -> None:
    import torch

    from .api import BitBSR
    [(_, (s, d, n), deg)] = standard_graphs([name])
    if not isinstance(s, torch.Tensor):
        s, d = torch.from_numpy(s).cuda(), torch.from_numpy(d).cuda()
    g = BitBSR(s, d, n, tile, orient_degree=deg)
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
    ap.add_argument("--autotune", action="store_true",
                    help="measured tile width per standard graph against the BTC-Lite rule")
    args = ap.parse_args()
    if args.count:
        count_once(args.count, args.tile, args.reps)
        return
    if args.autotune:
        print("| graph | BTC-Lite | measured best | 16x32 build+count ms | 16x128 build+count ms |")
        print("|---|---|---|---|---|")
        for name, (s_, d_, n_), deg in standard_graphs(["stencil27_64", "er_16384_16",
                                                        "rmat18_deg", "rmat20_deg"]):
            r = autotune(torch.from_numpy(s_).cuda(), torch.from_numpy(d_).cuda(), n_,
                         orient_degree=deg)
            t = r["table"]
            print(f"| {name} | 16x{r['lite_policy']} | 16x{r['tile_cols']} | "
                  f"{t[32]['build_ms']:.3f} + {t[32]['count_ms']:.3f} | "
                  f"{t[128]['build_ms']:.3f} + {t[128]['count_ms']:.3f} |", flush=True)
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


def sweep_specs():
    """(name, generator, degree_order) of the policy sweep."""
    from . import graphs as G
    specs = []
    for n in (4096, 16384, 65536, 262144):
        for d in (8, 16, 32):
            specs.append((f"er_{n}_{d}", lambda n=n, d=d: G.erdos_renyi(n, d, seed=5), False))
    for k in (16, 32, 64):
        specs.append((f"st27_{k}", lambda k=k: G.stencil27(k), False))
    for k in (32, 64):
        specs.append((f"st7_{k}", lambda k=k: G.stencil7(k), False))
    for sc in (12, 14, 16, 18, 20):
        for deg in (False, True):
            specs.append((f"rmat{sc}{'_deg' if deg else ''}", lambda sc=sc: G.rmat_raw_np(sc, 16, 7), deg))
    for n in (2048, 8192, 32768):
        for p in (0.05, 0.1, 0.3):
            specs.append((f"sbm_{n}_{p}", lambda n=n, p=p: G.sbm(n, 8, p, 0.001, seed=3), False))
    for n in (256, 1024):
        specs.append((f"K{n}", lambda n=n: G.complete(n), False))
    return specs


def sweep(reps: int = 5) -> list:
    """Both widths x three taus on every sweep graph (L2 flushed before each timing)."""
    import torch

    from .api import BitBSR
    flush = torch.empty(512 << 20, dtype=torch.uint8, device="cuda")

    def ev_ms(fn):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        flush.zero_()
        e0.record()
        fn()
        e1.record()
        e1.synchronize()
        return e0.elapsed_time(e1)

    out = []
    for name, gen, deg in sweep_specs():
        s_, d_, n = gen()
        src, dst = torch.from_numpy(s_).cuda(), torch.from_numpy(d_).cuda()
        row = dict(name=name, n=int(n), m_in=int(src.numel()), degree_order=deg)
        cnt = None
        for C in (32, 128):
            g = BitBSR(src, dst, n, C, orient_degree=deg)
            c = g.count()
            cnt = c if cnt is None else cnt
            if c != cnt:
                raise AssertionError(f"{name}: 16x{C} counted {c}, 16x32 {cnt}")
            b = statistics.median([ev_ms(lambda: g.rebuild(src, dst, n, C, orient_degree=deg))
                                   for _ in range(reps)])
            res = {}
            for tau in (-1, 0, 0x7FFFFFFF):
                ts = []
                for _ in range(reps):
                    flush.zero_()
                    cc, ms = g.count(tau=tau, timing=True)
                    if cc != cnt:
                        raise AssertionError(f"{name}: tau {tau} counted {cc}, expected {cnt}")
                    ts.append(ms)
                res[str(tau)] = statistics.median(ts)
            row[f"c{C}"] = dict(build_ms=b, count_ms=res, tiles=g.num_tiles, m_lower=g.num_edges)
            g.free()
        row["count"] = cnt
        out.append(row)
        print(json.dumps(row), file=sys.stderr, flush=True)
    return out


def policy_table(rows) -> str:
    """Markdown table of a sweep: measured best width, BTC-Lite's and the policy's picks."""
    import numpy as np

    from .api import lite_select_tile_cols, tile_policy
    lines = ["| graph | n | unique edges | 16x32 build + count ms | 16x128 build + count ms | "
             "best | BTC-Lite | policy |", "|---|---|---|---|---|---|---|---|"]
    slow = {"lite": [], "policy": []}
    gens = {nm: (gen, deg) for nm, gen, deg in sweep_specs()}
    for r in rows:
        t = {C: r[f"c{C}"]["build_ms"] + r[f"c{C}"]["count_ms"]["-1"] for C in (32, 128)}
        best = min(t, key=t.get)
        lite = lite_select_tile_cols(r["m_in"], r["n"])
        gen, deg = gens[r["name"]]
        s_, d_, n = gen()
        pol = tile_policy(np.asarray(s_), np.asarray(d_), n, orient_degree=deg)[0]
        slow["lite"].append(t[lite] / t[best])
        slow["policy"].append(t[pol] / t[best])
        fmt = lambda C: f"{r[f'c{C}']['build_ms']:.3f} + {r[f'c{C}']['count_ms']['-1']:.3f}"
        mark = lambda C: f"16x{C}" + ("" if C == best else f" (+{100 * (t[C] / t[best] - 1):.0f}%)")
        lines.append(f"| {r['name']} | {r['n']} | {r['c128']['m_lower']} | {fmt(32)} | {fmt(128)} | "
                     f"16x{best} | {mark(lite)} | {mark(pol)} |")
    gm = {k: math.exp(sum(math.log(x) for x in v) / len(v)) for k, v in slow.items()}
    lines.append("")
    lines.append(f"Slowdown against the measured best, geometric mean: BTC-Lite {gm['lite']:.3f}, "
                 f"policy {gm['policy']:.3f}; worst: BTC-Lite {max(slow['lite']):.2f}, policy "
                 f"{max(slow['policy']):.2f}; picks slower by more than 2%: BTC-Lite "
                 f"{sum(x > 1.02 for x in slow['lite'])}, policy {sum(x > 1.02 for x in slow['policy'])} "
                 f"of {len(rows)}.")
    return "\n".join(lines)


if __name__ == "__main__":
    import os
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    from btc_b200 import tune as _t
    if len(sys.argv) > 2 and sys.argv[1] == "--sweep":
        rows = _t.sweep()
        with open(sys.argv[2], "w") as f:
            json.dump({"graphs": rows}, f, indent=1)
        sys.exit(0)
    if len(sys.argv) > 2 and sys.argv[1] == "--table":
        with open(sys.argv[2]) as f:
            print(_t.policy_table(json.load(f)["graphs"]))
        sys.exit(0)
    _t.main()
