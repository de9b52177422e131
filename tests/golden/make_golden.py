"""Regenerates tests/golden/golden.json and tests/golden/small_graphs.npz.

Each fixture is a seeded graph from btc_b200.graphs.  Its triangle count is
computed by the reference's own CPU path (btc/operations/triangle_count_cpu.h:59-101,
built into oracle/_ref/libref_cpu.so by oracle/ref/Makefile) and cross-checked
against the CPU oracle's merge count and its Bit-BSR count for both tile widths.
The tile counts and array digests come from the oracle's Bit-BSR builder (the
reference's builder is GPU-only; the GPU tests compare the two on the device).

Run from the repository root:  python tests/golden/make_golden.py
(``--large`` writes golden_large.json instead: the full-size graphs, counts only;
``--serve`` writes golden_serve.json: the served stream's request pool, counts only.)
"""
from __future__ import annotations

import hashlib
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "btc-tc-artifact_b200"))

from btc_b200 import graphs as G  # noqa: E402
from oracle import oracle as O  # noqa: E402

OUT_DIR = os.path.dirname(os.path.abspath(__file__))
SMALL_EDGES = 20000  # fixtures at most this large also store their edge arrays


def specs():
    """(name, generator, kwargs).  Sizes stay small enough for the oracle to finish in
    seconds; the full 64^3 stencil is the one large closed-form case."""
    return [
        ("K4", "complete", dict(n=4)),
        ("K5", "complete", dict(n=5)),
        ("K33", "complete", dict(n=33)),
        ("K130", "complete", dict(n=130)),
        ("stencil7_8", "stencil7", dict(k=8)),
        ("stencil7_16", "stencil7", dict(k=16)),
        ("stencil27_4", "stencil27", dict(k=4)),
        ("stencil27_10", "stencil27", dict(k=10)),
        ("stencil27_16", "stencil27", dict(k=16)),
        ("stencil27_64", "stencil27", dict(k=64)),
        ("er_1000_8_s3", "erdos_renyi", dict(n=1000, mean_degree=8, seed=3)),
        ("er_5000_32_s5", "erdos_renyi", dict(n=5000, mean_degree=32, seed=5)),
        ("er_16384_16_s1", "erdos_renyi", dict(n=16384, mean_degree=16, seed=1)),
        ("rmat_12_16_s7", "rmat", dict(scale=12, edge_factor=16, seed=7)),
        ("rmat_12_16_s7_deg", "rmat", dict(scale=12, edge_factor=16, seed=7, degree_order=True)),
        ("rmat_15_16_s7_deg", "rmat", dict(scale=15, edge_factor=16, seed=7, degree_order=True)),
        ("rmat_10_8_s11", "rmat", dict(scale=10, edge_factor=8, seed=11)),
        ("sbm_2000_8_s2", "sbm", dict(n=2000, blocks=8, p_in=0.1, p_out=0.001, seed=2)),
        ("sbm_600_8_dense", "sbm", dict(n=600, blocks=8, p_in=0.9, p_out=0.05, seed=4)),
    ]


def generate(gen: str, kw: dict):
    return getattr(G, gen)(**kw)


def digest(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()[:16]


def large_specs():
    """Full-size graphs (the R-MAT scale-22 headline graph and the served stream's large
    requests), counted by the reference's CPU path; only counts and sizes are stored."""
    return [
        ("rmat_raw_22_16_s7", "rmat_raw_np", dict(scale=22, edge_factor=16, seed=7)),
        ("rmat_raw_20_16_s21", "rmat_raw_np", dict(scale=20, edge_factor=16, seed=21)),
        ("rmat_raw_18_16_s7", "rmat_raw_np", dict(scale=18, edge_factor=16, seed=7)),
        ("stencil7_128", "stencil7", dict(k=128)),
    ]


def main_large():
    if not O.ref_cpu_available():
        O.build(ref=True)
    threads = os.cpu_count() or 1
    fixtures = {}
    for name, gen, kw in large_specs():
        src, dst, n = generate(gen, kw)
        rpd, cold, _ = O.lower_csr(src, dst, n, "degree")
        ref = int(O.ref_cpu_count(rpd, cold, threads))
        entry = dict(generator=gen, kwargs=kw, n=int(n), m_input=int(len(src)),
                     m_lower=int(len(cold)), count=ref,
                     edges_digest=digest(np.stack([src, dst]).astype(np.int32)))
        for C in (32, 128):
            entry[f"tiles_{C}_degree"] = int(O.bitbsr_num_tiles(rpd, cold, n, C))
        fixtures[name] = entry
        print(f"{name:22s} n={n:8d} m={len(cold):9d} count={ref}", flush=True)
    with open(os.path.join(OUT_DIR, "golden_large.json"), "w") as f:
        json.dump(dict(
            source="counts from the reference's cpu_tc_intersection_lower_triangular "
                   "(oracle/_ref/libref_cpu.so) on the descending-degree lower CSR; tile "
                   "counts from oracle/oracle.c",
            fixtures=fixtures), f, indent=1, sort_keys=True)


SERVE_POOL = dict(num_graphs=512, n_min=256, n_max=65536, seed=13)


def main_serve():
    """Per-graph counts of the served stream's request pool (graphs.batch_mix with
    SERVE_POOL), by the reference's CPU path; bench.py checks every served result
    against them."""
    if not O.ref_cpu_available():
        O.build(ref=True)
    threads = os.cpu_count() or 1
    pool = G.batch_mix(**SERVE_POOL)
    counts, digests = [], []
    for s_, d_, n, kind in pool:
        rp, col, _ = O.lower_csr(s_, d_, n)
        counts.append(int(O.ref_cpu_count(rp, col, threads)))
        digests.append(digest(np.stack([s_, d_]).astype(np.int32)))
    with open(os.path.join(OUT_DIR, "golden_serve.json"), "w") as f:
        json.dump(dict(source="counts from the reference's cpu_tc_intersection_lower_triangular "
                              "(oracle/_ref/libref_cpu.so) of graphs.batch_mix(**pool)",
                       pool=SERVE_POOL, counts=counts, edges_digests=digests), f)
    print(len(counts), "graphs,", sum(counts), "triangles")


def main():
    if "--large" in sys.argv[1:]:
        main_large()
        return
    if "--serve" in sys.argv[1:]:
        main_serve()
        return
    if not O.ref_cpu_available():
        O.build(ref=True)
    fixtures = {}
    small = {}
    for name, gen, kw in specs():
        src, dst, n = generate(gen, kw)
        rp, col, _ = O.lower_csr(src, dst, n)
        ref = O.ref_cpu_count(rp, col)
        merge = O.tc_merge(rp, col)
        rpd, cold, _ = O.lower_csr(src, dst, n, "degree")
        ref_deg = O.ref_cpu_count(rpd, cold)
        entry = dict(generator=gen, kwargs=kw, n=int(n), m_input=int(len(src)),
                     m_lower=int(len(col)), count=int(ref), edges_digest=digest(
                         np.stack([src, dst]).astype(np.int32)))
        assert merge == ref, (name, merge, ref)
        assert ref_deg == ref, (name, ref_deg, ref)
        for C in (32, 128):
            b = O.bitbsr_build(rp, col, n, C)
            c = O.bitbsr_count(b)
            assert c == ref, (name, C, c, ref)
            hist = O.density_hist(b)
            entry[f"tiles_{C}"] = int(b["num_blocks"])
            entry[f"digest_{C}"] = {k: digest(b[k]) for k in ("indptr", "indices", "row_indices", "blocks")}
            entry[f"max_tile_bits_{C}"] = int(np.nonzero(hist)[0].max()) if b["num_blocks"] else 0
            bd = O.bitbsr_build(rpd, cold, n, C)
            entry[f"tiles_{C}_degree"] = int(bd["num_blocks"])
        fixtures[name] = entry
        if len(src) <= SMALL_EDGES:
            small[f"{name}__src"] = src
            small[f"{name}__dst"] = dst
        print(f"{name:22s} n={n:7d} m={len(col):9d} count={ref}")
    with open(os.path.join(OUT_DIR, "golden.json"), "w") as f:
        json.dump(dict(
            source="counts from the reference's cpu_tc_intersection_lower_triangular "
                   "(oracle/_ref/libref_cpu.so); tiles/digests from oracle/oracle.c",
            fixtures=fixtures), f, indent=1, sort_keys=True)
    np.savez_compressed(os.path.join(OUT_DIR, "small_graphs.npz"), **small)


if __name__ == "__main__":
    main()
