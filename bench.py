"""Benchmark: exact triangle counting (Bit-BSR build + hybrid count) on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl engine|reference]
                    [--workload rmat22_deg|stencil27_64|er_16384|batch|serve|dense]
                    [--tile 0|32|128]

A step is one pass of the hot path over one graph: build the Bit-BSR from the raw
undirected edge list (orient, dedup, tile) and count its triangles.  The default
workload is the largest single-GPU graph: R-MAT scale 22, edge factor 16, seed 7
(67,108,864 raw draws generated on the GPU, ~64M unique edges), ordered by
descending degree on the GPU, 16x128 tiles; every count must equal the golden count
the reference's CPU path gave (tests/golden).  The metric is unique undirected edges
per second (whole job; N ranks each count a replica of the graph: weak scaling, no
data-path collective).

  value      device-resident edge list in HBM, L2 flushed (512 MB write) before
             every timed step, CUDA events around each step, max over ranks
  e2e        the same through the public API with host buffers: H2D of the pinned
             edge list, build, count, D2H of the count, every step; a stream of
             steps on two handles and two streams, so one step's copy overlaps the
             previous step's build and count (e2e.serial: one step at a time)
  roofline   the count kernel (dominant kernel of the step at this size) against
             the measured HBM copy bandwidth
  cpu_baseline   the reference's own cpu_tc_intersection_lower_triangular
             (oracle/_ref/libref_cpu.so, all host threads) on the same L
  --impl reference   times that same reference CPU path as the reference arm

A count that differs from the golden count, or a baseline whose count differs from
the engine's, ends the run with a non-zero exit status.

Only rank 0 prints, and only one JSON line, to stdout.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "btc-tc-artifact_b200"))

import numpy as np  # noqa: E402

METRIC = "exact_tc_edges_per_s"
UNIT = "edges/s"
L2_FLUSH_BYTES = 512 << 20


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d.get("hbm_gbs", 6650.0)), "measured (MEASURED_PEAKS.json hbm_gbs)"
    return 6650.0, "fallback 6.65 TB/s"


GOLDEN = os.path.join(ROOT, "tests", "golden")


def golden_count(fixture: str) -> int:
    """Triangle count of a fixture graph, computed by the reference's own CPU path when the
    fixture files were made (tests/golden/make_golden.py)."""
    for fn in ("golden.json", "golden_large.json"):
        p = os.path.join(GOLDEN, fn)
        if os.path.exists(p):
            with open(p) as f:
                fx = json.load(f)["fixtures"]
            if fixture in fx:
                return int(fx[fixture]["count"])
    raise SystemExit(f"no golden count for {fixture}")


def workload(name: str, device="cuda"):
    """(src, dst, n, meta): int32 torch tensors on `device` holding the raw input pairs."""
    import torch
    from btc_b200 import graphs as G
    if name == "rmat22_deg":
        src, dst, n = G.rmat_raw_torch(22, 16, seed=7, device=device)
        return src, dst, n, dict(
            workload="R-MAT scale 22 ef 16 (a,b,c)=(.57,.19,.19) seed 7, raw draws "
                     "(self-loops, duplicates) deduplicated and ordered by descending degree "
                     "on the GPU", tile_cols=128, expected=golden_count("rmat_raw_22_16_s7"),
            orient_degree=True)
    if name == "stencil27_64":
        s_, d_, n = G.stencil27(64)
        meta = dict(workload="27-point stencil 64^3, natural order", tile_cols=128,
                    expected=golden_count("stencil27_64"))
    elif name == "er_16384":
        s_, d_, n = G.erdos_renyi(16384, 16, seed=1)
        meta = dict(workload="Erdos-Renyi n=16384 mean degree 16 seed 1", tile_cols=0,
                    expected=golden_count("er_16384_16_s1"))
    else:
        raise SystemExit(f"unknown workload {name}")
    return (torch.from_numpy(s_).to(device), torch.from_numpy(d_).to(device), n, meta)


def count_profile(workload_name: str, tile: int):
    """ncu figures of one count launch on this workload (profiles/count_kernel.json): DRAM
    bytes (read + write) and warp instructions per launch, with how they were taken."""
    p = os.path.join(ROOT, "profiles", "count_kernel.json")
    if not os.path.exists(p):
        return None
    with open(p) as f:
        return json.load(f).get(f"{workload_name}/{tile}")


class ClockSampler:
    """nvidia-smi clocks/throttle samples during the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.device_index = device_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        cmd = ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
               "-lms", "50"]
        try:
            import torch
            uuid = str(torch.cuda.get_device_properties(self.device_index).uuid)
            cmd += ["-i", uuid if uuid.startswith("GPU-") else f"GPU-{uuid}"]
        except Exception:
            cmd += ["-i", str(self.device_index)]
        try:
            self.proc = subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.DEVNULL,
                                         text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception as e:  # no nvidia-smi
            log("clock sampler unavailable:", e)
            self.proc = None
        time.sleep(0.15)
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.1)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in self.lines:
            parts = [p.strip() for p in l.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[0]))
                mx.append(float(parts[1]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[4:8]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def launches_per_step(n: int, tile_cols: int, orient_degree: bool, m: int, tiles: int) -> int:
    """Kernels the engine launches per build + count (csrc/capi.cu build_into): the
    bitmap builder (mark, chunk count, scan, emit, last indptr, fill) when the cell
    bitmap is small enough, with the row index (five kernels) for graphs averaging 8 or
    more tiles per row block, else the radix builder; plus the degree relabel and count."""
    R = (n + 15) // 16
    ncb = (n + tile_cols - 1) // tile_cols
    bm_bytes = 4 * R * ((ncb + 31) // 32)
    if bm_bytes <= (4 << 30) and bm_bytes <= 32 * m + (64 << 20):
        k = 4  # mark, chunk count + scan, emit (+ zero tiles, last indptr), fill
        if m >= 8 * R and tiles >= 8 * R:
            k += 5  # row index: totals, scan (reduce, scan, apply), fill
    else:
        t_bits = max(R - 1, 0).bit_length() + max(ncb - 1, 0).bit_length()
        k = 1 + 3 * (-(-t_bits // 8)) + 2 + 1 + 1  # keys, sort, segment (2), fill, indptr
    if orient_degree:
        db = min(32, max(1, (2 * m).bit_length()))
        k += 1 + 1 + 1 + 3 * (-(-db // 8)) + 1  # degree, rank keys, set count, sort, scatter
    return k + 1 + 1  # row-occupancy masks, count


def cpu_reference(rowptr, col, m_lower, budget_s=10.0):
    from oracle import oracle as O
    threads = os.cpu_count() or 1
    O.ref_cpu_count(rowptr, col, threads)  # warm-up
    times = []
    t_end = time.perf_counter() + budget_s
    while True:
        t0 = time.perf_counter()
        cnt = O.ref_cpu_count(rowptr, col, threads)
        times.append(time.perf_counter() - t0)
        if time.perf_counter() > t_end or len(times) >= 50:
            break
    t = statistics.median(times)
    return cnt, t, threads, len(times)


def run_reference(args, rank, world):
    """Reference arm: the reference's own CPU count (cpu_tc_intersection_lower_triangular,
    oracle/_ref/libref_cpu.so, all host threads) on the same L as the engine's arm (same
    graph, same vertex order), rank 0 only.  A step is one count of the whole graph; when
    one count takes more than a second (R-MAT scale 22: several seconds on 16 cores) a
    single untimed warm-up count replaces the W warm-up steps, so that the run stays
    within a few minutes."""
    if rank != 0:
        return
    from oracle import oracle as O
    if not O.ref_cpu_available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libref_cpu.so not built"}))
        return
    src, dst, n, meta = workload(args.workload, device="cpu")
    odeg = bool(meta.get("orient_degree", False))
    rp, col, _ = O.lower_csr(src.numpy(), dst.numpy(), n, "degree" if odeg else "natural")
    m_lower = len(col)
    threads = os.cpu_count() or 1
    t0 = time.perf_counter()
    cnt = O.ref_cpu_count(rp, col, threads)
    first_s = time.perf_counter() - t0
    if cnt != meta["expected"]:
        raise SystemExit(f"reference CPU count {cnt} != golden {meta['expected']}")
    warm = args.warmup if first_s <= 1.0 else 0
    for _ in range(max(warm - 1, 0)):
        O.ref_cpu_count(rp, col, threads)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        cnt = O.ref_cpu_count(rp, col, threads)
        times.append(time.perf_counter() - t0)
        if cnt != meta["expected"]:
            raise SystemExit(f"reference CPU count {cnt} != golden {meta['expected']}")
    total = sum(times)
    value = m_lower * args.steps / total
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup if first_s <= 1.0 else 1,
        "ms_per_step": 1e3 * total / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int32",
        "data": "synthetic", "config": {"workload": meta["workload"], "edges": m_lower,
                                        "count": cnt, "parallelism": f"openmp{threads}",
                                        "orientation": "descending degree" if odeg else "natural id"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "reference",
                         "sample": f"full graph ({m_lower} edges), {args.steps} counts of the "
                                   f"lower CSR"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def dense_triples(h, tile_cols: int, tau: int) -> int:
    """(tile, slice, matched column block) triples of the tiles whose popcount exceeds tau:
    each is two m16n8k128 binary MMAs (16 x 16 x 128 AND-popcount-accumulates) on the
    count kernel's dense path."""
    jpt = tile_cols // 16
    wpr = tile_cols // 32
    indptr, indices, rows = h["indptr"], h["indices"], h["row_indices"]
    blocks = h["blocks"].reshape(-1, 16, wpr)
    R = len(indptr) - 1
    total = 0
    for t in range(len(indices)):
        tile = blocks[t]
        if int(np.unpackbits(tile.view(np.uint8)).sum()) <= tau:
            continue
        I, JL = int(rows[t]), int(indices[t])
        la = indices[indptr[I]:indptr[I + 1]]
        for j in range(jpt):
            J = JL * jpt + j
            if J >= R:
                break
            sl = (tile[:, (16 * j) // 32] >> np.uint32((16 * j) % 32)) & np.uint32(0xFFFF)
            if not sl.any():
                continue
            total += len(np.intersect1d(la, indices[indptr[J]:indptr[J + 1]],
                                        assume_unique=True))
    return total


def run_dense(args, rank, world):
    """Dense class: the complete graph K_n (every 16x128 tile full, so every tile takes the
    binary tensor-core path), counted at tau = 0.  Reports the binary MMA throughput of the
    count against this GPU's measured b1 MMA peak (btc_b1_mma_peak)."""
    import ctypes as C

    import torch
    from btc_b200 import BitBSR, graphs as G
    from btc_b200._lib import lib
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    n = args.n_dense
    s_, d_, _ = G.complete(n)
    g = BitBSR(torch.from_numpy(s_).cuda(), torch.from_numpy(d_).cuda(), n, 128)
    want = n * (n - 1) * (n - 2) // 6
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device="cuda")
    for _ in range(args.warmup):
        assert g.count(tau=0) == want
    ts = []
    with ClockSampler(int(os.environ.get("LOCAL_RANK", "0"))) as clk:
        for _ in range(args.steps):
            flush.zero_()
            c, ms = g.count(tau=0, timing=True)
            assert c == want
            ts.append(ms)
    t = statistics.median(ts) / 1e3
    triples = dense_triples(g.to_host(), 128, 0)
    ops = triples * 16 * 16 * 128
    peak = C.c_double(0.0)
    lib().btc_b1_mma_peak(None, 4000, C.byref(peak))
    m_lower = n * (n - 1) // 2
    line = {
        "metric": METRIC, "value": m_lower / t, "unit": UNIT, "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": t * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "b1",
        "data": "synthetic",
        "config": {"workload": f"complete graph K_{n} (dense class), count only, tau = 0",
                   "edges": m_lower, "tiles": g.num_tiles, "tile": "16x128",
                   "l2": "flushed before every timed count (512 MB write)"},
        "tensor": {"triples": triples, "ops_b1": ops, "achieved_tops": ops / t / 1e12,
                   "peak_tops": peak.value / 1e12, "frac": ops / t / peak.value,
                   "peak_source": "btc_b1_mma_peak (mma.sync m16n8k128 b1 and.popc, this GPU)"},
        "clocks": clk.summary(),
    }
    g.free()
    print(json.dumps(line), flush=True)


BATCH_GROUP_EDGES = 1 << 30   # edges per batch launch (one Bit-BSR holds < 2^32)
E2E_SAMPLE_EDGES = 1 << 28    # host edges of the batched e2e sample (2 GB pinned)


def batch_groups(off, limit):
    """Consecutive graph ranges [g0, g1) of at most `limit` edges each (a larger graph is
    a range of its own)."""
    groups, g0 = [], 0
    G = len(off) - 1
    while g0 < G:
        g1 = g0 + 1
        while g1 < G and off[g1 + 1] - off[g0] <= limit:
            g1 += 1
        groups.append((g0, g1))
        g0 = g1
    return groups


def run_batch(args, rank, world):
    """Batched workload: the mixed graphs generated on the GPU (several 10^9 edges at full
    size), counted in a few batch launches (one build + one count per group of at most
    2^30 edges, one batch handle per group; a step -- every group's rebuild, enqueued
    without a wait, and its count -- is one replayed CUDA graph), against the plain path
    (one build + one count + one host sync per graph, reusing one handle).  Adds a
    breakdown by graph kind (plain: per-graph device time summed by kind; batched: one
    batch run per kind) and the largest graphs' share of the plain time."""
    import torch
    from btc_b200 import Batch, BitBSR, graphs as G
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    t0 = time.perf_counter()
    d_src, d_dst, off, nv, kinds_list = G.batch_mix_device(args.graphs, 256, args.n_max,
                                                           seed=11 + rank)
    torch.cuda.synchronize()
    gen_s = time.perf_counter() - t0
    m_raw = int(off[-1])
    main = torch.cuda.current_stream()
    side = torch.cuda.Stream()
    streams = [main, side]
    tile = args.tile if args.tile is not None else 32
    groups = batch_groups(off, BATCH_GROUP_EDGES)

    def group_args(g0, g1, src=d_src, dst=d_dst, offs=off, nvs=nv):
        a, z = int(offs[g0]), int(offs[g1])
        return dict(src=src[a:z], dst=dst[a:z], offsets=offs[g0:g1 + 1] - a,
                    num_vertices=nvs[g0:g1], tile_cols=tile)

    # One batch handle per group (each keeps its group's arrays), all on one stream: a step
    # enqueues every group's rebuild without a wait (same graphs' sizes as the first build)
    # and its count, so the whole step is captured once as a CUDA graph and replayed.
    ghandles = [Batch(**group_args(g0, g1), stream=main) for g0, g1 in groups]
    counts = np.zeros(args.graphs, np.uint64)
    for h, (g0, g1) in zip(ghandles, groups):
        counts[g0:g1] = h.count(stream=main)
    d_counts = torch.zeros(args.graphs, dtype=torch.int64, device="cuda")

    def enqueue_step(st):
        for h, (g0, g1) in zip(ghandles, groups):
            h.rebuild(**group_args(g0, g1), stream=st, asynchronous=True)
            h.count_async(d_counts[g0:].data_ptr(), stream=st)

    cap_stream = torch.cuda.Stream()
    cap_stream.wait_stream(main)
    enqueue_step(cap_stream)  # one enqueued step before capture
    cap_stream.synchronize()
    step_graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(step_graph, stream=cap_stream):
        enqueue_step(cap_stream)

    def batched_step_graph():
        cap_stream.wait_stream(main)
        with torch.cuda.stream(cap_stream):
            step_graph.replay()
        main.wait_stream(cap_stream)

    for _ in range(args.warmup):
        batched_step_graph()
    torch.cuda.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(args.steps)]
    with ClockSampler(int(os.environ.get("LOCAL_RANK", "0"))) as clk:
        for e0, e1 in ev:
            e0.record(main)
            batched_step_graph()
            e1.record(main)
        torch.cuda.synchronize()
    t_batch = sum(e0.elapsed_time(e1) for e0, e1 in ev) / args.steps / 1e3
    if not np.array_equal(d_counts.cpu().numpy().astype(np.uint64), counts):
        raise SystemExit("batched counts of the timed steps differ from the first pass")
    for h in ghandles:
        h.count(stream=main)  # the enqueued builds' status (raises on a failure)
    # the same step enqueued call by call (no graph), for comparison
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(main)
    enqueue_step(main)
    e1.record(main)
    e1.synchronize()
    t_enqueued = e0.elapsed_time(e1) / 1e3
    for h in ghandles:
        h.count(stream=main)
        h.free()
    del step_graph

    # two handles alternating over varying groups (waiting rebuilds): the per-kind runs
    handles = [Batch(**group_args(*groups[0]), stream=main)]
    if len(groups) > 1:
        handles.append(Batch(**group_args(*groups[1]), stream=side))

    def batched_step(grps, ga, out):
        side.wait_stream(main)
        for gi, (g0, g1) in enumerate(grps):
            h, st = handles[gi % len(handles)], streams[gi % len(handles)]
            h.rebuild(**ga(g0, g1), stream=st)
            h.count_async(out[g0:].data_ptr(), stream=st)
        main.wait_stream(side)

    # plain: one launch sequence and one host sync per graph; device time per graph too
    g1_ = BitBSR(d_src[: max(int(off[1]), 1)], d_dst[: max(int(off[1]), 1)], int(nv[0]), tile)
    plain_counts = np.zeros(args.graphs, np.uint64)
    per_graph_ms = np.zeros(args.graphs)
    pev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
           for _ in range(args.graphs)]
    torch.cuda.synchronize()
    tp0 = time.perf_counter()
    for i in range(args.graphs):
        a, z = int(off[i]), int(off[i + 1])
        pev[i][0].record(main)
        g1_.rebuild(d_src[a:z], d_dst[a:z], int(nv[i]), tile, stream=main)
        plain_counts[i] = g1_.count(stream=main)
        pev[i][1].record(main)
    torch.cuda.synchronize()
    t_plain = time.perf_counter() - tp0
    for i, (e0, e1) in enumerate(pev):
        per_graph_ms[i] = e0.elapsed_time(e1)
    g1_.free()
    if not np.array_equal(plain_counts, counts):
        raise SystemExit("batched and plain counts differ")

    # breakdown by kind: plain device time by kind; each kind batched on its own
    kinds_arr = np.array(kinds_list)
    sizes = np.diff(off)
    breakdown = {}
    for k in ("er", "sbm", "rmat"):
        idx = np.flatnonzero(kinds_arr == k)
        if idx.size == 0:
            continue
        ks = torch.cat([d_src[int(off[i]):int(off[i + 1])] for i in idx])
        kd = torch.cat([d_dst[int(off[i]):int(off[i + 1])] for i in idx])
        koff = np.zeros(idx.size + 1, np.int64)
        koff[1:] = np.cumsum(sizes[idx])
        knv = nv[idx]
        kgroups = batch_groups(koff, BATCH_GROUP_EDGES)
        kcounts = torch.zeros(idx.size, dtype=torch.int64, device="cuda")
        kga = lambda g0, g1: group_args(g0, g1, ks, kd, koff, knv)
        batched_step(kgroups, kga, kcounts)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(main)
        batched_step(kgroups, kga, kcounts)
        e1.record(main)
        e1.synchronize()
        if not np.array_equal(kcounts.cpu().numpy().astype(np.uint64), counts[idx]):
            raise SystemExit(f"batched counts of the {k} graphs differ")
        kb = e0.elapsed_time(e1)
        kp = float(per_graph_ms[idx].sum())
        breakdown[k] = {"graphs": int(idx.size), "raw_edge_pairs": int(sizes[idx].sum()),
                        "plain_device_ms": kp, "batched_ms": kb, "speedup": kp / kb if kb else None}
        del ks, kd
    top = np.argsort(-sizes)[: max(1, args.graphs // 20)]
    breakdown["largest_5pct"] = {"graphs": int(top.size), "raw_edge_pairs": int(sizes[top].sum()),
                                 "plain_device_ms": float(per_graph_ms[top].sum()),
                                 "share_of_plain_device_time": float(per_graph_ms[top].sum() /
                                                                     per_graph_ms.sum())}
    breakdown["plain_device_ms_total"] = float(per_graph_ms.sum())
    breakdown["plain_wall_ms_total"] = t_plain * 1e3

    # e2e: the leading graphs whose edges fit E2E_SAMPLE_EDGES (all of them when the batch
    # is that small), their edges in pinned host memory, H2D inside the step
    n_e2e = max(1, int(np.searchsorted(off, E2E_SAMPLE_EDGES, side="right")) - 1)
    m_e2e = int(off[n_e2e])
    e_groups = batch_groups(off[:n_e2e + 1], BATCH_GROUP_EDGES)
    h_src = d_src[:m_e2e].cpu().pin_memory()
    h_dst = d_dst[:m_e2e].cpu().pin_memory()
    np_src, np_dst = h_src.numpy(), h_dst.numpy()
    host_counts = np.zeros(n_e2e, np.uint64)
    e2e = []
    b = handles[0]
    for _ in range(max(1, min(args.steps, 5))):
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(main)
        for g0, g1 in e_groups:
            a, z = int(off[g0]), int(off[g1])
            b.rebuild(src=np_src[a:z], dst=np_dst[a:z], offsets=off[g0:g1 + 1] - a,
                      num_vertices=nv[g0:g1], tile_cols=tile, stream=main)
            host_counts[g0:g1] = b.count(stream=main)
        e1.record(main)
        e1.synchronize()
        e2e.append(e0.elapsed_time(e1) / 1e3)
    if not np.array_equal(host_counts, counts[:n_e2e]):
        raise SystemExit("e2e batched counts differ")
    t_e2e = statistics.median(e2e)
    # the same over a stream of steps: consecutive steps alternate between the two
    # handles and streams, so one step's copies overlap the previous step's work (every
    # step still copies its edges in and its counts out)
    pipe_steps = 2 * max(1, min(args.steps, 5))
    pipe_out = torch.zeros((2, n_e2e), dtype=torch.int64, device="cuda")
    h_pipe = torch.zeros((pipe_steps, n_e2e), dtype=torch.int64).pin_memory()
    torch.cuda.synchronize()
    p0, p1, j2 = (torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True),
                  torch.cuda.Event())
    p0.record(main)
    side.wait_event(p0)
    for i in range(pipe_steps):
        k = i % len(handles)
        h, st = handles[k], streams[k]
        for g0, g1 in e_groups:
            a, z = int(off[g0]), int(off[g1])
            h.rebuild(src=np_src[a:z], dst=np_dst[a:z], offsets=off[g0:g1 + 1] - a,
                      num_vertices=nv[g0:g1], tile_cols=tile, stream=st)
            h.count_async(pipe_out[k, g0:].data_ptr(), stream=st)
        with torch.cuda.stream(st):
            h_pipe[i].copy_(pipe_out[k], non_blocking=True)
    j2.record(side)
    main.wait_event(j2)
    p1.record(main)
    p1.synchronize()
    for i in range(pipe_steps):
        if not np.array_equal(h_pipe[i].numpy().astype(np.uint64), counts[:n_e2e]):
            raise SystemExit("pipelined e2e batched counts differ")
    t_pipe = p0.elapsed_time(p1) / 1e3 / pipe_steps
    kinds = {k: kinds_list.count(k) for k in ("er", "sbm", "rmat")}
    line = {
        "metric": "batched_graphs_per_s", "value": world * args.graphs / t_batch,
        "unit": "graphs/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": t_batch * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "int32", "data": "synthetic (generated on the GPU)",
        "config": {"workload": f"batch of {args.graphs} mixed graphs (ER/SBM/R-MAT), n "
                               f"log-uniform [256, {args.n_max}]", "graphs": args.graphs,
                   "kinds": kinds, "raw_edge_pairs": m_raw, "raw_edge_bytes": 8 * m_raw,
                   "batch_launches": len(groups), "edges_per_launch_max": BATCH_GROUP_EDGES,
                   "step": "one CUDA graph: every group's enqueued rebuild and count",
                   "tile": f"16x{tile}",
                   "triangles_total": int(counts.sum()), "generation_s": round(gen_s, 1),
                   "parallelism": f"replica x{world}" if world > 1 else "single GPU"},
        "plain": {"value": world * args.graphs / t_plain, "unit": "graphs/s",
                  "what": "one rebuild + one count + one host sync per graph, one reused handle"},
        "speedup_vs_plain": t_plain / t_batch,
        "enqueued_without_graph_ms": t_enqueued * 1e3,
        "edges_per_s": world * m_raw / t_batch,
        "breakdown": breakdown,
        "e2e": {"value": world * n_e2e / t_pipe, "unit": "graphs/s",
                "h2d_bytes_per_step": 8 * m_e2e, "d2h_bytes_per_step": 8 * n_e2e + 24 * len(e_groups),
                "sample": f"the first {n_e2e} graphs ({m_e2e} edge pairs) from pinned host memory",
                "how": f"a stream of {pipe_steps} steps on {len(handles)} handles and streams "
                       "(one step's copies overlap the previous step's work)",
                "serial": {"value": world * n_e2e / t_e2e,
                           "how": "one step at a time: copies, builds, counts, counts back"}},
        "clocks": clk.summary(),
    }
    if rank == 0:
        print(json.dumps(line), flush=True)


def serve_once(Server, cfg, pool, large, lam, n_req, seed, want, large_frac=0.05):
    """Poisson arrivals at rate lam (a large_frac share of large requests, the rest from
    the pool) into one server, after a warm-up that grows every slot's buffers; returns
    throughput and latency percentiles on the server's clock."""
    rng = np.random.default_rng(seed)
    gaps = rng.exponential(1.0 / lam, n_req)
    picks = [("L", int(rng.integers(len(large)))) if rng.random() < large_frac
             else ("S", int(rng.integers(len(pool)))) for _ in range(n_req)]
    srv = Server(**cfg)
    # warm-up (not measured): every large request, then the pool twice, on every slot
    warm = 0
    for _ in range(max(1, cfg.get("slots", 2))):
        for s_, d_, n_ in (large if large_frac > 0 else []) + pool + pool:
            srv.submit(s_, d_, n_, borrow=True)
            warm += 1
    got = 0
    while got < warm:
        got += len(srv.poll(wait_ms=100))
    st0 = srv.stats()  # the measured stream's figures are differences from here
    ids = {}
    results = []
    done_flag = threading.Event()

    def collector():
        while not done_flag.is_set() or len(results) < n_req:
            results.extend(srv.poll(wait_ms=20))
            if len(results) >= n_req:
                break

    th = threading.Thread(target=collector, daemon=True)
    th.start()
    t_next = time.perf_counter()
    for gap, (kind, k) in zip(gaps, picks):
        t_next += gap
        dt = t_next - time.perf_counter()
        if dt > 0:
            time.sleep(dt)
        s_, d_, n_ = (large if kind == "L" else pool)[k]
        ids[srv.submit(s_, d_, n_, borrow=True)] = (kind, k)
    done_flag.set()
    th.join(timeout=600)
    st = srv.stats()
    srv.close()
    assert len(results) == n_req, (len(results), n_req)
    lat = np.array([r["done_s"] - r["submit_s"] for r in results])
    for r in results:
        assert r["status"] == 0 and r["count"] == want[ids[r["id"]]], r
    span = max(r["done_s"] for r in results) - min(r["submit_s"] for r in results)
    edges = sum(r["m"] for r in results)
    return {"lambda": lam, "requests": n_req, "graphs_per_s": n_req / span,
            "edges_per_s": edges / span, "p50_ms": float(np.percentile(lat, 50) * 1e3),
            "p99_ms": float(np.percentile(lat, 99) * 1e3),
            "batches": int(st["batches"] - st0["batches"]),
            "peak_device_gb": st["peak_device_bytes"] / 1e9,
            "solo_launches": int(st["solo_launches"] - st0["solo_launches"]),
            "solo_stream_ms": float(st["solo_stream_ms"] - st0["solo_stream_ms"]),
            "batch_stream_ms": float(st["batch_stream_ms"] - st0["batch_stream_ms"]),
            "large_requests": sum(1 for r in results if ids[r["id"]][0] == "L")}


def run_serve(args, rank, world):
    """Served stream: Poisson arrivals of mixed requests into the continuous-batching
    server, against the plain per-request server, over a sweep of arrival rates."""
    import torch
    from btc_b200 import BitBSR, Server, graphs as G
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    def pinned(g):  # requests arrive in pinned host buffers (the server DMAs them directly)
        s_, d_, n_ = g
        return (torch.from_numpy(np.ascontiguousarray(s_)).pin_memory().numpy(),
                torch.from_numpy(np.ascontiguousarray(d_)).pin_memory().numpy(), n_)

    pool_args = dict(num_graphs=args.pool, n_min=256, n_max=args.n_max, seed=13)
    pool = [pinned((s, d, n)) for s, d, n, _ in G.batch_mix(**pool_args)]
    large = [pinned(G.rmat_raw_np(20, 16, 21)), pinned(G.stencil7(128))]
    tile = args.tile if args.tile is not None else 32
    # every served count is checked against the reference CPU path's count of the graph:
    # the pool's from tests/golden/golden_serve.json (make_golden.py --serve), the large
    # R-MAT's from golden_large.json, the 7-point stencil's is 0 (bipartite)
    with open(os.path.join(GOLDEN, "golden_serve.json")) as f:
        gs = json.load(f)
    if gs["pool"] != pool_args:
        raise SystemExit(f"golden_serve.json holds the pool {gs['pool']}, not {pool_args}")
    want = {("S", k): int(c) for k, c in enumerate(gs["counts"])}
    want[("L", 0)] = golden_count("rmat_raw_20_16_s21")
    want[("L", 1)] = 0
    lams = [float(x) for x in args.rates.split(",")]
    modes = {"batched": dict(slots=2, max_batch_graphs=4096, tile_cols=tile,
                             hbm_budget_bytes=150 << 30),
             "plain": dict(slots=1, max_batch_graphs=1, tile_cols=tile, hbm_budget_bytes=150 << 30)}
    sweep = []
    for lam in lams:
        row = {"lambda": lam}
        for name, cfg in modes.items():
            row[name] = serve_once(Server, cfg, pool, large, lam, args.requests, 99, want,
                                   args.large_frac)
            log(name, json.dumps(row[name]))
        sweep.append(row)
    top = sweep[-1]
    line = {
        "metric": "served_graphs_per_s", "value": world * top["batched"]["graphs_per_s"],
        "unit": "graphs/s", "n_gpus": world, "steps": len(lams), "warmup": 0,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int32",
        "data": "synthetic",
        "config": {"workload": f"Poisson stream, {100 - 100 * args.large_frac:g}% mixed graphs "
                               f"(n log-uniform [256, {args.n_max}]), {100 * args.large_frac:g}% "
                               f"large (R-MAT scale 20 ef 16, 7-point stencil 128^3)",
                   "requests_per_rate": args.requests,
                   "rates": lams, "hbm_budget_gb": 150, "tile": f"16x{tile}"},
        "p50_ms": top["batched"]["p50_ms"], "p99_ms": top["batched"]["p99_ms"],
        "plain": top["plain"], "speedup_vs_plain": top["batched"]["graphs_per_s"] /
        top["plain"]["graphs_per_s"], "sweep": sweep,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=300)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="engine", choices=["engine", "reference"])
    ap.add_argument("--workload", default="rmat22_deg")
    ap.add_argument("--tile", type=int, default=None)
    ap.add_argument("--no-ref-gpu", action="store_true")
    ap.add_argument("--cpu-budget", type=float, default=8.0)
    ap.add_argument("--graphs", type=int, default=4096, help="batch workload: graphs")
    ap.add_argument("--n-max", type=int, default=65536, help="batch workload: largest n")
    ap.add_argument("--pool", type=int, default=512, help="serve workload: distinct small graphs")
    ap.add_argument("--requests", type=int, default=2000, help="serve workload: requests per rate")
    ap.add_argument("--rates", default="50,200,1000,5000", help="serve workload: arrivals/s")
    ap.add_argument("--large-frac", type=float, default=0.05, help="serve workload: large share")
    ap.add_argument("--n-dense", type=int, default=4096, help="dense workload: K_n vertices")
    ap.add_argument("--shard", action="store_true",
                    help="one graph per job: every rank counts a cost-balanced tile range of the "
                         "same Bit-BSR and the counts are all-reduced (strong scaling); default: "
                         "one graph per rank (weak scaling)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if args.workload == "batch":
        run_batch(args, rank, world)
        return
    if args.workload == "serve":
        run_serve(args, rank, world)
        return
    if args.workload == "dense":
        if rank == 0:
            run_dense(args, rank, world)
        return

    import torch
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    from btc_b200 import BitBSR
    d_src, d_dst, n, meta = workload(args.workload, device=f"cuda:{local}")
    tile = args.tile if args.tile is not None else meta["tile_cols"]
    odeg = bool(meta.get("orient_degree", False))
    m_in = int(d_src.numel())
    h_src = d_src.cpu().pin_memory()
    h_dst = d_dst.cpu().pin_memory()
    np_src, np_dst = h_src.numpy(), h_dst.numpy()
    stream = torch.cuda.current_stream()

    g = BitBSR(d_src, d_dst, n, tile, orient_degree=odeg, stream=stream)
    tile = g.tile_cols
    m_lower = g.num_edges
    expected = int(meta["expected"])
    first = g.count(stream=stream)
    if first != expected:
        raise SystemExit(f"count {first} != golden {expected} (reference CPU count)")
    info = g.info()
    B = int(info.bcsr.num_blocks)
    R = int(info.bcsr.n_row_blocks)
    tw_bytes = 2 * tile  # 16 rows x tile bits / 8
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device="cuda")
    d_out = torch.zeros(1, dtype=torch.int64, device="cuda")
    # --shard: every rank holds the whole Bit-BSR and counts its tile range; one int64
    # all-reduce (NCCL) adds the ranges.  The bounds depend only on the graph.
    bounds = g.partition(world, stream=stream) if args.shard else None
    jobs = 1 if args.shard else world  # graphs counted per step, all ranks together

    def count_step(out):
        if args.shard:
            g.count_tiles(bounds[rank], bounds[rank + 1], stream=stream, out=out)
            if dist:
                dist.all_reduce(out)
        else:
            g.count_async(stream=stream, d_out=out.data_ptr())

    # a step enqueues the build and the count without a host wait (BTC_BUILD_ASYNC;
    # the handle's arrays from the first build have room)
    def step_device():
        g.rebuild(d_src, d_dst, n, tile, orient_degree=odeg, stream=stream, asynchronous=True)
        count_step(d_out)

    for _ in range(args.warmup):
        flush.zero_()
        step_device()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()

    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(args.steps)]
    with ClockSampler(local) as clk:
        for e0, e1 in ev:
            flush.zero_()
            e0.record(stream)
            step_device()
            e1.record(stream)
        torch.cuda.synchronize()
    step_ms = [e0.elapsed_time(e1) for e0, e1 in ev]
    total_ms = sum(step_ms)
    if int(d_out.item()) != expected:
        raise SystemExit(f"count {int(d_out.item())} != golden {expected} in the timed loop")
    if dist:
        t = torch.tensor([total_ms], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
        dist.barrier()
    torch.cuda.synchronize()

    # ---- phase times (same L2 flush): count kernel alone, build alone ----------
    reps = min(args.steps, 100)
    t_count, t_build = [], []
    for _ in range(reps):
        flush.zero_()
        cnt, ms = g.count(stream=stream, timing=True)
        if cnt != expected:
            raise SystemExit(f"count {cnt} != golden {expected}")
        t_count.append(ms)
        flush.zero_()
        b0, b1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        b0.record(stream)
        g.rebuild(d_src, d_dst, n, tile, orient_degree=odeg, stream=stream)
        b1.record(stream)
        torch.cuda.synchronize()
        t_build.append(b0.elapsed_time(b1))
    warm = []
    for _ in range(min(reps, 20)):
        cnt, ms = g.count(stream=stream, timing=True)
        warm.append(ms)
    tc_warm = statistics.median(warm)
    tc = statistics.median(t_count) / 1e3
    tb = statistics.median(t_build) / 1e3

    # ---- e2e through the public API with host buffers -----------------------
    e2e_steps = min(args.steps, 100)
    for _ in range(3):
        g.rebuild(np_src, np_dst, n, tile, orient_degree=odeg, stream=stream)
        if g.count(stream=stream) != expected:
            raise SystemExit("e2e warm-up count differs from the golden count")
    torch.cuda.synchronize()
    # A step: the edge list copied from pinned host memory, the build, the count into a
    # device word and that word copied back into pinned host memory, all on `stream`; the
    # end event follows the copy back on the device, so the host's wake-up is not timed.
    h_out = torch.zeros(1, dtype=torch.int64).pin_memory()
    e2e_ms = []
    for _ in range(e2e_steps):
        flush.zero_()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        g.rebuild(np_src, np_dst, n, tile, orient_degree=odeg, stream=stream, asynchronous=True)
        count_step(d_out)
        with torch.cuda.stream(stream):
            h_out.copy_(d_out, non_blocking=True)
        e1.record(stream)
        e1.synchronize()
        cnt = int(h_out[0])
        if cnt != expected:
            raise SystemExit(f"e2e count {cnt} != golden {expected}")
        e2e_ms.append(e0.elapsed_time(e1))
    e2e_total = sum(e2e_ms)
    if dist:
        t = torch.tensor([e2e_total], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_total = float(t.item())

    # e2e over a stream of steps: consecutive steps alternate between two handles on two
    # streams, so step i+1's copy from pinned host memory overlaps step i's build and
    # count -- how a service counting a stream of graphs uses the API.  Every step still
    # copies its whole edge list in and its count out; the inputs (537 MB a step) are
    # larger than L2.  (Not with --shard, whose steps end in a collective.)
    pipe = None
    if not args.shard:
        pipe_steps = max(2, e2e_steps - e2e_steps % 2)
        s2 = torch.cuda.Stream()
        g2 = BitBSR(np_src, np_dst, n, tile, orient_degree=odeg, stream=s2)
        hs, sts = (g, g2), (stream, s2)
        d_outs = torch.zeros(2, dtype=torch.int64, device="cuda")
        h_outs = torch.zeros(pipe_steps, dtype=torch.int64).pin_memory()
        for k in (0, 1):  # warm-up: both handles' enqueued rebuilds
            hs[k].rebuild(np_src, np_dst, n, tile, orient_degree=odeg, stream=sts[k], asynchronous=True)
            if hs[k].count(stream=sts[k]) != expected:
                raise SystemExit("pipelined e2e warm-up count differs from the golden count")
        torch.cuda.synchronize()
        p0, p1, j2 = (torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True),
                      torch.cuda.Event())
        p0.record(stream)
        s2.wait_event(p0)
        for i in range(pipe_steps):
            k = i & 1
            hs[k].rebuild(np_src, np_dst, n, tile, orient_degree=odeg, stream=sts[k], asynchronous=True)
            hs[k].count_async(stream=sts[k], d_out=d_outs[k:k + 1].data_ptr())
            with torch.cuda.stream(sts[k]):
                h_outs[i:i + 1].copy_(d_outs[k:k + 1], non_blocking=True)
        j2.record(s2)
        stream.wait_event(j2)
        p1.record(stream)
        p1.synchronize()
        bad = [int(x) for x in h_outs.tolist() if int(x) != expected]
        if bad:
            raise SystemExit(f"pipelined e2e counts {bad[:3]} != golden {expected}")
        pipe_total = p0.elapsed_time(p1)
        if dist:
            t = torch.tensor([pipe_total], dtype=torch.float64, device="cuda")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            pipe_total = float(t.item())
        pipe = (pipe_steps, pipe_total)
        g2.free()
        del d_outs

    # ---- roofline of the count kernel ----------------------------------------
    hbm, peak_src = peaks()
    bytes_count = 4 * (R + 1) + 8 * B + tw_bytes * B + 8
    bytes_build = 8 * m_in + 4 * (R + 1) + 8 * B + tw_bytes * B
    achieved = bytes_count / tc / 1e9
    # DRAM bytes and warp instructions of one count launch on this workload, from the
    # committed ncu data (profiles/count_kernel.json; per launch, scaled from a smaller
    # capture of the same graph family when the full size is too large to capture).  Its
    # warp-instruction rate against the SMs' (4 schedulers per SM, one warp instruction
    # each per cycle, at the median SM clock sampled during the timed region) is the
    # issue side of the bound; dependent-load latency is the other.
    prof = count_profile(args.workload, tile)
    traffic = int(prof["dram_bytes_per_launch"]) if prof else None
    warp_inst = float(prof["warp_instructions_per_launch"]) if prof else None
    clocks = clk.summary()
    issue = None
    if warp_inst:
        sms = torch.cuda.get_device_properties(local).multi_processor_count
        mhz = clocks.get("sm_mhz") or clocks.get("sm_max_mhz")
        if mhz:
            peak_issue = sms * 4 * mhz * 1e6
            issue = {"warp_instructions": warp_inst, "achieved_per_s": warp_inst / tc,
                     "peak_per_s": peak_issue, "frac": warp_inst / tc / peak_issue,
                     "source": f"warp instructions per launch: {prof['source']}; peak = "
                               f"{sms} SMs x 4 schedulers x {mhz:g} MHz"}

    line = {
        "metric": METRIC,
        "value": jobs * m_lower * args.steps / (total_ms / 1e3),
        "unit": UNIT,
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": total_ms / args.steps,
        "higher_is_better": True,
        "scaling": "strong" if args.shard else "weak",
        "vs_baseline": None,
        "dtype": "int32",
        "data": "synthetic",
        "config": {"workload": meta["workload"], "vertices": n, "edges": m_lower,
                   "input_pairs": m_in, "tile": f"16x{tile}", "tiles": B, "triangles": expected,
                   "triangles_source": "golden count from the reference's CPU path",
                   "orientation": "descending degree" if odeg else "natural id",
                   "parallelism": (f"tile-sharded x{world}, int64 all-reduce" if args.shard
                                   else f"replica x{world}" if world > 1 else "single GPU"),
                   "l2": "flushed before every timed step (512 MB write)"},
        "e2e": ({"value": jobs * m_lower * pipe[0] / (pipe[1] / 1e3), "unit": UNIT,
                 "h2d_bytes_per_step": 8 * m_in, "d2h_bytes_per_step": 8 + 24, "steps": pipe[0],
                 "ms_per_step": pipe[1] / pipe[0],
                 "how": "stream of steps on two handles and two streams (step i+1's H2D "
                        "overlaps step i's build and count)",
                 "serial": {"value": jobs * m_lower * e2e_steps / (e2e_total / 1e3),
                            "ms_per_step": e2e_total / e2e_steps,
                            "how": "one step at a time: H2D, build, count, count back"}}
                if pipe else
                {"value": jobs * m_lower * e2e_steps / (e2e_total / 1e3), "unit": UNIT,
                 "h2d_bytes_per_step": 8 * m_in, "d2h_bytes_per_step": 8 + 24}),
        "gpu_launches": launches_per_step(n, tile, odeg, m_in, B) * args.steps,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                     "frac": achieved / hbm, "traffic": traffic,
                     "traffic_source": prof["source"] if prof else None,
                     # DRAM bytes the launch really moves (ncu) over its live duration:
                     # how close the kernel runs to the HBM bound its random sector
                     # traffic sets
                     "traffic_gbs": traffic / tc / 1e9 if traffic else None,
                     "traffic_frac": traffic / tc / 1e9 / hbm if traffic else None,
                     "kernel": prof["kernel"] if prof else f"k_count<{tile}>",
                     "algorithmic_bytes": bytes_count,
                     "kernel_ms": tc * 1e3, "peak_source": peak_src},
        "issue": issue,
        "phases": {"count_ms": tc * 1e3, "build_ms": tb * 1e3,
                   "build_gbs": bytes_build / tb / 1e9,
                   "count_edges_per_s": m_lower / tc},
        "clocks": clocks,
    }

    if rank == 0 and world == 1:
        # Baselines on the same L.  A baseline that is not built is skipped; a baseline
        # whose count differs from the engine's ends the run with an error.
        from oracle import oracle as O
        rp, col, _ = O.lower_csr(np_src, np_dst, n, "degree" if odeg else "natural")
        if O.ref_cpu_available():
            cnt, t, threads, reps_cpu = cpu_reference(rp, col, m_lower, args.cpu_budget)
            if cnt != expected:
                raise SystemExit(f"reference CPU count {cnt} != engine count {expected}")
            line["cpu_baseline"] = {"value": m_lower / t, "unit": UNIT, "cores": threads,
                                    "kind": "reference",
                                    "sample": f"full graph ({m_lower} edges), median of "
                                              f"{reps_cpu} counts"}
        else:
            log("cpu baseline unavailable: oracle/_ref/libref_cpu.so not built")
        if O.ref_gpu_available() and not args.no_ref_gpu:
            rr, cc = rp_to_coo(rp, col)
            big = B > 2_000_000
            ref = O.ref_gpu_run(rr, cc, n, tile, warmup=1 if big else 3, repeat=3 if big else 20)
            if ref["count"] != expected:
                raise SystemExit(f"reference GPU count {ref['count']} != engine count {expected}")
            kms = statistics.median(ref["kernel_ms"])
            line["reference_gpu"] = {
                "what": "reference convert + adaptive count compiled for sm_100a, same box",
                "convert_ms": ref["convert_ms"], "kernel_ms": kms,
                "engine_build_ms": tb * 1e3, "engine_count_ms_l2_flushed": tc * 1e3,
                "engine_count_ms_l2_warm": tc_warm,
                "count_speedup_same_l2_state": kms / tc_warm,
                "note": "reference kernel timed by its own events, L2 warm"}
        else:
            log("reference GPU leg unavailable or disabled")
    if rank == 0:
        print(json.dumps(line), flush=True)
    g.free()
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def rp_to_coo(rowptr, col):
    rows = np.repeat(np.arange(len(rowptr) - 1, dtype=np.int32), np.diff(rowptr))
    return rows, col


if __name__ == "__main__":
    main()
