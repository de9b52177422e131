"""Seeded synthetic graph generators for the engine's workloads.

Every generator returns ``(src, dst, n)``: two int32 arrays holding each
undirected edge once (no self-loops, no duplicates), in a seeded random
orientation and order, and the vertex count.  The engine's builder orients,
deduplicates and tiles them itself, so the order carries no information.

Workloads (sizes as used by bench.py):
  * ``erdos_renyi(16384, 16, seed=1)``      G(n, m = n*d/2 draws), ~131k edges
  * ``stencil27(64)``                      27-point 3-D stencil, 262,144 vertices,
                                           3,298,428 edges, 11,049,696 triangles
  * ``rmat(22, 16, seed=7)``               R-MAT (.57,.19,.19,.05), ~64M edges
  * ``rmat_raw_torch(22, 16, seed=7)``     the same shape, counter-based draws generated
                                           on the GPU (``rmat_raw_np``: the CPU twin)
  * ``sbm(n, 8, p_in, 0.001, seed)``       8-community stochastic block model
  * ``stencil7(k)``                        7-point stencil (bipartite: 0 triangles)
  * ``complete(n)``                        K_n (C(n,3) triangles)

The reference ships no inputs for these (its SuiteSparse files are absent), so
seeded synthetic graphs with the stated shapes stand in for them.
"""
from __future__ import annotations

import numpy as np


def _finish(lo, hi, n, rng):
    """Dedup undirected pairs (lo < hi), then shuffle order and orientation."""
    key = np.unique(hi.astype(np.int64) * np.int64(n) + lo.astype(np.int64))
    hi = (key // n).astype(np.int32)
    lo = (key % n).astype(np.int32)
    if rng is None:
        return hi, lo, n
    perm = rng.permutation(len(key))
    hi, lo = hi[perm], lo[perm]
    flip = rng.random(len(key)) < 0.5
    src = np.where(flip, lo, hi).astype(np.int32)
    dst = np.where(flip, hi, lo).astype(np.int32)
    return src, dst, n


def _pairs_to_edges(u, v, n, rng):
    u = np.asarray(u, np.int64)
    v = np.asarray(v, np.int64)
    keep = u != v
    u, v = u[keep], v[keep]
    return _finish(np.minimum(u, v), np.maximum(u, v), n, rng)


def erdos_renyi(n: int, mean_degree: float, seed: int = 1):
    """G(n, m) with m = round(n * mean_degree / 2) uniform draws; self-loops and
    duplicate pairs removed."""
    rng = np.random.default_rng(seed)
    m = int(round(n * mean_degree / 2))
    u = rng.integers(0, n, m, dtype=np.int64)
    v = rng.integers(0, n, m, dtype=np.int64)
    return _pairs_to_edges(u, v, n, rng)


def _stencil(k: int, offsets, seed):
    idx = np.arange(k ** 3, dtype=np.int64)
    x, y, z = idx // (k * k), (idx // k) % k, idx % k
    us, vs = [], []
    for dx, dy, dz in offsets:
        ok = ((x + dx >= 0) & (x + dx < k) & (y + dy >= 0) & (y + dy < k)
              & (z + dz >= 0) & (z + dz < k))
        u = idx[ok]
        us.append(u)
        vs.append(u + dx * k * k + dy * k + dz)
    u = np.concatenate(us)
    v = np.concatenate(vs)
    rng = np.random.default_rng(seed) if seed is not None else None
    return _finish(np.minimum(u, v), np.maximum(u, v), k ** 3, rng)


def stencil27(k: int, seed: int | None = 0):
    """27-point stencil on a k^3 grid, vertex id x*k*k + y*k + z (natural
    lexicographic order); every pair of distinct cells at Chebyshev distance 1."""
    offs = [(dx, dy, dz) for dx in (-1, 0, 1) for dy in (-1, 0, 1) for dz in (-1, 0, 1)
            if (dx, dy, dz) > (0, 0, 0)]
    return _stencil(k, offs, seed)


def stencil7(k: int, seed: int | None = 0):
    """7-point stencil on a k^3 grid (bipartite, so it has no triangles)."""
    return _stencil(k, [(1, 0, 0), (0, 1, 0), (0, 0, 1)], seed)


def complete(n: int, seed: int | None = 0):
    u, v = np.triu_indices(n, 1)
    rng = np.random.default_rng(seed) if seed is not None else None
    return _finish(u, v, n, rng)


def rmat(scale: int, edge_factor: int, a=0.57, b=0.19, c=0.19, seed: int = 7,
         degree_order: bool = False):
    """R-MAT: edge_factor * 2^scale draws of recursive quadrant choices with
    probabilities (a, b, c, 1-a-b-c); symmetrised, deduplicated, self-loops
    removed.  degree_order=True relabels vertices by descending degree (ties by
    id), so hubs get the lowest ids."""
    rng = np.random.default_rng(seed)
    n = 1 << scale
    m = edge_factor << scale
    u = np.zeros(m, np.int64)
    v = np.zeros(m, np.int64)
    chunk = 1 << 22
    ab, abc = a + b, a + b + c
    for s in range(0, m, chunk):
        e = min(m, s + chunk)
        uu = np.zeros(e - s, np.int64)
        vv = np.zeros(e - s, np.int64)
        for _ in range(scale):
            r = rng.random(e - s, dtype=np.float32)
            row = r >= ab
            colb = ((r >= a) & (r < ab)) | (r >= abc)
            uu = (uu << 1) | row
            vv = (vv << 1) | colb
        u[s:e] = uu
        v[s:e] = vv
    src, dst, n = _pairs_to_edges(u, v, n, rng)
    if degree_order:
        src, dst = relabel_by_degree(src, dst, n)
    return src, dst, n


# Counter-based R-MAT: the quadrant of draw i at level l comes from a 64-bit hash of
# (seed, i, l) (the splitmix64 finaliser), compared as an integer with thresholds
# round(p * 2^32).  The numpy and torch versions below give identical draws on any
# device, so a graph generated on the GPU in milliseconds has the count computed once on
# the CPU from the numpy version.
_SM_GAMMA = 0x9E3779B97F4A7C15
_SM_M1 = 0xBF58476D1CE4E5B9
_SM_M2 = 0x94D049BB133111EB
_M64 = (1 << 64) - 1


def _rmat_thresholds(a, b, c):
    return (int(round(a * 2 ** 32)), int(round((a + b) * 2 ** 32)),
            int(round((a + b + c) * 2 ** 32)))


def _rmat_key_base(seed: int) -> int:
    return (int(seed) * _SM_GAMMA) & _M64


def rmat_raw_np(scale: int, edge_factor: int, seed: int = 7, a=0.57, b=0.19, c=0.19):
    """Raw counter-based R-MAT draws (self-loops and duplicates kept; the engine's
    builder and the oracle's lower_csr remove them) as int32 numpy arrays, plus n.
    Draw i's bit at level l (first level = most significant): the top 32 bits x of
    splitmix64(seed * gamma + 64 * i + l) pick the quadrant -- row bit x >= (a+b),
    column bit a <= x < a+b or x >= a+b+c, thresholds scaled by 2^32."""
    ta, tab, tabc = _rmat_thresholds(a, b, c)
    n = 1 << scale
    m = edge_factor << scale
    base = np.uint64(_rmat_key_base(seed))
    src = np.empty(m, np.int32)
    dst = np.empty(m, np.int32)
    chunk = 1 << 22
    with np.errstate(over="ignore"):
        for s0 in range(0, m, chunk):
            e0 = min(m, s0 + chunk)
            key0 = np.arange(s0, e0, dtype=np.uint64) * np.uint64(64) + base
            u = np.zeros(e0 - s0, np.uint32)
            v = np.zeros(e0 - s0, np.uint32)
            for lev in range(scale):
                z = key0 + np.uint64(lev) + np.uint64(_SM_GAMMA)
                z = (z ^ (z >> np.uint64(30))) * np.uint64(_SM_M1)
                z = (z ^ (z >> np.uint64(27))) * np.uint64(_SM_M2)
                z = z ^ (z >> np.uint64(31))
                x = z >> np.uint64(32)
                row = x >= np.uint64(tab)
                col = ((x >= np.uint64(ta)) & (x < np.uint64(tab))) | (x >= np.uint64(tabc))
                u = (u << np.uint32(1)) | row.astype(np.uint32)
                v = (v << np.uint32(1)) | col.astype(np.uint32)
            src[s0:e0] = u.astype(np.int32)
            dst[s0:e0] = v.astype(np.int32)
    return src, dst, n


def _as_signed64(x: int) -> int:
    x &= _M64
    return x - (1 << 64) if x >> 63 else x


def rmat_raw_torch(scale: int, edge_factor: int, seed: int = 7, a=0.57, b=0.19, c=0.19,
                   device="cuda"):
    """rmat_raw_np's draws generated by torch on `device` (int64 arithmetic wraps
    modulo 2^64; right shifts are made logical by masking).  Returns int32 tensors
    (src, dst) and n."""
    import torch
    ta, tab, tabc = _rmat_thresholds(a, b, c)
    n = 1 << scale
    m = edge_factor << scale
    base = _as_signed64(_rmat_key_base(seed) + _SM_GAMMA)
    m1, m2 = _as_signed64(_SM_M1), _as_signed64(_SM_M2)

    def lsr(z, k):
        return (z >> k) & ((1 << (64 - k)) - 1)

    src = torch.empty(m, dtype=torch.int32, device=device)
    dst = torch.empty(m, dtype=torch.int32, device=device)
    chunk = 1 << 24
    for s0 in range(0, m, chunk):
        e0 = min(m, s0 + chunk)
        key0 = torch.arange(s0, e0, dtype=torch.int64, device=device) * 64 + base
        u = torch.zeros(e0 - s0, dtype=torch.int64, device=device)
        v = torch.zeros_like(u)
        for lev in range(scale):
            z = key0 + lev
            z = (z ^ lsr(z, 30)) * m1
            z = (z ^ lsr(z, 27)) * m2
            z = z ^ lsr(z, 31)
            x = lsr(z, 32)
            row = x >= tab
            col = ((x >= ta) & (x < tab)) | (x >= tabc)
            u = (u << 1) | row.to(torch.int64)
            v = (v << 1) | col.to(torch.int64)
        src[s0:e0] = u.to(torch.int32)
        dst[s0:e0] = v.to(torch.int32)
    return src, dst, n


def relabel_by_degree(src, dst, n):
    """Relabel so that rank 0 has the highest degree (ties by lower id)."""
    deg = np.bincount(src, minlength=n) + np.bincount(dst, minlength=n)
    order = np.lexsort((np.arange(n), -deg))
    rank = np.empty(n, np.int32)
    rank[order] = np.arange(n, dtype=np.int32)
    return rank[src], rank[dst]


def sbm(n: int, blocks: int, p_in: float, p_out: float, seed: int = 0):
    """Stochastic block model with `blocks` equal communities: each block pair
    draws Binomial(pairs, p) uniform vertex pairs (duplicates then removed)."""
    rng = np.random.default_rng(seed)
    bounds = np.linspace(0, n, blocks + 1).astype(np.int64)
    us, vs = [], []
    for i in range(blocks):
        for j in range(i, blocks):
            ni = bounds[i + 1] - bounds[i]
            nj = bounds[j + 1] - bounds[j]
            pairs = ni * (ni - 1) // 2 if i == j else ni * nj
            p = p_in if i == j else p_out
            k = rng.binomial(pairs, p) if pairs > 0 else 0
            if k == 0:
                continue
            us.append(rng.integers(bounds[i], bounds[i + 1], k))
            vs.append(rng.integers(bounds[j], bounds[j + 1], k))
    if not us:
        return np.zeros(0, np.int32), np.zeros(0, np.int32), n
    return _pairs_to_edges(np.concatenate(us), np.concatenate(vs), n, rng)


def lower_coo(src, dst, n):
    """Sorted unique lower-triangular COO (row > col) of an edge list, in numpy.
    Used to feed the reference-shaped entry points that expect a preprocessed COO."""
    src = np.asarray(src, np.int64)
    dst = np.asarray(dst, np.int64)
    keep = src != dst
    r = np.maximum(src[keep], dst[keep])
    c = np.minimum(src[keep], dst[keep])
    key = np.unique(r * np.int64(max(n, 1)) + c)
    return (key // max(n, 1)).astype(np.int32), (key % max(n, 1)).astype(np.int32)


def write_bin_csr(path: str, rowptr, col, n: int):
    """Write the reference's binary CSR file (btc/utils/io/read.h:255-299):
    int32 nrow, ncol, nnz; int32 row_ptr[nrow+1]; int32 col[nnz]; float val[nnz]."""
    rowptr = np.asarray(rowptr, np.int32)
    col = np.asarray(col, np.int32)
    with open(path, "wb") as f:
        np.array([n, n, len(col)], np.int32).tofile(f)
        rowptr.tofile(f)
        col.tofile(f)
        np.ones(len(col), np.float32).tofile(f)


def write_mtx(path: str, src, dst, n: int):
    """Write an edge list as a Matrix Market coordinate pattern file (the format the
    reference reads in btc/utils/io/read.h:33-189): each undirected edge once, in the lower
    triangle (row > col), 1-based, self-loops and duplicates removed."""
    r, c = lower_coo(src, dst, n)
    with open(path, "w") as f:
        f.write("%%MatrixMarket matrix coordinate pattern symmetric\n")
        f.write(f"{n} {n} {len(r)}\n")
        np.savetxt(f, np.stack([r + 1, c + 1], axis=1), fmt="%d")


def union_graph(graphs):
    """Block-diagonal union of graphs, laid out as a batch lays them out: graph g's
    vertex v becomes 16 * (row blocks of graphs before g) + v."""
    srcs, dsts = [], []
    base = 0
    for s, d, n in graphs:
        srcs.append(np.asarray(s, np.int64) + base)
        dsts.append(np.asarray(d, np.int64) + base)
        base += 16 * ((n + 15) // 16)
    src = np.concatenate(srcs).astype(np.int32) if srcs else np.zeros(0, np.int32)
    dst = np.concatenate(dsts).astype(np.int32) if dsts else np.zeros(0, np.int32)
    return src, dst, base


def batch_mix_plan(num_graphs: int, n_min: int = 256, n_max: int = 65536, seed: int = 0):
    """The parameters of batch_mix's graphs without their edges: per graph (kind, n,
    segments), a segment being (u_lo, u_hi, v_lo, v_hi, k) -- k pairs drawn uniformly from
    [u_lo, u_hi) x [v_lo, v_hi) -- or, for R-MAT, ("rmat", scale, m).  Kinds, vertex counts,
    degrees and R-MAT scales are batch_mix's (same seeds); the SBM block-pair edge counts
    come from the same binomials, drawn in a different order."""
    rng = np.random.default_rng(seed)
    plan = []
    for g in range(num_graphs):
        gr = np.random.default_rng((seed, g))
        kind = int(rng.integers(0, 3))
        n = int(round(np.exp(rng.uniform(np.log(n_min), np.log(n_max)))))
        if kind == 0:
            d = rng.uniform(8, 32)
            plan.append(("er", n, [(0, n, 0, n, int(round(n * d / 2)))]))
        elif kind == 1:
            p_in = rng.uniform(0.05, 0.3)
            bounds = np.linspace(0, n, 9).astype(np.int64)
            segs = []
            for i in range(8):
                for j in range(i, 8):
                    ni, nj = bounds[i + 1] - bounds[i], bounds[j + 1] - bounds[j]
                    pairs = ni * (ni - 1) // 2 if i == j else ni * nj
                    k = int(gr.binomial(pairs, p_in if i == j else 0.001)) if pairs > 0 else 0
                    if k:
                        segs.append((int(bounds[i]), int(bounds[i + 1]), int(bounds[j]),
                                     int(bounds[j + 1]), k))
            plan.append(("sbm", n, segs))
        else:
            scale = int(rng.integers(10, 17))
            plan.append(("rmat", 1 << scale, [("rmat", scale, 8 << scale)]))
    return plan


def batch_mix_device(num_graphs: int, n_min: int = 256, n_max: int = 65536, seed: int = 0,
                     device="cuda", select=None):
    """batch_mix generated on the GPU: the same kinds, sizes and distributions (plan from
    batch_mix_plan), the edges drawn by torch's seeded device generator (one per graph)
    straight into two int32 device arrays, so batches of billions of edges need no host
    memory.  select (optional): indices of the graphs to generate, in that order; graph g
    gets the same edges as in the whole mix.  Returns (src, dst, offsets int64[G+1],
    num_vertices int32[G], kinds) over the generated graphs."""
    import torch
    full = batch_mix_plan(num_graphs, n_min, n_max, seed)
    which = list(range(num_graphs)) if select is None else [int(i) for i in select]
    plan = [full[i] for i in which]
    sizes = [sum(sg[-1] for sg in segs) for _, _, segs in plan]
    offsets = np.zeros(len(plan) + 1, np.int64)
    offsets[1:] = np.cumsum(sizes)
    src = torch.empty(int(offsets[-1]), dtype=torch.int32, device=device)
    dst = torch.empty_like(src)
    for gi, (kind, n, segs) in enumerate(plan):
        g = which[gi]
        a = int(offsets[gi])
        gen = torch.Generator(device=device)
        gen.manual_seed(int(seed) * 1_000_003 + g)
        for sg in segs:
            if sg[0] == "rmat":
                _, scale, m = sg
                u = torch.zeros(m, dtype=torch.int32, device=device)
                v = torch.zeros_like(u)
                for _ in range(scale):
                    r = torch.rand(m, generator=gen, device=device)
                    u = (u << 1) | (r >= 0.76).to(torch.int32)
                    v = (v << 1) | (((r >= 0.57) & (r < 0.76)) | (r >= 0.95)).to(torch.int32)
                src[a:a + m] = u
                dst[a:a + m] = v
                a += m
                continue
            u_lo, u_hi, v_lo, v_hi, k = sg
            torch.randint(u_lo, u_hi, (k,), generator=gen, device=device, dtype=torch.int32,
                          out=src[a:a + k])
            torch.randint(v_lo, v_hi, (k,), generator=gen, device=device, dtype=torch.int32,
                          out=dst[a:a + k])
            a += k
    nv = np.array([n for _, n, _ in plan], np.int32)
    return src, dst, offsets, nv, [kind for kind, _, _ in plan]


def batch_mix(num_graphs: int, n_min: int = 256, n_max: int = 65536, seed: int = 0):
    """The mixed batch workload: vertex counts log-uniform in [n_min, n_max]; each graph
    (seeded per graph) is Erdos-Renyi with mean degree U[8, 32], an 8-community SBM with
    p_in U[0.05, 0.3] and p_out 0.001, or R-MAT with scale U{10..16} and edge factor 8,
    chosen uniformly.  Edges are raw draws: duplicates and self-loops are kept (the
    builder removes them) so that generation stays cheap.  R-MAT graphs take their
    vertex count from their scale.  Returns a list of (src, dst, n, kind)."""
    rng = np.random.default_rng(seed)
    out = []
    for g in range(num_graphs):
        gr = np.random.default_rng((seed, g))
        kind = int(rng.integers(0, 3))
        n = int(round(np.exp(rng.uniform(np.log(n_min), np.log(n_max)))))
        if kind == 0:
            d = rng.uniform(8, 32)
            m = int(round(n * d / 2))
            src = gr.integers(0, n, m, dtype=np.int32)
            dst = gr.integers(0, n, m, dtype=np.int32)
            out.append((src, dst, n, "er"))
        elif kind == 1:
            p_in = rng.uniform(0.05, 0.3)
            bounds = np.linspace(0, n, 9).astype(np.int64)
            us, vs = [], []
            for i in range(8):
                for j in range(i, 8):
                    ni, nj = bounds[i + 1] - bounds[i], bounds[j + 1] - bounds[j]
                    pairs = ni * (ni - 1) // 2 if i == j else ni * nj
                    k = gr.binomial(pairs, p_in if i == j else 0.001) if pairs > 0 else 0
                    if k:
                        us.append(gr.integers(bounds[i], bounds[i + 1], k, dtype=np.int64))
                        vs.append(gr.integers(bounds[j], bounds[j + 1], k, dtype=np.int64))
            src = np.concatenate(us).astype(np.int32) if us else np.zeros(0, np.int32)
            dst = np.concatenate(vs).astype(np.int32) if vs else np.zeros(0, np.int32)
            out.append((src, dst, n, "sbm"))
        else:
            scale = int(rng.integers(10, 17))
            n = 1 << scale
            m = 8 << scale
            u = np.zeros(m, np.int64)
            v = np.zeros(m, np.int64)
            for _ in range(scale):
                r = gr.random(m, dtype=np.float32)
                u = (u << 1) | (r >= 0.76)
                v = (v << 1) | (((r >= 0.57) & (r < 0.76)) | (r >= 0.95))
            out.append((u.astype(np.int32), v.astype(np.int32), n, "rmat"))
    return out
