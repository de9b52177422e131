"""ctypes front end of the CPU oracle and of the reference builds.

TEST INFRASTRUCTURE ONLY.  Imported by tests/, by ``__graft_entry__.smoke()`` and
by bench.py's CPU-baseline and reference legs, and nowhere else.  It is the
checker, never the thing measured as the engine.

* ``liboracle.so`` (oracle/oracle.c): CPU restatement of the reference path
  (convert.h:280-324, bcsr_16x{128,32}.h, tc_16x128_mma_v5.h / tc_16x32_mma_v6.h,
  triangle_count_cpu.h:59-101).
* ``_ref/libref_cpu.so``: the reference's own ``cpu_tc_intersection_lower_triangular``
  (btc/operations/triangle_count_cpu.h:59-101) compiled from its header.
* ``_ref/libref_gpu.so``: the reference's own Bit-BSR convert + adaptive count
  kernels and its GPU HashOrder (reorder.h:443-587), compiled for sm_100a (GPU only).
* ``libhashparams.so`` (oracle/hashparams.cpp): the HashOrder hash parameters, drawn
  with C++ <random> as reorder.h:495-506 draws them.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")

_i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_u32p = np.ctypeslib.ndpointer(dtype=np.uint32, flags="C_CONTIGUOUS")
_i64p = np.ctypeslib.ndpointer(dtype=np.int64, flags="C_CONTIGUOUS")
_f32p = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")

_lib = None
_ref_cpu = None
_ref_gpu = None


def build(ref: bool = True) -> None:
    """Compile liboracle.so and, when a reference checkout is present (oracle/ref/Makefile
    finds it, or BTC_REF_DIR names it), oracle/_ref."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    if ref:
        subprocess.run(["make", "-s", "-C", os.path.join(HERE, "ref")], check=True)


def lib():
    global _lib
    if _lib is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            build(ref=False)
        L = C.CDLL(path)
        L.orc_lower_csr.restype = C.c_int64
        L.orc_lower_csr.argtypes = [_i32p, _i32p, C.c_int64, C.c_int32, C.c_int, _i32p, _i32p, _i32p]
        L.orc_tc_merge.restype = C.c_uint64
        L.orc_tc_merge.argtypes = [_i32p, _i32p, C.c_int32, C.c_int]
        L.orc_bitbsr_num_tiles.restype = C.c_int64
        L.orc_bitbsr_num_tiles.argtypes = [_i32p, _i32p, C.c_int32, C.c_int]
        L.orc_bitbsr_build.restype = C.c_int64
        L.orc_bitbsr_build.argtypes = [_i32p, _i32p, C.c_int32, C.c_int, _u32p, _u32p, _u32p, _u32p]
        L.orc_bitbsr_density_hist.restype = None
        L.orc_bitbsr_density_hist.argtypes = [_u32p, C.c_int64, C.c_int, _i64p]
        L.orc_bitbsr_count.restype = C.c_uint64
        L.orc_bitbsr_count.argtypes = [_u32p, _u32p, _u32p, _u32p, C.c_int32, C.c_int64, C.c_int, C.c_int]
        L.orc_bitbsr_count_range.restype = C.c_uint64
        L.orc_bitbsr_count_range.argtypes = [_u32p, _u32p, _u32p, _u32p, C.c_int32, C.c_int64,
                                             C.c_int64, C.c_int, C.c_int]
        _lib = L
    return _lib


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def lower_csr(src, dst, n: int, order: str = "natural"):
    """Lower-triangular CSR (row > col, unique, sorted) of an edge list.

    order: "natural" keeps ids (convert.h:280-324); "degree" relabels by descending
    degree first (ties by id).  Returns (rowptr, col, rank)."""
    src, dst = _i32(src), _i32(dst)
    m = len(src)
    rowptr = np.zeros(n + 1, np.int32)
    col = np.zeros(max(m, 1), np.int32)
    rank = np.zeros(max(n, 1), np.int32)
    mode = {"natural": 0, "degree": 1}[order]
    mL = lib().orc_lower_csr(src, dst, m, n, mode, rowptr, col, rank)
    if mL < 0:
        raise ValueError("vertex id out of range")
    return rowptr, col[:mL].copy(), rank[:n].copy()


def tc_merge(rowptr, col, threads: int = 0) -> int:
    rowptr, col = _i32(rowptr), _i32(col)
    if len(col) == 0:
        col = np.zeros(1, np.int32)
    return int(lib().orc_tc_merge(rowptr, col, len(rowptr) - 1, threads))


def bitbsr_num_tiles(rowptr, col, n: int, tile_cols: int) -> int:
    """Number of tiles of the Bit-BSR of a lower CSR (no arrays built)."""
    rowptr, col = _i32(rowptr), _i32(col)
    if len(col) == 0:
        col = np.zeros(1, np.int32)
    return int(lib().orc_bitbsr_num_tiles(rowptr, col, n, tile_cols))


def bitbsr_build(rowptr, col, n: int, tile_cols: int):
    """Bit-BSR of a lower CSR as a dict of numpy arrays (reference layout)."""
    rowptr, col = _i32(rowptr), _i32(col)
    if len(col) == 0:
        col = np.zeros(1, np.int32)
    B = int(lib().orc_bitbsr_num_tiles(rowptr, col, n, tile_cols))
    R = (n + 15) // 16
    tw = 16 * (tile_cols // 32)
    indptr = np.zeros(R + 1, np.uint32)
    indices = np.zeros(max(B, 1), np.uint32)
    row_indices = np.zeros(max(B, 1), np.uint32)
    blocks = np.zeros(max(B, 1) * tw, np.uint32)
    B2 = int(lib().orc_bitbsr_build(rowptr, col, n, tile_cols, indptr, indices, row_indices, blocks))
    assert B2 == B
    return dict(n=n, tile_cols=tile_cols, n_row_blocks=R, num_blocks=B, indptr=indptr,
                indices=indices[:B], row_indices=row_indices[:B], blocks=blocks[:B * tw])


def bitbsr_count(bsr, threads: int = 0) -> int:
    B = bsr["num_blocks"]
    pad = lambda a: a if len(a) else np.zeros(1, np.uint32)
    return int(lib().orc_bitbsr_count(bsr["indptr"], pad(bsr["indices"]), pad(bsr["row_indices"]),
                                      pad(bsr["blocks"]), bsr["n"], B, bsr["tile_cols"], threads))


def bitbsr_count_range(bsr, t0: int, t1: int, threads: int = 0) -> int:
    """Count of the sample tiles [t0, t1) of an oracle Bit-BSR."""
    pad = lambda a: a if len(a) else np.zeros(1, np.uint32)
    return int(lib().orc_bitbsr_count_range(bsr["indptr"], pad(bsr["indices"]),
                                            pad(bsr["row_indices"]), pad(bsr["blocks"]), bsr["n"],
                                            int(t0), int(t1), bsr["tile_cols"], threads))


def density_hist(bsr):
    C_ = bsr["tile_cols"]
    hist = np.zeros(16 * C_ + 1, np.int64)
    blocks = bsr["blocks"] if len(bsr["blocks"]) else np.zeros(1, np.uint32)
    lib().orc_bitbsr_density_hist(blocks, bsr["num_blocks"], C_, hist)
    return hist


# ---------------------------------------------------------------------------
# HashOrder (btc/operations/reorder.h:411-587), restated in numpy
# ---------------------------------------------------------------------------
_HASH_P = 4294967291  # the largest prime below 2^32 (reorder.h:415)
_hashparams = None


def hashorder_params(num_hashes: int = 16):
    """(a, b) uint32 arrays drawn as reorder.h:495-506 draws them (oracle/hashparams.cpp)."""
    global _hashparams
    if _hashparams is None:
        path = os.path.join(HERE, "libhashparams.so")
        if not os.path.exists(path):
            build(ref=False)
        L = C.CDLL(path)
        L.oracle_hashorder_params.restype = None
        L.oracle_hashorder_params.argtypes = [C.c_int, _u32p, _u32p]
        _hashparams = L
    a = np.zeros(num_hashes, np.uint32)
    b = np.zeros(num_hashes, np.uint32)
    _hashparams.oracle_hashorder_params(int(num_hashes), a, b)
    return a, b


def hashorder(rows, cols, n: int, num_hashes: int = 16, num_hops: int = 1):
    """reorder_hashorder_gpu (reorder.h:443-587) on a COO of n vertices: per hash j,
    h_j(v) = (a_j v + b_j) mod P (411-418), num_hops rounds of
    h(v) <- min(h(v), min over the neighbours u of h(u)) over the symmetric edge set
    (421-441, 466-526), the vertices ordered lexicographically by (h_0, ..., h_{H-1}) with
    ties by id (the stable LSD passes of 536-549), perm[order[i]] = i (556-563), both
    endpoints relabelled and every entry oriented to (max, min) (569-584).
    Returns (rows, cols, perm) as numpy arrays."""
    rows = np.asarray(rows, np.int64)
    cols = np.asarray(cols, np.int64)
    a, b = hashorder_params(num_hashes)
    v = np.arange(n, dtype=np.uint64)
    h = (a.astype(np.uint64)[:, None] * v[None, :] + b.astype(np.uint64)[:, None]) % np.uint64(_HASH_P)
    for _ in range(num_hops):
        nxt = h.copy()
        for j in range(num_hashes):
            np.minimum.at(nxt[j], rows, h[j][cols])
            np.minimum.at(nxt[j], cols, h[j][rows])
        h = nxt
    order = np.lexsort((np.arange(n),) + tuple(h[j] for j in range(num_hashes - 1, -1, -1)))
    perm = np.empty(n, np.int64)
    perm[order] = np.arange(n)
    r, c = perm[rows], perm[cols]
    return (np.maximum(r, c).astype(np.int32), np.minimum(r, c).astype(np.int32),
            perm.astype(np.int32))


# ---------------------------------------------------------------------------
# reference builds (oracle/_ref)
# ---------------------------------------------------------------------------

def ref_cpu_available() -> bool:
    return os.path.exists(os.path.join(REF_DIR, "libref_cpu.so"))


def ref_cpu():
    global _ref_cpu
    if _ref_cpu is None:
        L = C.CDLL(os.path.join(REF_DIR, "libref_cpu.so"))
        L.ref_cpu_tc_lower.restype = C.c_uint64
        L.ref_cpu_tc_lower.argtypes = [_i32p, _i32p, C.c_int, C.c_int]
        L.ref_cpu_max_threads.restype = C.c_int
        _ref_cpu = L
    return _ref_cpu


def ref_cpu_count(rowptr, col, threads: int = 0) -> int:
    """The reference's own cpu_tc_intersection_lower_triangular."""
    rowptr, col = _i32(rowptr), _i32(col)
    if len(col) == 0:
        col = np.zeros(1, np.int32)
    return int(ref_cpu().ref_cpu_tc_lower(rowptr, col, len(rowptr) - 1, threads))


def ref_gpu_available() -> bool:
    return os.path.exists(os.path.join(REF_DIR, "libref_gpu.so"))


def ref_gpu():
    global _ref_gpu
    if _ref_gpu is None:
        L = C.CDLL(os.path.join(REF_DIR, "libref_gpu.so"))
        L.ref_gpu_run.restype = C.c_int
        L.ref_gpu_run.argtypes = [_i32p, _i32p, C.c_int64, C.c_int, C.c_int, C.c_int, C.c_int,
                                  C.POINTER(C.c_ulonglong), C.POINTER(C.c_float), _f32p,
                                  C.POINTER(C.c_uint32), C.c_void_p, C.c_void_p, C.c_void_p,
                                  C.c_void_p, C.c_int64]
        L.ref_hashorder_gpu.restype = C.c_int
        L.ref_hashorder_gpu.argtypes = [_i32p, _i32p, C.c_int64, C.c_int, C.c_int, C.c_int]
        _ref_gpu = L
    return _ref_gpu


def ref_hashorder(rows, cols, n: int, num_hashes: int = 16, num_hops: int = 1):
    """The reference's own reorder_hashorder_gpu (GPU): returns the relabelled, oriented
    (rows, cols)."""
    r = np.ascontiguousarray(rows, np.int32).copy()
    c = np.ascontiguousarray(cols, np.int32).copy()
    with _StdoutToStderr():
        rc = ref_gpu().ref_hashorder_gpu(r if len(r) else np.zeros(1, np.int32),
                                         c if len(c) else np.zeros(1, np.int32), len(r), int(n),
                                         int(num_hashes), int(num_hops))
    if rc != 0:
        raise RuntimeError(f"ref_hashorder_gpu failed ({rc})")
    return r, c


class _StdoutToStderr:
    """The reference's convert prints to stdout; keep bench stdout to one JSON line."""

    def __enter__(self):
        import sys
        sys.stdout.flush()
        self.saved = os.dup(1)
        os.dup2(2, 1)

    def __exit__(self, *a):
        import sys
        sys.stdout.flush()
        os.dup2(self.saved, 1)
        os.close(self.saved)


def ref_gpu_run(rows, cols, n: int, tile_cols: int, warmup: int = 1, repeat: int = 5,
                export: bool = False):
    """Reference GPU convert + adaptive count on a lower COO.  Returns a dict with
    count, convert_ms, kernel_ms list and, with export=True, the Bit-BSR arrays."""
    rows, cols = _i32(rows), _i32(cols)
    if len(rows) == 0:
        raise ValueError("the reference build needs at least one edge")
    cnt = C.c_ulonglong(0)
    conv = C.c_float(0)
    kms = np.zeros(max(repeat, 1), np.float32)
    B = C.c_uint32(0)
    R = (n + 15) // 16
    tw = 16 * (tile_cols // 32)
    cap = len(rows)
    bufs = None
    ptrs = [None] * 4
    if export:
        bufs = [np.zeros(R + 1, np.uint32), np.zeros(cap, np.uint32), np.zeros(cap, np.uint32),
                np.zeros(cap * tw, np.uint32)]
        ptrs = [b.ctypes.data for b in bufs]
    with _StdoutToStderr():
        rc = ref_gpu().ref_gpu_run(rows, cols, len(rows), n, tile_cols, warmup, repeat,
                                   C.byref(cnt), C.byref(conv), kms, C.byref(B),
                                   ptrs[0], ptrs[1], ptrs[2], ptrs[3], cap)
    if rc != 0:
        raise RuntimeError(f"reference GPU run failed rc={rc}")
    out = dict(count=int(cnt.value), convert_ms=float(conv.value),
               kernel_ms=[float(x) for x in kms[:repeat]], num_blocks=int(B.value))
    if export:
        nb = int(B.value)
        out.update(indptr=bufs[0], indices=bufs[1][:nb], row_indices=bufs[2][:nb],
                   blocks=bufs[3][:nb * tw])
    return out
