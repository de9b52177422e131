"""Python host mirror of the reference's Bit-BSR build + count interface.

Names, argument meaning and call order follow fanna1234/btc-tc-artifact's
``namespace btc`` (btc/btc.h):

    coo = CooMatrix.from_edges(src, dst, n)                # btc/formats/coo.h
    preprocess_for_triangle_counting(coo)                  # convert.h:600
    bcsr = BCSR_16x128_Device()                            # bcsr_16x128.h:24
    convert_coo_to_bcsr_16x128_gpu(bcsr, coo)              # bcsr_16x128.h:136
    count = count_triangles_16x128_adaptive(bcsr, 2048)    # tc_16x128_adaptive.h:12
    bcsr.free()

Every call goes through libbtc_b200.so (include/btc_c.h).  Where the reference
printed and returned on failure, these raise ``BtcError``.  Device arrays are
torch CUDA int32 tensors (torch is only the allocator and stream provider here);
host arrays are numpy.

``BitBSR`` is the stream-ordered handle API (btc_build_bitbsr / btc_count).
"""
from __future__ import annotations

import ctypes as C

import os

import numpy as np

from . import _lib
from ._lib import BtcError, check, lib

__all__ = [
    "BtcError", "CooMatrix", "BCSR_16x128_Device", "BCSR_16x32_Device",
    "convert_coo_to_bcsr_16x128_gpu", "convert_coo_to_bcsr_16x32_gpu",
    "count_triangles_16x128_adaptive", "count_triangles_16x32_adaptive",
    "preprocess_for_triangle_counting", "lite_select_tile_cols", "BitBSR", "default_tau",
    "tile_policy", "tile_policy_from_features",
    "Batch", "Server",
]


def _torch():
    import torch
    return torch


def _stream_ptr(stream) -> int | None:
    if stream is None:
        return None
    if isinstance(stream, int):
        return stream
    return int(stream.cuda_stream)


# ---------------------------------------------------------------------------
# reference-shaped surface
# ---------------------------------------------------------------------------

class CooMatrix:
    """Device COO matrix (btc/formats/coo.h:10-33): int32 row/column index tensors."""

    def __init__(self, row_indices, column_indices, num_rows: int, num_cols: int | None = None):
        torch = _torch()
        self.row_indices = torch.as_tensor(row_indices, dtype=torch.int32, device="cuda").contiguous()
        self.column_indices = torch.as_tensor(column_indices, dtype=torch.int32,
                                              device="cuda").contiguous()
        self.num_rows = int(num_rows)
        self.num_cols = int(num_cols if num_cols is not None else num_rows)

    @classmethod
    def from_edges(cls, src, dst, n: int) -> "CooMatrix":
        return cls(src, dst, n)

    @property
    def num_entries(self) -> int:
        return int(self.row_indices.numel())

    def free(self):
        torch = _torch()
        self.row_indices = torch.zeros(0, dtype=torch.int32, device="cuda")
        self.column_indices = torch.zeros(0, dtype=torch.int32, device="cuda")


def preprocess_for_triangle_counting(coo: CooMatrix, force_cpu: bool = False,
                                     lower_triangular: bool = True, input_file: str = "",
                                     remap: bool = True, reorder: int | None = None) -> None:
    """convert.h:600-690: orient to (max,min), drop self-loops, sort, unique, compact ids
    (remap), then the reorder step the reference selects with BTC_REORDER: 0 none, 8 GPU
    HashOrder, 9 HashOrder when should_reorder_gpu says so (input_file's base name is
    the dataset hint).  `reorder` overrides the environment; with neither, no reorder
    (the reference defaults to 9: ids here stay stable unless asked).  Runs on the GPU
    whatever `force_cpu` says (the engine has no CPU path); `lower_triangular=False` is
    not supported."""
    if reorder is None:
        reorder = int(os.environ.get("BTC_REORDER", "0"))
    if reorder not in (0, 8, 9):
        raise BtcError(_lib.BTC_E_INVAL, f"reorder mode {reorder} (0, 8 and 9 are supported)")
    if not lower_triangular:
        raise BtcError(_lib.BTC_E_INVAL, "preprocess_for_triangle_counting(lower_triangular=False)")
    nnz = C.c_int64(coo.num_entries)
    rows = C.c_int32(coo.num_rows)
    st = lib().btc_preprocess_for_triangle_counting(coo.row_indices.data_ptr(),
                                                    coo.column_indices.data_ptr(),
                                                    C.byref(nnz), C.byref(rows), int(remap))
    check(st, "preprocess_for_triangle_counting")
    coo.row_indices = coo.row_indices[: nnz.value].clone()
    coo.column_indices = coo.column_indices[: nnz.value].clone()
    coo.num_rows = coo.num_cols = int(rows.value)
    hint = os.path.splitext(os.path.basename(input_file))[0] if input_file else ""
    if reorder == 8 or (reorder == 9 and should_reorder_gpu(coo, hint)):
        hashes, hops = hashorder_env()
        reorder_hashorder_gpu(coo, hashes, hops)


def hashorder_env() -> tuple[int, int]:
    """(num_hashes, num_hops) for the HashOrder step of preprocess_for_triangle_counting:
    BTC_HASHORDER_HASHES and BTC_HASHORDER_HOPS, 16 and 1 when unset (convert.h:668-683,
    which parses them with atoi)."""
    def atoi(name: str, default: int) -> int:
        v = os.environ.get(name)
        if v is None:
            return default
        digits = ""
        for ch in v.strip():
            if ch.isdigit() or (not digits and ch in "+-"):
                digits += ch
            else:
                break
        try:
            return int(digits)
        except ValueError:
            return 0
    return atoi("BTC_HASHORDER_HASHES", 16), atoi("BTC_HASHORDER_HOPS", 1)


def reorder_hashorder_gpu(coo: CooMatrix, num_hashes: int = 16, num_hops: int = 1):
    """reorder.h:443-587 (btc_reorder_hashorder): relabels coo in place by MinHash
    signature order and orients it to (max, min); returns the permutation as an int32
    CUDA tensor (new id = perm[old id])."""
    torch = _torch()
    perm = torch.empty(max(coo.num_rows, 1), dtype=torch.int32, device=coo.row_indices.device)
    check(lib().btc_reorder_hashorder(coo.row_indices.data_ptr(), coo.column_indices.data_ptr(),
                                      int(coo.row_indices.numel()), int(coo.num_rows),
                                      int(num_hashes), int(num_hops), perm.data_ptr(),
                                      _stream_ptr(None)), "btc_reorder_hashorder")
    return perm[: coo.num_rows]


def hashorder_params(num_hashes: int = 16):
    """The MinHash parameters (a, b) btc_reorder_hashorder uses, as uint32 arrays."""
    a = np.zeros(num_hashes, np.uint32)
    b = np.zeros(num_hashes, np.uint32)
    check(lib().btc_hashorder_params(int(num_hashes), a.ctypes.data, b.ctypes.data),
          "btc_hashorder_params")
    return a, b


def should_reorder(num_rows: int, nnz: int, sm_version: int, dataset_hint: str = "") -> bool:
    """convert.h:443-596 (btc_should_reorder): the reference's automatic reorder rule."""
    return bool(lib().btc_should_reorder(int(num_rows), int(nnz), int(sm_version),
                                         dataset_hint.encode() if dataset_hint else None))


def should_reorder_gpu(coo: CooMatrix, dataset_hint: str = "") -> bool:
    """should_reorder_gpu (convert.h:579-596) for the current device."""
    torch = _torch()
    major, minor = torch.cuda.get_device_capability()
    return should_reorder(coo.num_rows, int(coo.row_indices.numel()), 10 * major + minor,
                          dataset_hint)


class _BcsrDevice:
    TILE_COLS = 0
    WORDS = 0

    def __init__(self):
        self._s = _lib.BtcBcsrDevice()

    # reference fields
    @property
    def n(self): return self._s.n

    @property
    def n_row_blocks(self): return self._s.n_row_blocks

    @property
    def num_blocks(self): return self._s.num_blocks

    @property
    def indptr(self): return self._s.indptr

    @property
    def indices(self): return self._s.indices

    @property
    def row_indices(self): return self._s.row_indices

    @property
    def blocks(self): return self._s.blocks

    @property
    def result(self): return self._s.result

    def free(self):
        lib().btc_bcsr_free(C.byref(self._s))

    def reset_result(self):
        check(lib().btc_bcsr_reset_result(C.byref(self._s)), "reset_result")

    def get_result(self) -> int:
        v = C.c_ulonglong(0)
        check(lib().btc_bcsr_get_result(C.byref(self._s), C.byref(v)), "get_result")
        return int(v.value)

    def to_host(self) -> dict:
        """Copy the arrays out (for inspection and parity checks)."""
        return _copy_out(self._s, self.TILE_COLS)

    def __del__(self):
        try:
            if self._s.indptr:
                self.free()
        except Exception:
            pass


class BCSR_16x128_Device(_BcsrDevice):
    TILE_COLS = 128


class BCSR_16x32_Device(_BcsrDevice):
    TILE_COLS = 32


class _DeviceWords:
    """Zero-copy view of `count` 32-bit words of engine-owned device memory."""

    def __init__(self, ptr: int, count: int):
        self.__cuda_array_interface__ = {"shape": (count,), "typestr": "<i4",
                                         "data": (ptr, False), "version": 3}


def _copy_out(s, tile_cols: int) -> dict:
    torch = _torch()
    tw = 16 * (tile_cols // 32)
    B = int(s.num_blocks)
    R = int(s.n_row_blocks)

    def grab(ptr, count):
        if count <= 0 or not ptr:
            return np.zeros(max(count, 0), np.uint32)
        view = _DeviceWords(int(ptr), int(count))
        return torch.as_tensor(view, device="cuda").cpu().numpy().view(np.uint32).copy()

    return dict(n=int(s.n), tile_cols=tile_cols, n_row_blocks=R, num_blocks=B,
                indptr=grab(s.indptr, R + 1), indices=grab(s.indices, B),
                row_indices=grab(s.row_indices, B), blocks=grab(s.blocks, B * tw))


def _convert(fn, bcsr: _BcsrDevice, coo: CooMatrix):
    if bcsr._s.indptr:
        bcsr.free()
    st = fn(C.byref(bcsr._s), coo.row_indices.data_ptr(), coo.column_indices.data_ptr(),
            coo.num_entries, coo.num_rows)
    check(st, fn.__name__)


def convert_coo_to_bcsr_16x128_gpu(bcsr: BCSR_16x128_Device, coo: CooMatrix) -> None:
    """bcsr_16x128.h:136-241."""
    _convert(lib().btc_convert_coo_to_bcsr_16x128_gpu, bcsr, coo)


def convert_coo_to_bcsr_16x32_gpu(bcsr: BCSR_16x32_Device, coo: CooMatrix) -> None:
    """bcsr_16x32.h:144-249."""
    _convert(lib().btc_convert_coo_to_bcsr_16x32_gpu, bcsr, coo)


def _count(fn, bcsr: _BcsrDevice, threshold_blocks: int, kernel_ms):
    out = C.c_ulonglong(0)
    ms = C.c_float(0.0)
    st = fn(C.byref(bcsr._s), int(threshold_blocks), C.byref(ms) if kernel_ms is not None else None,
            C.byref(out))
    check(st, fn.__name__)
    if kernel_ms is not None:
        kernel_ms.append(float(ms.value))
    return int(out.value)


def count_triangles_16x128_adaptive(bcsr: BCSR_16x128_Device, threshold_blocks: int = 2048,
                                    kernel_ms: list | None = None) -> int:
    """tc_16x128_adaptive.h:12-29.  `kernel_ms`, if a list, receives the kernel time."""
    return _count(lib().btc_count_triangles_16x128_adaptive, bcsr, threshold_blocks, kernel_ms)


def count_triangles_16x32_adaptive(bcsr: BCSR_16x32_Device, threshold_blocks: int = 40000,
                                   kernel_ms: list | None = None) -> int:
    """tc_16x32_adaptive.h:14-31."""
    return _count(lib().btc_count_triangles_16x32_adaptive, bcsr, threshold_blocks, kernel_ms)


def lite_select_tile_cols(nnz: int, num_rows: int, mode: int = 0) -> int:
    """BTC-Lite O(1) policy (apps/btc_tc_lite.cu:45-65)."""
    return int(lib().btc_lite_select_tile_cols(int(nnz), int(num_rows), int(mode)))


def default_tau(tile_cols: int) -> int:
    return int(lib().btc_default_tau(int(tile_cols)))


def tile_policy_from_features(m: int, n: int, orient_degree: bool = False,
                              locality: float = 0.0) -> tuple[int, int]:
    """The engine's tile policy (btc_tile_policy_from_features): (tile_cols, tau) from the
    edge count, vertex count, degree-ordering request and id locality."""
    c, t = C.c_int(0), C.c_int(0)
    flags = _lib.BTC_ORIENT_DEGREE if orient_degree else 0
    check(lib().btc_tile_policy_from_features(int(m), int(n), flags, float(locality), C.byref(c),
                                              C.byref(t)), "btc_tile_policy_from_features")
    return int(c.value), int(t.value)


def tile_policy(src, dst, n: int, orient_degree: bool = False, stream=None) -> tuple[int, int]:
    """(tile_cols, tau) the engine picks for this edge list (btc_select_tile_policy; what
    tile_cols=0 applies).  numpy arrays are sampled on the host, CUDA tensors on the GPU."""
    sp, dp, m, flags, keep = _edge_ptrs(src, dst)
    if orient_degree:
        flags |= _lib.BTC_ORIENT_DEGREE
    c, t = C.c_int(0), C.c_int(0)
    check(lib().btc_select_tile_policy(sp, dp, m, int(n), flags, _stream_ptr(stream), C.byref(c),
                                       C.byref(t)), "btc_select_tile_policy")
    del keep
    return int(c.value), int(t.value)


# ---------------------------------------------------------------------------
# stream-ordered handle API
# ---------------------------------------------------------------------------

def _edge_ptrs(src, dst):
    """(src_ptr, dst_ptr, m, flags, keepalive) for torch CUDA tensors or numpy arrays."""
    if isinstance(src, np.ndarray) or isinstance(dst, np.ndarray):
        s = np.ascontiguousarray(src, dtype=np.int32)
        d = np.ascontiguousarray(dst, dtype=np.int32)
        if s.shape != d.shape:
            raise BtcError(_lib.BTC_E_INVAL, "edge arrays differ in length")
        return s.ctypes.data, d.ctypes.data, int(s.size), _lib.BTC_INPUT_ON_HOST, (s, d)
    torch = _torch()
    if src.dtype != torch.int32 or dst.dtype != torch.int32:
        raise BtcError(_lib.BTC_E_INVAL, "edge tensors must be int32")
    if src.numel() != dst.numel():
        raise BtcError(_lib.BTC_E_INVAL, "edge arrays differ in length")
    s = src.contiguous()
    d = dst.contiguous()
    flags = _lib.BTC_INPUT_ON_HOST if not s.is_cuda else 0
    return s.data_ptr(), d.data_ptr(), int(s.numel()), flags, (s, d)


class BitBSR:
    """Device-resident Bit-BSR handle (btc_build_bitbsr ... btc_free)."""

    def __init__(self, src, dst, n: int, tile_cols: int = 0, orient_degree: bool = False,
                 stream=None, radix: bool = False):
        self._h = C.c_void_p(None)
        sp, dp, m, flags, self._keep = _edge_ptrs(src, dst)
        if orient_degree:
            flags |= _lib.BTC_ORIENT_DEGREE
        if radix:
            flags |= _lib.BTC_BUILD_RADIX
        st = lib().btc_build_bitbsr(sp, dp, m, int(n), int(tile_cols), flags, _stream_ptr(stream),
                                    C.byref(self._h))
        check(st, "btc_build_bitbsr")
        self._keep = None

    def rebuild(self, src, dst, n: int, tile_cols: int = 0, orient_degree: bool = False,
                stream=None, radix: bool = False, asynchronous: bool = False) -> None:
        """Rebuild into this handle.  asynchronous=True enqueues the build without waiting
        when the handle's arrays from the previous build have room (BTC_BUILD_ASYNC); its
        status then comes with the next call that waits (count, info, ...).  The inputs
        (and any converted copies, kept on the handle) must outlive the enqueued build."""
        sp, dp, m, flags, keep = _edge_ptrs(src, dst)
        if orient_degree:
            flags |= _lib.BTC_ORIENT_DEGREE
        if radix:
            flags |= _lib.BTC_BUILD_RADIX
        if asynchronous:
            flags |= _lib.BTC_BUILD_ASYNC
        check(lib().btc_rebuild_bitbsr(self._h, sp, dp, m, int(n), int(tile_cols), flags,
                                       _stream_ptr(stream)), "btc_rebuild_bitbsr")
        self._keep = keep if asynchronous else None

    def count(self, tau: int = _lib.BTC_TAU_DEFAULT, stream=None, timing: bool = False):
        out = C.c_ulonglong(0)
        ms = C.c_float(0.0)
        check(lib().btc_count(self._h, int(tau), _stream_ptr(stream), C.byref(out),
                              C.byref(ms) if timing else None), "btc_count")
        return (int(out.value), float(ms.value)) if timing else int(out.value)

    def count_async(self, tau: int = _lib.BTC_TAU_DEFAULT, stream=None, d_out: int | None = None):
        check(lib().btc_count_async(self._h, int(tau), _stream_ptr(stream), d_out), "btc_count_async")

    def partition(self, parts: int, stream=None) -> list[int]:
        """Tile bounds [b_0 = 0, ..., b_parts = num_tiles] of `parts` ranges of about equal
        estimated count cost (btc_partition_tiles)."""
        b = np.zeros(int(parts) + 1, np.uint32)
        check(lib().btc_partition_tiles(self._h, int(parts), _stream_ptr(stream), b.ctypes.data),
              "btc_partition_tiles")
        return [int(x) for x in b]

    def count_tiles(self, tile_begin: int, tile_end: int, tau: int = _lib.BTC_TAU_DEFAULT,
                    stream=None, out=None):
        """Enqueues the count of sample tiles [tile_begin, tile_end) into `out`, a one-element
        int64 CUDA tensor (made on the current device when None), and returns `out`."""
        import torch
        if out is None:
            out = torch.zeros(1, dtype=torch.int64, device=f"cuda:{torch.cuda.current_device()}")
        check(lib().btc_count_tiles_async(self._h, int(tile_begin), int(tile_end), int(tau),
                                          _stream_ptr(stream), out.data_ptr()),
              "btc_count_tiles_async")
        return out

    def info(self) -> _lib.BtcBitbsrView:
        v = _lib.BtcBitbsrView()
        check(lib().btc_bitbsr_info(self._h, C.byref(v)), "btc_bitbsr_info")
        return v

    @property
    def num_tiles(self) -> int:
        return int(self.info().bcsr.num_blocks)

    @property
    def tile_cols(self) -> int:
        return int(self.info().tile_cols)

    @property
    def num_edges(self) -> int:
        return int(self.info().num_edges)

    def density_hist(self, stream=None) -> np.ndarray:
        tc = self.tile_cols
        h = np.zeros(16 * tc + 1, np.uint64)
        check(lib().btc_density_hist(self._h, _stream_ptr(stream), h.ctypes.data), "btc_density_hist")
        return h

    def to_host(self) -> dict:
        v = self.info()
        return _copy_out(v.bcsr, int(v.tile_cols))

    def free(self) -> None:
        if self._h:
            lib().btc_free(self._h)
            self._h = C.c_void_p(None)

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class Batch:
    """Many graphs in one Bit-BSR build and one count launch (btc_batch_*).

    graphs: list of (src, dst, n) with local vertex ids; or pass concatenated arrays
    with ``offsets`` (num_graphs+1) and ``num_vertices``.  Arrays may be numpy (host) or
    torch CUDA int32 tensors."""

    def __init__(self, graphs=None, tile_cols: int = 0, stream=None, *, src=None, dst=None,
                 offsets=None, num_vertices=None):
        self._h = C.c_void_p(None)
        self._build(lib().btc_batch_build, graphs, tile_cols, stream, src, dst, offsets,
                    num_vertices, first=True)

    @staticmethod
    def concat(graphs):
        srcs = [np.asarray(s, np.int32) for s, _, _ in graphs]
        dsts = [np.asarray(d, np.int32) for _, d, _ in graphs]
        offsets = np.zeros(len(graphs) + 1, np.int64)
        offsets[1:] = np.cumsum([len(s) for s in srcs])
        nv = np.array([n for _, _, n in graphs], np.int32)
        src = np.concatenate(srcs) if srcs else np.zeros(0, np.int32)
        dst = np.concatenate(dsts) if dsts else np.zeros(0, np.int32)
        return src, dst, offsets, nv

    def _build(self, fn, graphs, tile_cols, stream, src, dst, offsets, num_vertices, first,
               asynchronous=False):
        if graphs is not None:
            src, dst, offsets, num_vertices = Batch.concat(graphs)
        offsets = np.ascontiguousarray(offsets, np.int64)
        num_vertices = np.ascontiguousarray(num_vertices, np.int32)
        sp, dp, m, flags, keep = _edge_ptrs(src, dst)
        if asynchronous:
            flags |= _lib.BTC_BUILD_ASYNC
        if m != int(offsets[-1]):
            raise BtcError(_lib.BTC_E_INVAL, "offsets[-1] != number of edges")
        self.num_graphs = len(num_vertices)
        args = [sp, dp, offsets.ctypes.data, num_vertices.ctypes.data, self.num_graphs,
                int(tile_cols), flags, _stream_ptr(stream)]
        if first:
            check(fn(*args, C.byref(self._h)), "btc_batch_build")
        else:
            check(fn(self._h, *args), "btc_batch_rebuild")
        # an enqueued build reads the edges after this call returns
        self._keep = keep if asynchronous else None

    def rebuild(self, graphs=None, tile_cols: int = 0, stream=None, *, src=None, dst=None,
                offsets=None, num_vertices=None, asynchronous: bool = False) -> None:
        """asynchronous=True enqueues the rebuild without host work or a wait when the graphs'
        sizes equal the last build's and the edges are on the device (btc_batch_rebuild with
        BTC_BUILD_ASYNC); its status comes with the next waiting call.  The edge tensors
        must outlive the enqueued build."""
        self._build(lib().btc_batch_rebuild, graphs, tile_cols, stream, src, dst, offsets,
                    num_vertices, first=False, asynchronous=asynchronous)

    def count(self, tau: int = _lib.BTC_TAU_DEFAULT, stream=None) -> np.ndarray:
        """Per-graph triangle counts (uint64 numpy array); waits for them."""
        out = np.zeros(self.num_graphs, np.uint64)
        check(lib().btc_batch_count(self._h, int(tau), _stream_ptr(stream), None,
                                    out.ctypes.data), "btc_batch_count")
        return out

    def count_async(self, d_counts: int, tau: int = _lib.BTC_TAU_DEFAULT, stream=None) -> None:
        """Counts into device memory d_counts (num_graphs uint64) without waiting."""
        check(lib().btc_batch_count(self._h, int(tau), _stream_ptr(stream), d_counts, None),
              "btc_batch_count")

    def info(self) -> _lib.BtcBitbsrView:
        v = _lib.BtcBitbsrView()
        check(lib().btc_batch_info(self._h, C.byref(v)), "btc_batch_info")
        return v

    def row_offsets(self) -> np.ndarray:
        out = np.zeros(self.num_graphs + 1, np.uint32)
        check(lib().btc_batch_row_offsets(self._h, out.ctypes.data), "btc_batch_row_offsets")
        return out

    def to_host(self) -> dict:
        v = self.info()
        return _copy_out(v.bcsr, int(v.tile_cols))

    def free(self) -> None:
        if self._h:
            lib().btc_batch_free(self._h)
            self._h = C.c_void_p(None)

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class Server:
    """Continuous-batching count server (btc_server_*).  slots=1, max_batch_graphs=1 is
    the plain one-request-at-a-time path."""

    def __init__(self, hbm_budget_bytes: int | None = None, max_batch_graphs: int | None = None,
                 slots: int | None = None, max_batch_edges: int | None = None,
                 tile_cols: int | None = None, tau: int | None = None,
                 solo_edges: int | None = None):
        cfg = _lib.BtcServerConfig()
        lib().btc_server_default_config(C.byref(cfg))
        for k, v in dict(hbm_budget_bytes=hbm_budget_bytes, max_batch_graphs=max_batch_graphs,
                         slots=slots, max_batch_edges=max_batch_edges, tile_cols=tile_cols,
                         tau=tau, solo_edges=solo_edges).items():
            if v is not None:
                setattr(cfg, k, v)
        self._h = C.c_void_p(None)
        self._keep = {}
        check(lib().btc_server_create(C.byref(cfg), C.byref(self._h)), "btc_server_create")

    def submit(self, src, dst, n: int, borrow: bool = False) -> int:
        """Queue one request (numpy int32 arrays).  borrow=True reads the arrays in place
        (they are kept referenced here until the result is polled)."""
        s = np.ascontiguousarray(src, np.int32)
        d = np.ascontiguousarray(dst, np.int32)
        rid = C.c_uint64(0)
        check(lib().btc_server_submit(self._h, s.ctypes.data, d.ctypes.data, len(s), int(n),
                                      _lib.BTC_SUBMIT_BORROW if borrow else 0, C.byref(rid)),
              "btc_server_submit")
        if borrow:
            self._keep[int(rid.value)] = (s, d)
        return int(rid.value)

    def poll(self, max_results: int = 4096, wait_ms: int = 0) -> list:
        buf = (_lib.BtcServerResult * max_results)()
        k = C.c_int(0)
        check(lib().btc_server_poll(self._h, buf, max_results, C.byref(k), int(wait_ms)),
              "btc_server_poll")
        out = []
        for i in range(k.value):
            r = buf[i]
            self._keep.pop(int(r.id), None)
            out.append(dict(id=int(r.id), count=int(r.count), status=int(r.status), n=int(r.n),
                            m=int(r.m), submit_s=float(r.submit_s), done_s=float(r.done_s)))
        return out

    def stats(self) -> dict:
        st = _lib.BtcServerStats()
        check(lib().btc_server_stats_get(self._h, C.byref(st)), "btc_server_stats_get")
        return {k: getattr(st, k) for k, _ in st._fields_}

    def close(self) -> None:
        if self._h:
            lib().btc_server_destroy(self._h)
            self._h = C.c_void_p(None)
            self._keep.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
