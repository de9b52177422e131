"""Loader and ctypes signatures for libbtc_b200.so (the C ABI of include/btc_c.h).

The engine has no CPU fallback: if the shared library is missing this module
raises, and every call goes through the sm_100a kernels."""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libbtc_b200.so")

BTC_OK = 0
BTC_E_INVAL = -1
BTC_E_NOMEM = -2
BTC_E_CUDA = -3
BTC_E_TIMEOUT = -4
BTC_E_RANGE = -5
BTC_E_CAPACITY = -6

BTC_INPUT_ON_HOST = 0x1
BTC_ORIENT_DEGREE = 0x2
BTC_BUILD_RADIX = 0x4
BTC_BUILD_ASYNC = 0x8
BTC_TAU_DEFAULT = -1
BTC_TAU_ALL_SPARSE = 0x7FFFFFFF

# every symbol include/btc_c.h declares
EXPORTS = [
    "btc_convert_coo_to_bcsr_16x128_gpu",
    "btc_convert_coo_to_bcsr_16x32_gpu",
    "btc_count_triangles_16x128_adaptive",
    "btc_count_triangles_16x32_adaptive",
    "btc_bcsr_free",
    "btc_bcsr_reset_result",
    "btc_bcsr_get_result",
    "btc_preprocess_for_triangle_counting",
    "btc_reorder_hashorder",
    "btc_hashorder_params",
    "btc_should_reorder",
    "btc_lite_select_tile_cols",
    "btc_tile_policy_from_features",
    "btc_select_tile_policy",
    "btc_build_bitbsr",
    "btc_rebuild_bitbsr",
    "btc_count",
    "btc_count_async",
    "btc_bitbsr_info",
    "btc_density_hist",
    "btc_free",
    "btc_default_tau",
    "btc_strerror",
    "btc_abi_version",
    "btc_count_bcsr_noalloc",
    "btc_batch_build",
    "btc_batch_rebuild",
    "btc_batch_count",
    "btc_batch_info",
    "btc_batch_row_offsets",
    "btc_batch_free",
    "btc_server_default_config",
    "btc_server_create",
    "btc_server_submit",
    "btc_server_poll",
    "btc_server_stats_get",
    "btc_server_destroy",
    "btc_partition_tiles",
    "btc_partition_from_costs",
    "btc_count_tiles_async",
    "btc_b1_mma_peak",
]


class BtcBcsrDevice(C.Structure):
    """Field layout of btc::BCSR_16x128_Device / BCSR_16x32_Device
    (btc/operations/bcsr_16x128.h:24-32, bcsr_16x32.h:109-117)."""

    _fields_ = [
        ("indptr", C.c_void_p),
        ("indices", C.c_void_p),
        ("blocks", C.c_void_p),
        ("row_indices", C.c_void_p),
        ("result", C.c_void_p),
        ("n", C.c_int),
        ("n_row_blocks", C.c_int),
        ("num_blocks", C.c_uint32),
    ]


class BtcBitbsrView(C.Structure):
    _fields_ = [
        ("bcsr", BtcBcsrDevice),
        ("tile_cols", C.c_int),
        ("device", C.c_int),
        ("num_edges", C.c_int64),
        ("input_edges", C.c_int64),
        ("device_bytes", C.c_size_t),
    ]


class BtcServerConfig(C.Structure):
    _fields_ = [("hbm_budget_bytes", C.c_uint64), ("max_batch_graphs", C.c_int32),
                ("slots", C.c_int32), ("max_batch_edges", C.c_int64), ("tile_cols", C.c_int),
                ("tau", C.c_int), ("solo_edges", C.c_int64)]


class BtcServerResult(C.Structure):
    _fields_ = [("id", C.c_uint64), ("count", C.c_ulonglong), ("status", C.c_int32),
                ("n", C.c_int32), ("m", C.c_int64), ("submit_s", C.c_double),
                ("done_s", C.c_double)]


class BtcServerStats(C.Structure):
    _fields_ = [("batches", C.c_uint64), ("graphs", C.c_uint64), ("edges", C.c_uint64),
                ("rejected", C.c_uint64), ("queued", C.c_uint64),
                ("peak_device_bytes", C.c_uint64), ("now_s", C.c_double),
                ("solo_launches", C.c_uint64), ("solo_stream_ms", C.c_double),
                ("batch_stream_ms", C.c_double)]


BTC_SUBMIT_BORROW = 0x1


class BtcError(RuntimeError):
    def __init__(self, status: int, where: str):
        self.status = status
        super().__init__(f"{where}: {strerror(status)} (status {status})")


_L = None


def lib():
    global _L
    if _L is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"libbtc_b200.so is not built ({LIB_PATH}); run `make -C btc-tc-artifact_b200` "
                "or __graft_entry__.build()")
        L = C.CDLL(LIB_PATH)
        vp, i32, i64, u32 = C.c_void_p, C.c_int32, C.c_int64, C.c_uint32
        P = C.POINTER
        L.btc_convert_coo_to_bcsr_16x128_gpu.argtypes = [P(BtcBcsrDevice), vp, vp, i64, i32]
        L.btc_convert_coo_to_bcsr_16x32_gpu.argtypes = [P(BtcBcsrDevice), vp, vp, i64, i32]
        L.btc_count_triangles_16x128_adaptive.argtypes = [P(BtcBcsrDevice), C.c_int, P(C.c_float),
                                                          P(C.c_ulonglong)]
        L.btc_count_triangles_16x32_adaptive.argtypes = [P(BtcBcsrDevice), C.c_int, P(C.c_float),
                                                         P(C.c_ulonglong)]
        L.btc_bcsr_free.argtypes = [P(BtcBcsrDevice)]
        L.btc_bcsr_free.restype = None
        L.btc_bcsr_reset_result.argtypes = [P(BtcBcsrDevice)]
        L.btc_bcsr_get_result.argtypes = [P(BtcBcsrDevice), P(C.c_ulonglong)]
        L.btc_preprocess_for_triangle_counting.argtypes = [vp, vp, P(C.c_int64), P(C.c_int32), C.c_int]
        L.btc_reorder_hashorder.argtypes = [vp, vp, i64, i32, C.c_int, C.c_int, vp, vp]
        L.btc_hashorder_params.argtypes = [C.c_int, vp, vp]
        L.btc_should_reorder.argtypes = [i32, i64, C.c_int, C.c_char_p]
        L.btc_lite_select_tile_cols.argtypes = [i64, i32, C.c_int]
        L.btc_tile_policy_from_features.argtypes = [i64, i32, C.c_uint32, C.c_double,
                                                    C.POINTER(C.c_int), C.POINTER(C.c_int)]
        L.btc_select_tile_policy.argtypes = [vp, vp, i64, i32, C.c_uint32, vp,
                                             C.POINTER(C.c_int), C.POINTER(C.c_int)]
        L.btc_build_bitbsr.argtypes = [vp, vp, i64, i32, C.c_int, u32, vp, P(vp)]
        L.btc_rebuild_bitbsr.argtypes = [vp, vp, vp, i64, i32, C.c_int, u32, vp]
        L.btc_count.argtypes = [vp, C.c_int, vp, P(C.c_ulonglong), P(C.c_float)]
        L.btc_count_async.argtypes = [vp, C.c_int, vp, vp]
        L.btc_bitbsr_info.argtypes = [vp, P(BtcBitbsrView)]
        L.btc_density_hist.argtypes = [vp, vp, vp]
        L.btc_free.argtypes = [vp]
        L.btc_free.restype = None
        L.btc_default_tau.argtypes = [C.c_int]
        L.btc_strerror.argtypes = [C.c_int]
        L.btc_strerror.restype = C.c_char_p
        L.btc_abi_version.argtypes = []
        L.btc_count_bcsr_noalloc.argtypes = [P(BtcBcsrDevice), C.c_int, C.c_int, vp, vp]
        L.btc_batch_build.argtypes = [vp, vp, vp, vp, i32, C.c_int, u32, vp, P(vp)]
        L.btc_batch_rebuild.argtypes = [vp, vp, vp, vp, vp, i32, C.c_int, u32, vp]
        L.btc_batch_count.argtypes = [vp, C.c_int, vp, vp, vp]
        L.btc_batch_info.argtypes = [vp, P(BtcBitbsrView)]
        L.btc_batch_row_offsets.argtypes = [vp, vp]
        L.btc_batch_free.argtypes = [vp]
        L.btc_batch_free.restype = None
        L.btc_server_default_config.argtypes = [P(BtcServerConfig)]
        L.btc_server_default_config.restype = None
        L.btc_server_create.argtypes = [P(BtcServerConfig), P(vp)]
        L.btc_server_submit.argtypes = [vp, vp, vp, i64, i32, u32, P(C.c_uint64)]
        L.btc_server_poll.argtypes = [vp, P(BtcServerResult), C.c_int, P(C.c_int), C.c_int]
        L.btc_server_stats_get.argtypes = [vp, P(BtcServerStats)]
        L.btc_server_destroy.argtypes = [vp]
        L.btc_server_destroy.restype = None
        L.btc_partition_tiles.argtypes = [vp, C.c_int, vp, vp]
        L.btc_partition_from_costs.argtypes = [vp, C.c_uint64, u32, u32, C.c_int, vp]
        L.btc_count_tiles_async.argtypes = [vp, u32, u32, C.c_int, vp, vp]
        L.btc_b1_mma_peak.argtypes = [vp, C.c_int, C.POINTER(C.c_double)]
        for name in EXPORTS:
            if name not in ("btc_bcsr_free", "btc_free", "btc_strerror", "btc_batch_free",
                            "btc_server_default_config", "btc_server_destroy"):
                getattr(L, name).restype = C.c_int
        _L = L
    return _L


def strerror(status: int) -> str:
    try:
        return lib().btc_strerror(status).decode()
    except ImportError:
        return f"status {status}"


def check(status: int, where: str) -> None:
    if status != BTC_OK:
        raise BtcError(status, where)
