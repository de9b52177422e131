"""B200-native exact triangle counting (Bit-BSR build + hybrid count), Python side.

The compute path is libbtc_b200.so (sm_100a CUDA behind the C ABI in
include/btc_c.h); this package is the host-side mirror of the reference's
``btc`` interface plus seeded graph generators."""
from ._lib import BtcError, LIB_PATH, EXPORTS  # noqa: F401
from .api import (  # noqa: F401
    BCSR_16x128_Device, BCSR_16x32_Device, Batch, BitBSR, Server, CooMatrix, convert_coo_to_bcsr_16x128_gpu,
    convert_coo_to_bcsr_16x32_gpu, count_triangles_16x128_adaptive, count_triangles_16x32_adaptive,
    default_tau, lite_select_tile_cols, preprocess_for_triangle_counting, reorder_hashorder_gpu,
    hashorder_params, should_reorder, should_reorder_gpu, tile_policy, tile_policy_from_features)
from . import graphs  # noqa: F401
