"""birdwing_b200 -- B200-native (sm_100a) big-integer multiply.

The product pipeline (limb split, RNS NTTs, pointwise product, Garner CRT,
carry look-back) runs in libbirdwing.so behind the C ABI of
include/birdwing.h; this package is the Python host mirror of the
reference's multiply API.
"""
from ._lib import (BW_PATH_AUTO, BW_PATH_P32, BW_PATH_P64, BW_PTR_DEVICE, BW_PTR_HOST,
                   BwError, lib, LIB_PATH)
from .api import (Batch, Context, Plan, Server, host_multiply_merge, host_multiply_merge_native,
                  host_once_cache_limit, int_to_limbs, limbs_to_int, limits, load_tune_table, multiply,
                  set_tune_entry, size_supported, square, tune_table)

__all__ = [
    "BW_PATH_AUTO", "BW_PATH_P32", "BW_PATH_P64", "BW_PTR_DEVICE", "BW_PTR_HOST", "BwError",
    "Context", "Plan", "host_multiply_merge", "host_multiply_merge_native", "int_to_limbs",
    "limbs_to_int", "limits", "multiply", "size_supported", "square", "lib", "LIB_PATH",
    "Batch", "Server", "tune_table", "set_tune_entry", "load_tune_table", "host_once_cache_limit",
]
