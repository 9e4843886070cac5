"""fastlanesgpu_b200 -- B200-native (sm_100a) FastLanes decode fused into
Crystal-style query kernels.

The compute lives in libfls_gpu.so (hand-written CUDA behind the C ABI in
include/fls_gpu.h); this package is its Python host face.  There is no CPU
path: the operators fail if the library or a CUDA device is missing.
"""
from ._lib import (LAYOUT_NORMAL, LAYOUT_TRANSPOSED, ORDER_ORIGINAL, ORDER_STORED, SCHEME_CONST, SCHEME_DELTA,
                   SCHEME_DICT, SCHEME_FOR, SCHEME_NAMES, SCHEME_RLE, FlsError)
from .column import DeviceColumn, EncodedColumn

__all__ = ["EncodedColumn", "DeviceColumn", "FlsError", "SCHEME_FOR", "SCHEME_DELTA", "SCHEME_RLE", "SCHEME_CONST",
           "SCHEME_DICT", "SCHEME_NAMES", "LAYOUT_NORMAL", "LAYOUT_TRANSPOSED", "ORDER_STORED", "ORDER_ORIGINAL"]
