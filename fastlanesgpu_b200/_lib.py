"""ctypes binding of libfls_gpu.so (the C ABI declared in include/fls_gpu.h).

The library is built in-tree (``python -m fastlanesgpu_b200.build``).  There is
no fallback: if the shared library is missing or fails to load, importing the
operators raises.
"""
from __future__ import annotations

import ctypes
import os

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "libfls_gpu.so")

FLS_OK = 0
STATUS_NAMES = {0: "FLS_OK", 1: "FLS_ERR_INVALID_ARG", 2: "FLS_ERR_BAD_BW", 3: "FLS_ERR_ALIGNMENT",
                4: "FLS_ERR_CUDA", 5: "FLS_ERR_DEVICE", 6: "FLS_ERR_TIMEOUT", 7: "FLS_ERR_UNSUPPORTED",
                8: "FLS_ERR_CAPACITY", 9: "FLS_ERR_NO_DEVICE"}

SCHEME_FOR, SCHEME_DELTA, SCHEME_RLE, SCHEME_CONST, SCHEME_DICT = 0, 1, 2, 3, 4
SCHEME_NAMES = ["FOR", "DELTA", "RLE", "CONST", "DICT"]
LAYOUT_NORMAL, LAYOUT_TRANSPOSED = 0, 1
RFOR_TILE = 512  # values per tile of the RFOR format (FLS_RFOR_TILE)
ORDER_STORED, ORDER_ORIGINAL = 0, 1
MAX_QUERY_COLS, MAX_FILTERS, MAX_PROBES = 8, 4, 4
TUNE_SPARSE_ROWS, TUNE_JIT, TUNE_GROUP_SMEM, TUNE_LATE_MEASURE, TUNE_TABLE_KB, TUNE_HALF_VECTORS = 0, 1, 2, 3, 4, 5
MLP_IN, MLP_HIDDEN, MLP_OUT = 16, 64, 5
MLP_N_PARAMS = 64 * 16 + 64 + 64 * 64 + 64 + 5 * 64 + 5


class FlsError(RuntimeError):
    """A non-OK fls_status, with the library's message."""

    def __init__(self, status: int, where: str, msg: str):
        super().__init__(f"{where}: {STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


class VecMeta(ctypes.Structure):
    _fields_ = [("offset", ctypes.c_uint64), ("base", ctypes.c_int32), ("scheme", ctypes.c_uint8),
                ("bw", ctypes.c_uint8), ("aux", ctypes.c_uint16)]


class Column(ctypes.Structure):
    _fields_ = [("data", ctypes.c_void_p), ("meta", ctypes.c_void_p), ("n_values", ctypes.c_uint64),
                ("n_words", ctypes.c_uint64), ("layout", ctypes.c_uint32), ("scheme", ctypes.c_uint32),
                ("bw", ctypes.c_uint32), ("base", ctypes.c_int32), ("max_vec_words", ctypes.c_uint32),
                ("scheme_mask", ctypes.c_uint32)]


class Filter(ctypes.Structure):
    _fields_ = [("col", ctypes.c_uint32), ("lo", ctypes.c_int32), ("hi", ctypes.c_int32)]


class FilterAggDesc(ctypes.Structure):
    _fields_ = [("cols", ctypes.POINTER(Column)), ("n_cols", ctypes.c_uint32),
                ("filters", Filter * MAX_FILTERS), ("n_filters", ctypes.c_uint32),
                ("agg_a", ctypes.c_int32), ("agg_b", ctypes.c_int32)]


class BatchQuery(ctypes.Structure):
    _fields_ = [("col", ctypes.c_uint32), ("lo", ctypes.c_int32), ("hi", ctypes.c_int32), ("agg_col", ctypes.c_uint32),
                ("n_values", ctypes.c_uint64)]


class Probe(ctypes.Structure):
    _fields_ = [("col", ctypes.c_uint32), ("ht", ctypes.c_void_p), ("ht_len", ctypes.c_int32),
                ("keys_min", ctypes.c_int32), ("kind", ctypes.c_int32)]


class JoinAggDesc(ctypes.Structure):
    _fields_ = [("cols", ctypes.POINTER(Column)), ("n_cols", ctypes.c_uint32),
                ("probes", Probe * MAX_PROBES), ("n_probes", ctypes.c_uint32), ("agg_col", ctypes.c_uint32),
                ("key_a", ctypes.c_int32), ("key_b", ctypes.c_int32), ("group_mul", ctypes.c_int32),
                ("group_sub", ctypes.c_int32), ("n_groups", ctypes.c_int32)]


MAX_GROUP_KEYS = 3


class JoinGroupbyDesc(ctypes.Structure):
    _fields_ = [("cols", ctypes.POINTER(Column)), ("n_cols", ctypes.c_uint32),
                ("probes", Probe * MAX_PROBES), ("n_probes", ctypes.c_uint32), ("agg_col", ctypes.c_uint32),
                ("agg_sub_col", ctypes.c_int32), ("n_keys", ctypes.c_uint32),
                ("key_probe", ctypes.c_int32 * MAX_GROUP_KEYS), ("key_mul", ctypes.c_int32 * MAX_GROUP_KEYS),
                ("key_slot", ctypes.c_int32 * MAX_GROUP_KEYS), ("group_sub", ctypes.c_int32),
                ("n_groups", ctypes.c_int32), ("res_stride", ctypes.c_uint32), ("sum_slot", ctypes.c_uint32),
                ("sum_bits", ctypes.c_uint32)]


class RforColumnDesc(ctypes.Structure):
    _fields_ = [("values", ctypes.c_void_p), ("run_lengths", ctypes.c_void_p), ("val_offsets", ctypes.c_void_p),
                ("rl_offsets", ctypes.c_void_p), ("n_values", ctypes.c_uint64), ("n_val_words", ctypes.c_uint64),
                ("n_rl_words", ctypes.c_uint64)]


class JitStats(ctypes.Structure):
    _fields_ = [("compiled", ctypes.c_uint64), ("launches", ctypes.c_uint64), ("failures", ctypes.c_uint64),
                ("cached", ctypes.c_uint64)]


_u32p = ctypes.POINTER(ctypes.c_uint32)
_i32p = ctypes.POINTER(ctypes.c_int32)
_VP = ctypes.c_void_p

# name -> (restype, argtypes)
_SIGS = {
    "fls_last_error": (ctypes.c_char_p, []),
    "fls_check_device_error": (ctypes.c_int, [_VP]),
    "fls_bind_error_word": (ctypes.c_int, [_VP, _VP]),
    "fls_pack_u32": (ctypes.c_int, [_VP, _VP, ctypes.c_uint8]),
    "fls_transpose_i_u32": (ctypes.c_int, [_VP, _VP]),
    "fls_untranspose_u32": (ctypes.c_int, [_VP, _VP]),
    "fls_unrsum_u32": (ctypes.c_int, [_VP, _VP]),
    "fls_vector_rle": (ctypes.c_int, [_VP, _VP, _VP, _VP, _VP]),
    "fls_encode_bound_words": (ctypes.c_uint64, [ctypes.c_uint64]),
    "fls_encode_uniform": (ctypes.c_int, [_VP, ctypes.c_uint64, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint8,
                                          ctypes.c_int32, _VP, _VP, _VP]),
    "fls_encode_column": (ctypes.c_int, [_VP, ctypes.c_uint64, _VP, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_int,
                                         _VP, _VP, _VP, _VP, _VP]),
    "fls_encode_exhaustive": (ctypes.c_int, [_VP, ctypes.c_uint64, _VP, _VP, ctypes.c_int]),
    "fls_vector_stats": (ctypes.c_int, [_VP, ctypes.c_uint64, _VP, ctypes.c_int]),
    "fls_decode_u32": (ctypes.c_int, [ctypes.POINTER(Column), _VP, ctypes.c_uint32, _VP]),
    "fls_decode_sum_u32": (ctypes.c_int, [ctypes.POINTER(Column), _VP, _VP]),
    "fls_query_filter_agg": (ctypes.c_int, [ctypes.POINTER(FilterAggDesc), _VP, _VP]),
    "fls_pht_build": (ctypes.c_int, [_VP, ctypes.c_int32, _VP, _VP, ctypes.c_uint64, _VP, ctypes.c_int32,
                                     ctypes.c_int32, _VP]),
    "fls_query_probe_groupby": (ctypes.c_int, [ctypes.POINTER(JoinAggDesc), _VP, _VP]),
    "fls_pht_build_ranges": (ctypes.c_int, [_VP] + [ctypes.c_int32] * 4 + [_VP, _VP, ctypes.c_uint64, _VP,
                                                                            ctypes.c_int32, ctypes.c_int32, _VP]),
    "fls_query_probe_groupby_ws": (ctypes.c_int, [ctypes.POINTER(JoinAggDesc), _VP, _VP, ctypes.c_uint64, _VP]),
    "fls_probe_workspace_bytes": (ctypes.c_uint64, [ctypes.POINTER(JoinAggDesc)]),
    "fls_set_launch_config": (ctypes.c_int, [ctypes.c_uint32] * 4),
    "fls_get_launch_config": (ctypes.c_int, [_VP, _VP, _VP, _VP]),
    "fls_kernel_launch_count": (ctypes.c_uint64, []),
    "fls_crystal_q11": (ctypes.c_int, [_VP, ctypes.c_uint32] * 4 + [ctypes.c_uint64] + [ctypes.c_int32] * 5
                        + [_VP, _VP]),
    "fls_crystal_q21_probe": (ctypes.c_int, [_VP, ctypes.c_uint32] * 4 + [ctypes.c_uint64]
                              + [_VP, ctypes.c_int32] * 3 + [ctypes.c_int32, _VP, _VP]),
    "fls_set_tuning": (ctypes.c_int, [ctypes.c_uint32, ctypes.c_int64]),
    "fls_vector_stats_gpu": (ctypes.c_int, [_VP, ctypes.c_uint64, _VP, _VP]),
    "fls_batch_create": (ctypes.c_int, [ctypes.POINTER(Column), ctypes.c_uint32, ctypes.POINTER(BatchQuery),
                                        ctypes.c_uint32, ctypes.c_uint32, _VP]),
    "fls_batch_workspace_bytes": (ctypes.c_uint64, [_VP]),
    "fls_batch_items": (ctypes.c_uint32, [_VP]),
    "fls_batch_upload": (ctypes.c_int, [_VP, _VP, ctypes.c_uint64, _VP]),
    "fls_batch_run": (ctypes.c_int, [_VP, _VP, _VP]),
    "fls_batch_destroy": (None, [_VP]),
    "fls_mlp_init": (ctypes.c_int, [_VP, ctypes.c_uint64, _VP]),
    "fls_mlp_workspace_bytes": (ctypes.c_uint64, [ctypes.c_uint32]),
    "fls_mlp_gradients": (ctypes.c_int, [_VP, _VP, _VP, ctypes.c_uint32, _VP, ctypes.c_uint64, _VP, _VP, _VP]),
    "fls_mlp_gradients_static": (ctypes.c_int, [_VP, _VP, _VP, ctypes.c_uint32, _VP, _VP, _VP]),
    "fls_mlp_adam_step": (ctypes.c_int, [_VP, _VP, _VP, _VP, ctypes.c_float, ctypes.c_float, ctypes.c_float,
                                         ctypes.c_float, ctypes.c_uint32, _VP]),
    "fls_mlp_infer": (ctypes.c_int, [_VP, _VP, ctypes.c_uint64, _VP, _VP, _VP, _VP]),
    "fls_get_tuning": (ctypes.c_int, [ctypes.c_uint32, _VP]),
    "fls_encode_gpu_workspace_bytes": (ctypes.c_uint64, [ctypes.c_uint64]),
    "fls_encode_column_gpu": (ctypes.c_int, [_VP, ctypes.c_uint64, _VP, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_int,
                                             _VP, ctypes.c_uint64, _VP, _VP, _VP, ctypes.c_uint64, _VP]),
    "fls_selftest_bounded_wait": (ctypes.c_int, [ctypes.c_uint32, _VP]),
    "fls_pack_u8": (ctypes.c_int, [_VP, _VP, ctypes.c_uint8]),
    "fls_pack_u16": (ctypes.c_int, [_VP, _VP, ctypes.c_uint8]),
    "fls_pack_u64": (ctypes.c_int, [_VP, _VP, ctypes.c_uint8]),
    "fls_unpack_u8": (ctypes.c_int, [_VP, _VP, ctypes.c_uint8]),
    "fls_unpack_u16": (ctypes.c_int, [_VP, _VP, ctypes.c_uint8]),
    "fls_unpack_u64": (ctypes.c_int, [_VP, _VP, ctypes.c_uint8]),
    "fls_pack_column": (ctypes.c_int, [_VP, ctypes.c_uint64, ctypes.c_uint32, ctypes.c_uint8, ctypes.c_uint64, _VP]),
    "fls_decode_u8": (ctypes.c_int, [_VP, ctypes.c_uint64, ctypes.c_uint8, ctypes.c_uint8, _VP, _VP, _VP]),
    "fls_decode_u16": (ctypes.c_int, [_VP, ctypes.c_uint64, ctypes.c_uint8, ctypes.c_uint16, _VP, _VP, _VP]),
    "fls_decode_u64": (ctypes.c_int, [_VP, ctypes.c_uint64, ctypes.c_uint8, ctypes.c_uint64, _VP, _VP, _VP]),
    "fls_column_container_bytes": (ctypes.c_uint64, [ctypes.POINTER(Column)]),
    "fls_column_write_container": (ctypes.c_int, [ctypes.POINTER(Column), _VP, ctypes.c_uint64, _VP]),
    "fls_column_open_container": (ctypes.c_int, [_VP, ctypes.c_uint64, ctypes.POINTER(Column)]),
    "fls_encode_learned_workspace_bytes": (ctypes.c_uint64, [ctypes.c_uint64]),
    "fls_encode_learned_gpu": (ctypes.c_int, [_VP, ctypes.c_uint64, _VP, ctypes.c_float, ctypes.c_double,
                                              ctypes.c_uint32, _VP, ctypes.c_uint64, _VP, _VP, _VP, _VP,
                                              ctypes.c_uint64, _VP]),
    "fls_get_jit_stats": (ctypes.c_int, [ctypes.POINTER(JitStats)]),
    "fls_jit_last_log": (ctypes.c_char_p, []),
    "fls_jit_precompile": (ctypes.c_int, [ctypes.POINTER(FilterAggDesc)]),
    "fls_jit_precompile_probe": (ctypes.c_int, [ctypes.POINTER(JoinAggDesc)]),
    "fls_jit_precompile_join": (ctypes.c_int, [ctypes.POINTER(JoinGroupbyDesc)]),
    "fls_query_join_groupby": (ctypes.c_int, [ctypes.POINTER(JoinGroupbyDesc), _VP, _VP]),
    "fls_query_join_groupby_ws": (ctypes.c_int, [ctypes.POINTER(JoinGroupbyDesc), _VP, _VP, ctypes.c_uint64, _VP]),
    "fls_join_workspace_bytes": (ctypes.c_uint64, [ctypes.POINTER(JoinGroupbyDesc)]),
    "fls_rfor_bound_words": (ctypes.c_uint64, [ctypes.c_uint64]),
    "fls_rfor_encode": (ctypes.c_int, [_VP, ctypes.c_uint64, _VP, _VP, _VP, _VP, _VP, _VP]),
    "fls_rfor_decode_u32": (ctypes.c_int, [ctypes.POINTER(RforColumnDesc), _VP, _VP]),
    "fls_rfor_decode_sum_u32": (ctypes.c_int, [ctypes.POINTER(RforColumnDesc), _VP, _VP]),
}

_LIB = None


def lib() -> ctypes.CDLL:
    """The loaded library (raises if it has not been built)."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise FlsError(9, "load", f"{LIB_PATH} is not built; run python -m fastlanesgpu_b200.build")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _LIB = L
    return _LIB


def check(status: int, where: str) -> None:
    if status != FLS_OK:
        raise FlsError(status, where, (lib().fls_last_error() or b"").decode())


def declared_symbols() -> list[str]:
    return list(_SIGS)
