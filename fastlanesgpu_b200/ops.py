"""Operators of the B200 FastLanes library (Python face of include/fls_gpu.h).

Every call enqueues CUDA work on the current torch stream and returns device
tensors; nothing here computes on the CPU.  Names follow the reference's
operators:

=============================  ==============================================
this module                    reference (FastLanesGPU)
=============================  ==============================================
``pack`` / ``transpose_i`` /   fastlanes/src/pack.cpp:29607, transpose.cpp:4110,
``unrsum`` / ``vector_rle``    unrsum.cpp:120, fls_gen/rle/rle.hpp:29 (host)
``unpack_global``              fls_gen/unpack/unpack.cuh:3436 and
                               delta_global_memory.cu:24 (decode to HBM)
``query_aggregate``            bitpack_shared_memory.cu:21 QueryKernel (decode+sum)
``query_filter_agg``           ssb/fls_q11.cu:29 QueryKernel_v1
``build_pht``                  ssb/fls_q21.cu:197-263 build_hashtable_{s,p,d}
``probe_groupby``              ssb/fls_q21.cu:21 probe_v1
=============================  ==============================================
"""
from __future__ import annotations

import ctypes

import numpy as np

from ._lib import (MAX_FILTERS, MAX_GROUP_KEYS, MAX_PROBES, ORDER_STORED, Column, FilterAggDesc, JitStats, JoinAggDesc,
                   JoinGroupbyDesc, check, lib)
from .column import DeviceColumn, columns_array


def _stream():
    import torch
    return torch.cuda.current_stream().cuda_stream


def _p(a: np.ndarray) -> int:
    return a.ctypes.data


# ---------------------------------------------------------------- host side

def pack(vec: np.ndarray, bw: int) -> np.ndarray:
    """FastLanes 32-bit bit-packing of one 1024-value vector (32*bw words)."""
    v = np.ascontiguousarray(vec, dtype=np.uint32)
    assert v.size == 1024
    out = np.zeros(max(32 * bw, 1), dtype=np.uint32)
    check(lib().fls_pack_u32(_p(v), _p(out), bw), "fls_pack_u32")
    return out[:32 * bw]


def transpose_i(vec: np.ndarray) -> np.ndarray:
    v = np.ascontiguousarray(vec, dtype=np.uint32)
    out = np.empty(1024, dtype=np.uint32)
    check(lib().fls_transpose_i_u32(_p(v), _p(out)), "fls_transpose_i_u32")
    return out


def untranspose(vec: np.ndarray) -> np.ndarray:
    v = np.ascontiguousarray(vec, dtype=np.uint32)
    out = np.empty(1024, dtype=np.uint32)
    check(lib().fls_untranspose_u32(_p(v), _p(out)), "fls_untranspose_u32")
    return out


def unrsum(vec: np.ndarray) -> np.ndarray:
    v = np.ascontiguousarray(vec, dtype=np.uint32)
    out = np.empty(1024, dtype=np.uint32)
    check(lib().fls_unrsum_u32(_p(v), _p(out)), "fls_unrsum_u32")
    return out


def vector_rle(vec: np.ndarray):
    """rle.hpp VECTOR_RLE: (n_dict, idx[1024] uint8, dict[n_dict], dict4[4])."""
    v = np.ascontiguousarray(vec, dtype=np.int32)
    idx = np.zeros(1024, np.uint8)
    dic = np.zeros(1024, np.int32)
    d4 = np.zeros(4, np.uint16)
    n = ctypes.c_uint32()
    check(lib().fls_vector_rle(_p(v), _p(idx), _p(dic), _p(d4), ctypes.addressof(n)), "fls_vector_rle")
    return n.value, idx, dic[:n.value].copy(), d4


def encode_exhaustive(values: np.ndarray, n_threads: int = 0):
    """Exact per-vector sizes of all 5 schemes and the argmin (n_vec x 5, n_vec)."""
    v = np.ascontiguousarray(values, dtype=np.int32)
    nv = (v.size + 1023) // 1024
    sizes = np.zeros((nv, 5), np.uint32)
    best = np.zeros(nv, np.uint8)
    check(lib().fls_encode_exhaustive(_p(v), v.size, _p(sizes), _p(best), n_threads), "fls_encode_exhaustive")
    return sizes, best


def vector_stats(values: np.ndarray, n_threads: int = 0) -> np.ndarray:
    v = np.ascontiguousarray(values, dtype=np.int32)
    nv = (v.size + 1023) // 1024
    out = np.zeros((nv, 16), np.float32)
    check(lib().fls_vector_stats(_p(v), v.size, _p(out), n_threads), "fls_vector_stats")
    return out


# -------------------------------------------------------------- device side

def unpack_global(col: DeviceColumn, order: int = ORDER_STORED, out=None):
    """Decode every vector to HBM (n_vec*1024 int32 values, device)."""
    import torch
    if out is None:
        out = torch.empty(col.n_vec * 1024, dtype=torch.int32, device=col.data.device)
    check(lib().fls_decode_u32(ctypes.byref(col.desc), out.data_ptr(), order, _stream()), "fls_decode_u32")
    return out


def query_aggregate(col: DeviceColumn, out=None):
    """Decode fused with a uint64 sum of all values (device int64[1])."""
    import torch
    if out is None:
        out = torch.empty(1, dtype=torch.int64, device=col.data.device)
    check(lib().fls_decode_sum_u32(ctypes.byref(col.desc), out.data_ptr(), _stream()), "fls_decode_sum_u32")
    return out


def rfor_decode(col, out=None):
    """Decode an RFOR column (DeviceRforColumn) to n_values int32 values (device)."""
    import torch
    if out is None:
        out = torch.empty(col.n_values, dtype=torch.int32, device=col.values.device)
    check(lib().fls_rfor_decode_u32(ctypes.byref(col.desc), out.data_ptr(), _stream()), "fls_rfor_decode_u32")
    return out


def rfor_decode_sum(col, out=None):
    """RFOR decode fused with a uint64 sum of all values (device int64[1])."""
    import torch
    if out is None:
        out = torch.empty(1, dtype=torch.int64, device=col.values.device)
    check(lib().fls_rfor_decode_sum_u32(ctypes.byref(col.desc), out.data_ptr(), _stream()), "fls_rfor_decode_sum_u32")
    return out


def query_filter_agg(cols, filters, agg_a: int = -1, agg_b: int = -1, out=None):
    """Filters [(col, lo, hi)] (inclusive int32 ranges) ANDed; returns the int64
    sum of cols[agg_a] (* cols[agg_b]) over the selected rows, or the count."""
    import torch
    d, _keep = _filter_agg_desc(columns_array(cols), len(cols), filters, agg_a, agg_b)
    if out is None:
        out = torch.empty(1, dtype=torch.int64, device=cols[0].data.device)
    check(lib().fls_query_filter_agg(ctypes.byref(d), out.data_ptr(), _stream()), "fls_query_filter_agg")
    return out


def _filter_agg_desc(arr, n_cols: int, filters, agg_a: int, agg_b: int):
    if len(filters) > MAX_FILTERS:
        raise ValueError("at most 4 filters")
    d = FilterAggDesc()
    d.cols = arr
    d.n_cols = n_cols
    for i, (c, lo, hi) in enumerate(filters):
        d.filters[i].col, d.filters[i].lo, d.filters[i].hi = c, lo, hi
    d.n_filters = len(filters)
    d.agg_a, d.agg_b = agg_a, agg_b
    return d, arr


def jit_precompile(col_descs, filters, agg_a: int = -1, agg_b: int = -1) -> None:
    """Compiles the specialised filter-aggregate kernel for this query shape
    (column descriptors: `Column` structs, or DeviceColumns).  Needs no GPU."""
    descs = [c.desc if hasattr(c, "desc") else c for c in col_descs]
    arr = (Column * len(descs))(*descs)
    d, _keep = _filter_agg_desc(arr, len(descs), filters, agg_a, agg_b)
    check(lib().fls_jit_precompile(ctypes.byref(d)), "fls_jit_precompile")


def jit_stats() -> dict:
    """Counters of the specialised-kernel cache."""
    s = JitStats()
    check(lib().fls_get_jit_stats(ctypes.byref(s)), "fls_get_jit_stats")
    return {"compiled": s.compiled, "launches": s.launches, "failures": s.failures, "cached": s.cached}


def jit_last_log() -> str:
    return (lib().fls_jit_last_log() or b"").decode(errors="replace")


def build_pht(keys, ht_len: int, vals=None, filt=None, filter_eq: int = 1, keys_min: int = 0, out=None,
              ranges=None):
    """Selective perfect-hash table on device int32 columns: PHT_1 (vals None,
    ht_len slots) or PHT_2 (2*ht_len slots).  Rows with filt == filter_eq, or,
    with ranges=[(lo, hi)] (one or two inclusive ranges), rows whose filt lies
    in one of them."""
    import torch
    size = ht_len if vals is None else 2 * ht_len
    if out is None:
        out = torch.zeros(size, dtype=torch.int32, device=keys.device)
    else:
        out.zero_()
    if ranges is None:
        ranges = [(filter_eq, filter_eq)]
    if not 1 <= len(ranges) <= 2:
        raise ValueError("one or two filter ranges")
    (lo0, hi0), (lo1, hi1) = ranges[0], ranges[1] if len(ranges) == 2 else (1, 0)
    check(lib().fls_pht_build_ranges(0 if filt is None else filt.data_ptr(), lo0, hi0, lo1, hi1, keys.data_ptr(),
                                     0 if vals is None else vals.data_ptr(), keys.numel(), out.data_ptr(), ht_len,
                                     keys_min, _stream()), "fls_pht_build_ranges")
    return out


def _join_workspace(workspace, n_bytes: int, device):
    """(pointer, bytes, tensor kept alive) of a join call's workspace:
    "auto" allocates the bytes the call asks for, None passes none (the
    kernels then build their shared-memory bitmaps per CTA), a uint8 device
    tensor is used as given."""
    import torch
    if workspace is None or (isinstance(workspace, str) and n_bytes == 0):
        return None, 0, None
    if isinstance(workspace, str):
        if workspace != "auto":
            raise ValueError("workspace must be 'auto', None or a device tensor")
        workspace = torch.empty(n_bytes, dtype=torch.uint8, device=device)
    return workspace.data_ptr(), workspace.numel() * workspace.element_size(), workspace


def probe_groupby(cols, probes, agg_col: int, key_a: int, key_b: int, group_mul: int, group_sub: int,
                  n_groups: int, out=None, workspace="auto"):
    """probes: [(col, ht tensor, ht_len, keys_min, kind)].  Returns the
    reference's result array int32[4*n_groups]: [key_b value, key_a value,
    int64 sum (2 words)] per group."""
    import torch
    d, _keep = _join_desc(columns_array(cols), len(cols), probes, agg_col, key_a, key_b, group_mul, group_sub,
                          n_groups)
    if out is None:
        out = torch.empty(4 * n_groups, dtype=torch.int32, device=cols[0].data.device)
    n_ws = int(lib().fls_probe_workspace_bytes(ctypes.byref(d))) if workspace is not None else 0
    ws, ws_bytes, _ws = _join_workspace(workspace, n_ws, out.device)
    check(lib().fls_query_probe_groupby_ws(ctypes.byref(d), out.data_ptr(), ws, ws_bytes, _stream()),
          "fls_query_probe_groupby")
    return out


def _join_desc(arr, n_cols: int, probes, agg_col, key_a, key_b, group_mul, group_sub, n_groups):
    if len(probes) > MAX_PROBES:
        raise ValueError("at most 4 probes")
    d = JoinAggDesc()
    d.cols = arr
    d.n_cols = n_cols
    for i, (c, ht, ln, kmin, kind) in enumerate(probes):
        d.probes[i].col, d.probes[i].ht_len = c, ln
        d.probes[i].ht = ht if isinstance(ht, int) else ht.data_ptr()
        d.probes[i].keys_min, d.probes[i].kind = kmin, kind
    d.n_probes = len(probes)
    d.agg_col, d.key_a, d.key_b = agg_col, key_a, key_b
    d.group_mul, d.group_sub, d.n_groups = group_mul, group_sub, n_groups
    return d, arr


def _groupby_desc(arr, n_cols: int, probes, agg_col, keys, group_sub, n_groups, res_stride, sum_slot, agg_sub_col,
                  sum_bits=64):
    if len(probes) > MAX_PROBES or not 1 <= len(keys) <= MAX_GROUP_KEYS:
        raise ValueError("1..4 probes and 1..3 group keys")
    d = JoinGroupbyDesc()
    d.cols = arr
    d.n_cols = n_cols
    for i, (c, ht, ln, kmin, kind) in enumerate(probes):
        d.probes[i].col, d.probes[i].ht_len = c, ln
        d.probes[i].ht = ht if isinstance(ht, int) else ht.data_ptr()
        d.probes[i].keys_min, d.probes[i].kind = kmin, kind
    d.n_probes = len(probes)
    d.agg_col, d.agg_sub_col = agg_col, agg_sub_col
    d.n_keys = len(keys)
    for k, (probe, mul, slot) in enumerate(keys):
        d.key_probe[k], d.key_mul[k], d.key_slot[k] = probe, mul, slot
    d.group_sub, d.n_groups, d.res_stride, d.sum_slot = group_sub, n_groups, res_stride, sum_slot
    d.sum_bits = sum_bits
    return d, arr


def join_groupby(cols, probes, agg_col: int, keys, group_sub: int, n_groups: int, res_stride: int, sum_slot: int,
                 agg_sub_col: int = -1, out=None, workspace="auto", sum_bits: int = 64):
    """The general probe + group-by (fls_q21/q31/q41.cu probe_v1): probes
    [(col, ht, ht_len, keys_min, kind)]; keys [(probe, multiplier, record word
    or -1)]; group = (sum of payload * multiplier - group_sub) % n_groups;
    records of res_stride int32 words with the int64 sum of cols[agg_col]
    (minus cols[agg_sub_col]) at word sum_slot (sum_bits 32: a wrapping int32
    sum in that one word).  Returns the device int32 array."""
    import torch
    d, _keep = _groupby_desc(columns_array(cols), len(cols), probes, agg_col, keys, group_sub, n_groups, res_stride,
                             sum_slot, agg_sub_col, sum_bits)
    if out is None:
        out = torch.empty(res_stride * n_groups, dtype=torch.int32, device=cols[0].data.device)
    n_ws = int(lib().fls_join_workspace_bytes(ctypes.byref(d))) if workspace is not None else 0
    ws, ws_bytes, _ws = _join_workspace(workspace, n_ws, out.device)
    check(lib().fls_query_join_groupby_ws(ctypes.byref(d), out.data_ptr(), ws, ws_bytes, _stream()),
          "fls_query_join_groupby")
    return out


def jit_precompile_join(col_descs, probes, agg_col, keys, group_sub, n_groups, res_stride, sum_slot,
                        agg_sub_col: int = -1, sum_bits: int = 64) -> None:
    """Compiles the specialised join + group-by kernel for this query shape."""
    descs = [c.desc if hasattr(c, "desc") else c for c in col_descs]
    arr = (Column * len(descs))(*descs)
    d, _keep = _groupby_desc(arr, len(descs), probes, agg_col, keys, group_sub, n_groups, res_stride, sum_slot,
                             agg_sub_col, sum_bits)
    check(lib().fls_jit_precompile_join(ctypes.byref(d)), "fls_jit_precompile_join")


def join_workspace_bytes(col_descs, probes, agg_col, keys, group_sub, n_groups, res_stride, sum_slot,
                         agg_sub_col: int = -1, sum_bits: int = 64) -> int:
    """Bytes of device workspace join_groupby can use for this query (0: none);
    needs no GPU."""
    descs = [c.desc if hasattr(c, "desc") else c for c in col_descs]
    arr = (Column * len(descs))(*descs)
    d, _keep = _groupby_desc(arr, len(descs), probes, agg_col, keys, group_sub, n_groups, res_stride, sum_slot,
                             agg_sub_col, sum_bits)
    return int(lib().fls_join_workspace_bytes(ctypes.byref(d)))


def jit_precompile_probe(col_descs, probes, agg_col: int, key_a: int, key_b: int, group_mul: int, group_sub: int,
                         n_groups: int) -> None:
    """Compiles the specialised probe + group-by kernel for this query shape
    (probe tables may be given as integer addresses).  Needs no GPU."""
    descs = [c.desc if hasattr(c, "desc") else c for c in col_descs]
    arr = (Column * len(descs))(*descs)
    d, _keep = _join_desc(arr, len(descs), probes, agg_col, key_a, key_b, group_mul, group_sub, n_groups)
    check(lib().fls_jit_precompile_probe(ctypes.byref(d)), "fls_jit_precompile_probe")


def crystal_q11(cols, n_rows: int, date_gt: int, date_lt: int, qty_lt: int, disc_ge: int, disc_le: int, out=None):
    """fls_q11.cu QueryKernel_v1 on the drop-in primitive API.  cols: uniform
    DeviceColumns (date, discount, quantity, price)."""
    import torch
    if out is None:
        out = torch.empty(1, dtype=torch.int64, device=cols[0].data.device)
    args = []
    for c in cols:
        args += [c.data.data_ptr(), c.host.bw]
    check(lib().fls_crystal_q11(*args, n_rows, date_gt, date_lt, qty_lt, disc_ge, disc_le, out.data_ptr(),
                                _stream()), "fls_crystal_q11")
    return out


def crystal_q21_probe(cols, n_rows: int, ht_s, ht_p, ht_d, d_keys_min: int = 0, out=None):
    """fls_q21.cu probe_v1 on the drop-in primitive API.  cols: uniform
    DeviceColumns (suppkey, partkey, orderdate, revenue)."""
    import torch
    if out is None:
        out = torch.empty(4 * 7000, dtype=torch.int32, device=cols[0].data.device)
    args = []
    for c in cols:
        args += [c.data.data_ptr(), c.host.bw]
    check(lib().fls_crystal_q21_probe(*args, n_rows, ht_s.data_ptr(), ht_s.numel(), ht_p.data_ptr(), ht_p.numel() // 2,
                                      ht_d.data_ptr(), ht_d.numel() // 2, d_keys_min, out.data_ptr(), _stream()),
          "fls_crystal_q21_probe")
    return out


def check_device_error(stream=None) -> None:
    """Take the error bits of `stream` (default: the current stream) and raise
    if a kernel launched on it flagged bad input or a timeout."""
    st = _stream() if stream is None else stream.cuda_stream
    check(lib().fls_check_device_error(st), "device")


def bind_error_word(words, stream=None) -> None:
    """Give `stream` (default: the current stream) its own error word: `words`
    is a zeroed device tensor of two int32 (None removes the binding)."""
    st = _stream() if stream is None else stream.cuda_stream
    if words is not None:
        assert words.is_cuda and words.numel() * words.element_size() >= 8
    check(lib().fls_bind_error_word(st, None if words is None else words.data_ptr()), "fls_bind_error_word")


def set_launch_config(warps: int = 0, stages: int = 0, ctas_per_sm: int = 0, tile_bytes: int = 0) -> None:
    """0 keeps the library default of that field."""
    check(lib().fls_set_launch_config(warps, stages, ctas_per_sm, tile_bytes), "fls_set_launch_config")


def get_launch_config():
    w, s, c, t = ctypes.c_uint32(), ctypes.c_uint32(), ctypes.c_uint32(), ctypes.c_uint32()
    lib().fls_get_launch_config(ctypes.addressof(w), ctypes.addressof(s), ctypes.addressof(c), ctypes.addressof(t))
    return w.value, s.value, c.value, t.value


def set_tuning(param: int, value: int) -> None:
    check(lib().fls_set_tuning(param, value), "fls_set_tuning")


def get_tuning(param: int) -> int:
    v = ctypes.c_int64()
    check(lib().fls_get_tuning(param, ctypes.addressof(v)), "fls_get_tuning")
    return v.value


def kernel_launch_count() -> int:
    return int(lib().fls_kernel_launch_count())


# ------------------------------------------------- 8/16/64-bit lane widths

_WIDTH_DTYPES = {8: np.uint8, 16: np.uint16, 32: np.uint32, 64: np.uint64}


def pack_vector(values: np.ndarray, bw: int) -> np.ndarray:
    """FastLanes packing of one vector of 1024 uint8/uint16/uint64 values
    (fls_pack_u8/u16/u64): (1024/T)*bw words of the values' type."""
    v = np.ascontiguousarray(values)
    bits = v.dtype.itemsize * 8
    assert v.size == 1024 and bits in (8, 16, 64)
    out = np.zeros(1024 // bits * bw + 1, dtype=v.dtype)
    check(getattr(lib(), f"fls_pack_u{bits}")(v.ctypes.data, out.ctypes.data, bw), f"fls_pack_u{bits}")
    return out[: 1024 // bits * bw]


def unpack_vector(packed: np.ndarray, bw: int) -> np.ndarray:
    p = np.ascontiguousarray(packed)
    bits = p.dtype.itemsize * 8
    src = np.concatenate([p, np.zeros(1, p.dtype)])
    out = np.zeros(1024, dtype=p.dtype)
    check(getattr(lib(), f"fls_unpack_u{bits}")(src.ctypes.data, out.ctypes.data, bw), f"fls_unpack_u{bits}")
    return out


def pack_column_width(values: np.ndarray, bw: int, base: int = 0) -> np.ndarray:
    """A column of uint8/uint16/uint32/uint64 values minus `base`, packed
    vector after vector (fls_pack_column); returns the packed words."""
    v = np.ascontiguousarray(values)
    bits = v.dtype.itemsize * 8
    n_vec = (v.size + 1023) // 1024
    out = np.zeros(n_vec * 1024 // bits * bw + 16 // v.dtype.itemsize, dtype=v.dtype)
    check(lib().fls_pack_column(v.ctypes.data, v.size, bits, bw, base & ((1 << bits) - 1), out.ctypes.data),
          "fls_pack_column")
    return out


def decode_width_into(packed, n: int, bits: int, bw: int, base: int, out=None, sum_out=None) -> None:
    """Stream-ordered form of decode_width: writes into `out` (device tensor of
    the width's values, or None) and `sum_out` (device int64[1], or None)."""
    check(getattr(lib(), f"fls_decode_u{bits}")(packed.data_ptr(), n, bw, base & ((1 << bits) - 1),
                                               None if out is None else out.data_ptr(),
                                               None if sum_out is None else sum_out.data_ptr(), _stream()),
          f"fls_decode_u{bits}")


def decode_width(packed, n: int, bits: int, bw: int, base: int = 0, out=None, want_sum: bool = True):
    """GPU decode of a packed 8/16/64-bit column (fls_decode_u8/u16/u64):
    packed is a 16-byte aligned device tensor of the packed bytes.  Returns
    (decoded values tensor of the width's torch dtype or None, uint64 sum as
    a Python int or None)."""
    import torch
    n_vec = (n + 1023) // 1024
    tdt = {8: torch.uint8, 16: torch.int16, 64: torch.int64}[bits]
    if out is None:
        out = torch.empty(n_vec * 1024, dtype=tdt, device=packed.device)
    s = torch.zeros(1, dtype=torch.int64, device=packed.device) if want_sum else None
    check(getattr(lib(), f"fls_decode_u{bits}")(packed.data_ptr(), n, bw, base & ((1 << bits) - 1),
                                               None if out is False else out.data_ptr(),
                                               None if s is None else s.data_ptr(), _stream()),
          f"fls_decode_u{bits}")
    total = None if s is None else int(s.cpu()[0]) & 0xFFFFFFFFFFFFFFFF
    return (None if out is False else out), total


def selftest_bounded_wait(polls: int = 64) -> None:
    """Runs the pipelines' bounded device wait on a barrier nothing arrives
    on (fls_selftest_bounded_wait); the next check_device_error raises
    FLS_ERR_TIMEOUT."""
    check(lib().fls_selftest_bounded_wait(polls, _stream()), "fls_selftest_bounded_wait")
