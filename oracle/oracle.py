"""TEST INFRASTRUCTURE ONLY: ctypes access to the CPU oracle and to the
reference's own code built from its sources.

* ``Oracle`` wraps ``oracle/liboracle.so`` (the C restatement, fls_oracle.c).
* ``Reference`` wraps ``oracle/_ref/libflsref.so`` (pack.cpp, transpose.cpp,
  unrsum.cpp, unpack.cuh, unpack_fused.cuh, hardcoded_16.cuh, rsum.cuh, rle.hpp
  and the query loops of fls_q11.cu / fls_q21.cu, compiled by oracle/Makefile).

Only tests/, the smoke entry point and bench.py's CPU-baseline / reference
legs import this module; the library itself never does.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libflsref.so")

FOR, DELTA, RLE, CONST, DICT = 0, 1, 2, 3, 4
N_GROUPS = 7000

_u32p = ctypes.POINTER(ctypes.c_uint32)
_i32p = ctypes.POINTER(ctypes.c_int32)
_u16p = ctypes.POINTER(ctypes.c_uint16)
_u8p = ctypes.POINTER(ctypes.c_uint8)


def _p(a, t):
    return a.ctypes.data_as(t)


def build(with_reference: bool = True) -> None:
    """Compile the oracle (and, when its sources are present, the reference)."""
    target = "all" if with_reference else "oracle"
    subprocess.run(["make", "-s", "-C", HERE, target], check=True)


class OrcProbe(ctypes.Structure):
    _fields_ = [("col", _i32p), ("ht", _i32p), ("len", ctypes.c_int32), ("keys_min", ctypes.c_int32),
                ("kind", ctypes.c_int32)]


class OrcVec(ctypes.Structure):
    _fields_ = [("scheme", ctypes.c_uint32), ("bw", ctypes.c_uint32), ("aux", ctypes.c_uint32),
                ("n_words", ctypes.c_uint32), ("base", ctypes.c_int32)]


class Oracle:
    def __init__(self, path: str = ORACLE_SO):
        if not os.path.exists(path):
            build(with_reference=False)
        L = ctypes.CDLL(path)
        self.L = L
        L.orc_tpos.restype = ctypes.c_uint32
        L.orc_bit_width.restype = ctypes.c_uint
        L.orc_vector_rle.restype = ctypes.c_int
        L.orc_encode_vec.restype = ctypes.c_int
        L.orc_rfor_bound.restype = ctypes.c_uint64
        L.orc_rfor_bound.argtypes = [ctypes.c_uint64]
        L.orc_rfor_encode.argtypes = [_u32p, ctypes.c_uint64] + [_u32p] * 4 + [ctypes.c_void_p] * 2
        L.orc_rfor_decode.argtypes = [_u32p] * 4 + [ctypes.c_uint64, _u32p]
        L.orc_filter_agg.restype = ctypes.c_int64
        L.orc_filter_agg.argtypes = [_i32p, _i32p, _i32p, _i32p, ctypes.c_uint64] + [ctypes.c_int32] * 5
        L.orc_pht1_build.argtypes = [_i32p, ctypes.c_int32, _i32p, ctypes.c_uint64, _i32p, ctypes.c_int32,
                                     ctypes.c_int32]
        L.orc_pht2_build.argtypes = [_i32p, ctypes.c_int32, _i32p, _i32p, ctypes.c_uint64, _i32p, ctypes.c_int32,
                                     ctypes.c_int32]
        L.orc_probe_groupby.argtypes = [_i32p, _i32p, _i32p, _i32p, ctypes.c_uint64, _i32p, ctypes.c_int32, _i32p,
                                        ctypes.c_int32, _i32p, ctypes.c_int32, ctypes.c_int32, _i32p]
        L.orc_q31_groupby.argtypes = ([_i32p] * 4 + [ctypes.c_uint64] + [_i32p, ctypes.c_int32] * 3
                                      + [ctypes.c_int32, _i32p])
        L.orc_q41_groupby.argtypes = ([_i32p] * 6 + [ctypes.c_uint64] + [_i32p, ctypes.c_int32] * 4
                                      + [ctypes.c_int32, _i32p])
        L.orc_pht_build_ranges.argtypes = ([_i32p] + [ctypes.c_int32] * 4 + [_i32p, _i32p, ctypes.c_uint64, _i32p]
                                           + [ctypes.c_int32] * 2)
        L.orc_join_groupby.argtypes = [ctypes.c_uint64, ctypes.POINTER(OrcProbe), ctypes.c_uint32, _i32p, _i32p,
                                       ctypes.c_uint32, _i32p, _i32p, _i32p, ctypes.c_int32, ctypes.c_int32,
                                       ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32, _i32p]

    # -- layout / packing -------------------------------------------------
    def tpos(self) -> np.ndarray:
        return np.array([self.L.orc_tpos(j) for j in range(1024)], dtype=np.int64)

    def pack(self, vec: np.ndarray, bw: int) -> np.ndarray:
        vec = np.ascontiguousarray(vec, dtype=np.uint32)
        out = np.zeros(32 * bw, dtype=np.uint32)
        self.L.orc_pack(_p(vec, _u32p), _p(out, _u32p), ctypes.c_uint(bw))
        return out

    def unpack(self, packed: np.ndarray, bw: int) -> np.ndarray:
        packed = np.ascontiguousarray(packed, dtype=np.uint32)
        out = np.zeros(1024, dtype=np.uint32)
        self.L.orc_unpack(_p(packed, _u32p), _p(out, _u32p), ctypes.c_uint(bw))
        return out

    def unpack_quarter(self, packed_q: np.ndarray, bw: int) -> np.ndarray:
        packed_q = np.ascontiguousarray(packed_q, dtype=np.uint32)
        out = np.zeros(256, dtype=np.uint32)
        self.L.orc_unpack_quarter(_p(packed_q, _u32p), _p(out, _u32p), ctypes.c_uint(bw))
        return out

    def transpose_i(self, vec):
        vec = np.ascontiguousarray(vec, dtype=np.uint32)
        out = np.zeros(1024, dtype=np.uint32)
        self.L.orc_transpose_i(_p(vec, _u32p), _p(out, _u32p))
        return out

    def untranspose(self, vec):
        vec = np.ascontiguousarray(vec, dtype=np.uint32)
        out = np.zeros(1024, dtype=np.uint32)
        self.L.orc_untranspose(_p(vec, _u32p), _p(out, _u32p))
        return out

    def unrsum(self, vec):
        vec = np.ascontiguousarray(vec, dtype=np.uint32)
        out = np.zeros(1024, dtype=np.uint32)
        self.L.orc_unrsum(_p(vec, _u32p), _p(out, _u32p))
        return out

    def rsum(self, deltas, base):
        deltas = np.ascontiguousarray(deltas, dtype=np.uint32)
        base = np.ascontiguousarray(base, dtype=np.uint32)
        out = np.zeros(1024, dtype=np.uint32)
        self.L.orc_rsum(_p(deltas, _u32p), _p(out, _u32p), _p(base, _u32p))
        return out

    def vector_rle(self, vec):
        vec = np.ascontiguousarray(vec, dtype=np.int32)
        idx = np.zeros(1024, np.uint8)
        dic = np.zeros(1024, np.int32)
        d4 = np.zeros(4, np.uint16)
        n = self.L.orc_vector_rle(_p(vec, _i32p), _p(idx, _u8p), _p(dic, _i32p), _p(d4, _u16p))
        return n, idx, dic[:n].copy(), d4

    # -- tile-based RLE (RFOR) --------------------------------------------
    def rfor_encode(self, values):
        """tile_based/src/rlebinpack.cpp:9-146 on values padded to whole tiles
        with the last value: (value stream, run-length stream, val_offsets,
        rl_offsets)."""
        v = np.ascontiguousarray(values).view(np.uint32)
        n = (v.size + 511) // 512 * 512
        x = np.concatenate([v, np.full(n - v.size, v[-1], np.uint32)])
        bound = int(self.L.orc_rfor_bound(n))
        val, rl = np.zeros(bound, np.uint32), np.zeros(bound, np.uint32)
        vo, ro = np.zeros(n // 512 + 1, np.uint32), np.zeros(n // 512 + 1, np.uint32)
        nv, nr = ctypes.c_uint64(), ctypes.c_uint64()
        self.L.orc_rfor_encode(_p(x, _u32p), n, _p(val, _u32p), _p(rl, _u32p), _p(vo, _u32p), _p(ro, _u32p),
                               ctypes.byref(nv), ctypes.byref(nr))
        return val[:nv.value].copy(), rl[:nr.value].copy(), vo, ro

    def rfor_decode(self, val, rl, vo, ro, n):
        out = np.zeros(n, np.uint32)
        rc = self.L.orc_rfor_decode(_p(val, _u32p), _p(rl, _u32p), _p(vo, _u32p), _p(ro, _u32p), n, _p(out, _u32p))
        return None if rc != 0 else out

    # -- encoded vectors ---------------------------------------------------
    def encode_vec(self, vec, scheme: int, transposed: bool = True, round4: bool = False):
        vec = np.ascontiguousarray(vec, dtype=np.int32)
        out = np.zeros(2048, dtype=np.uint32)
        m = OrcVec()
        rc = self.L.orc_encode_vec(_p(vec, _i32p), ctypes.c_uint32(scheme), ctypes.c_int(int(transposed)),
                                   ctypes.c_int(int(round4)), _p(out, _u32p), ctypes.byref(m))
        if rc != 0:
            return None, None
        return out[:m.n_words].copy(), m

    def decode_vec(self, payload, meta: OrcVec, transposed: bool = True) -> np.ndarray:
        buf = np.zeros(max(2048, payload.size + 4), dtype=np.uint32)
        buf[:payload.size] = payload
        out = np.zeros(1024, dtype=np.int32)
        self.L.orc_decode_vec(_p(buf, _u32p), ctypes.byref(meta), ctypes.c_int(int(transposed)), _p(out, _i32p))
        return out

    def scheme_sizes(self, vec) -> np.ndarray:
        vec = np.ascontiguousarray(vec, dtype=np.int32)
        out = np.zeros(5, np.uint32)
        self.L.orc_scheme_sizes(_p(vec, _i32p), _p(out, _u32p))
        return out

    def vector_stats(self, vec) -> np.ndarray:
        vec = np.ascontiguousarray(vec, dtype=np.int32)
        out = np.zeros(16, np.float32)
        self.L.orc_vector_stats(_p(vec, _i32p), out.ctypes.data_as(ctypes.POINTER(ctypes.c_float)))
        return out

    def mlp_loss_grad(self, params, x, y):
        params = np.ascontiguousarray(params, np.float32)
        x = np.ascontiguousarray(x, np.float32)
        y = np.ascontiguousarray(y, np.uint8)
        g = np.zeros(5573, np.float64)
        fp = ctypes.POINTER(ctypes.c_float)
        self.L.orc_mlp_loss_grad.restype = ctypes.c_double
        loss = self.L.orc_mlp_loss_grad(params.ctypes.data_as(fp), x.ctypes.data_as(fp), _p(y, _u8p),
                                        ctypes.c_uint32(y.size), g.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
        return float(loss), g

    # -- query path ----------------------------------------------------------
    def filter_agg(self, date, disc, qty, price, date_lo, date_hi, disc_lo, disc_hi, qty_lt) -> int:
        cols = [np.ascontiguousarray(c, dtype=np.int32) for c in (date, disc, qty, price)]
        return int(self.L.orc_filter_agg(*[_p(c, _i32p) for c in cols], ctypes.c_uint64(cols[0].size),
                                         date_lo, date_hi, disc_lo, disc_hi, qty_lt))

    def pht1_build(self, filt, eq, keys, length, keys_min=0):
        ht = np.zeros(length, np.int32)
        keys = np.ascontiguousarray(keys, np.int32)
        f = None if filt is None else np.ascontiguousarray(filt, np.int32)
        self.L.orc_pht1_build(None if f is None else _p(f, _i32p), eq, _p(keys, _i32p), keys.size,
                              _p(ht, _i32p), length, keys_min)
        return ht

    def pht2_build(self, filt, eq, keys, vals, length, keys_min=0):
        ht = np.zeros(2 * length, np.int32)
        keys = np.ascontiguousarray(keys, np.int32)
        vals = np.ascontiguousarray(vals, np.int32)
        f = None if filt is None else np.ascontiguousarray(filt, np.int32)
        self.L.orc_pht2_build(None if f is None else _p(f, _i32p), eq, _p(keys, _i32p), _p(vals, _i32p),
                              keys.size, _p(ht, _i32p), length, keys_min)
        return ht

    def probe_groupby(self, supp, part, date, rev, ht_s, ht_p, ht_d, d_keys_min=0):
        cols = [np.ascontiguousarray(c, dtype=np.int32) for c in (supp, part, date, rev)]
        res = np.zeros(4 * N_GROUPS, np.int32)
        self.L.orc_probe_groupby(*[_p(c, _i32p) for c in cols], ctypes.c_uint64(cols[0].size),
                                 _p(ht_s, _i32p), ht_s.size, _p(ht_p, _i32p), ht_p.size // 2,
                                 _p(ht_d, _i32p), ht_d.size // 2, d_keys_min, _p(res, _i32p))
        return res


    def q31_groupby(self, supp, cust, date, rev, ht_s, ht_c, ht_d, d_keys_min=0):
        """fls_q31.cu probe_v1 restated: int32[6 * 4375] group records."""
        cols = [np.ascontiguousarray(c, dtype=np.int32) for c in (supp, cust, date, rev)]
        res = np.zeros(6 * 4375, np.int32)
        self.L.orc_q31_groupby(*[_p(c, _i32p) for c in cols], ctypes.c_uint64(cols[0].size),
                               _p(ht_s, _i32p), ht_s.size // 2, _p(ht_c, _i32p), ht_c.size // 2,
                               _p(ht_d, _i32p), ht_d.size // 2, d_keys_min, _p(res, _i32p))
        return res

    def q41_groupby(self, supp, cust, part, date, rev, cost, ht_s, ht_c, ht_p, ht_d, d_keys_min=0):
        """fls_q41.cu probe_v1 restated: int32[4 * 175] group records."""
        cols = [np.ascontiguousarray(c, dtype=np.int32) for c in (supp, cust, part, date, rev, cost)]
        res = np.zeros(4 * 175, np.int32)
        self.L.orc_q41_groupby(*[_p(c, _i32p) for c in cols], ctypes.c_uint64(cols[0].size),
                               _p(ht_s, _i32p), ht_s.size, _p(ht_c, _i32p), ht_c.size // 2,
                               _p(ht_p, _i32p), ht_p.size, _p(ht_d, _i32p), ht_d.size // 2, d_keys_min,
                               _p(res, _i32p))
        return res


    @staticmethod
    def filter_agg_ranges(cols, filters, agg_a: int, agg_b: int) -> int:
        """crystal-opt src/ssb/q12.cu:68-100 (and q11, q13): rows with
        lo <= cols[c] <= hi for every filter (c, lo, hi), exact int64 sum of
        cols[agg_a] * cols[agg_b] (numpy integer arithmetic)."""
        sel = np.ones(np.asarray(cols[0]).size, bool)
        for c, lo, hi in filters:
            x = np.asarray(cols[c]).astype(np.int64)
            sel &= (x >= lo) & (x <= hi)
        a = np.asarray(cols[agg_a])[sel].astype(np.int64)
        b = np.asarray(cols[agg_b])[sel].astype(np.int64)
        return int((a * b).sum())

    def pht_build_ranges(self, filt, ranges, keys, vals, length, keys_min=0):
        """Selective build of a PHT_1 (vals None) or PHT_2 over rows whose
        filter value lies in one of one or two inclusive ranges."""
        ht = np.zeros(length if vals is None else 2 * length, np.int32)
        keys = np.ascontiguousarray(keys, np.int32)
        v = None if vals is None else np.ascontiguousarray(vals, np.int32)
        f = None if filt is None else np.ascontiguousarray(filt, np.int32)
        (lo0, hi0), (lo1, hi1) = ranges[0], ranges[1] if len(ranges) == 2 else (1, 0)
        self.L.orc_pht_build_ranges(None if f is None else _p(f, _i32p), lo0, hi0, lo1, hi1, _p(keys, _i32p),
                                    None if v is None else _p(v, _i32p), keys.size, _p(ht, _i32p), length, keys_min)
        return ht

    def join_groupby(self, probes, agg, keys, group_sub, n_groups, res_stride, sum_slot, agg_sub=None,
                     sum_bits=64):
        """probes: [(fact column, table, table length, keys_min, kind)];
        keys: [(probe, multiplier, record word or -1)].  Returns the records."""
        cols = [np.ascontiguousarray(p[0], np.int32) for p in probes]
        hts = [np.ascontiguousarray(p[1], np.int32) for p in probes]
        arr = (OrcProbe * len(probes))()
        for i, (p, c, h) in enumerate(zip(probes, cols, hts)):
            arr[i] = OrcProbe(_p(c, _i32p), _p(h, _i32p), p[2], p[3], p[4])
        agg = np.ascontiguousarray(agg, np.int32)
        sub = None if agg_sub is None else np.ascontiguousarray(agg_sub, np.int32)
        kp = np.array([k[0] for k in keys], np.int32)
        km = np.array([k[1] for k in keys], np.int32)
        ks = np.array([k[2] for k in keys], np.int32)
        res = np.zeros(res_stride * n_groups, np.int32)
        self.L.orc_join_groupby(agg.size, arr, len(probes), _p(agg, _i32p), None if sub is None else _p(sub, _i32p),
                                len(keys), _p(kp, _i32p), _p(km, _i32p), _p(ks, _i32p), group_sub, n_groups,
                                res_stride, sum_slot, sum_bits, _p(res, _i32p))
        return res


class Reference:
    """The reference's own FastLanes code, compiled from its sources."""

    def __init__(self, path: str = REF_SO):
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} not built (make -C oracle ref, needs the reference sources)")
        L = ctypes.CDLL(path)
        self.L = L
        L.ref_helper_arr.restype = _u32p
        L.ref_vector_rle.restype = ctypes.c_int
        L.ref_unpack_u32.restype = ctypes.c_int
        L.ref_unpack_fused_u32.restype = ctypes.c_int
        L.ref_unpack8_u32.restype = ctypes.c_int
        L.ref_unpack_h16.restype = ctypes.c_int
        L.ref_q11_sum.restype = ctypes.c_uint64
        L.ref_q11_sum.argtypes = [_u32p, ctypes.c_uint] * 4 + [ctypes.c_uint64] + [ctypes.c_int32] * 5 + [ctypes.c_int]
        L.ref_q21_groupby.restype = None
        L.ref_q21_groupby.argtypes = ([_u32p, ctypes.c_uint] * 4 + [ctypes.c_uint64]
                                      + [_i32p, ctypes.c_int32] * 3 + [ctypes.c_int32, _i32p, ctypes.c_int])
        L.ref_q31_groupby.restype = None
        L.ref_q31_groupby.argtypes = ([_u32p, ctypes.c_uint] * 4 + [ctypes.c_uint64]
                                      + [_i32p, ctypes.c_int32] * 3 + [ctypes.c_int32, _i32p, ctypes.c_int])
        L.ref_q41_groupby.restype = None
        L.ref_q41_groupby.argtypes = ([_u32p, ctypes.c_uint] * 6 + [ctypes.c_uint64]
                                      + [_i32p, ctypes.c_int32] * 4 + [ctypes.c_int32, _i32p, ctypes.c_int])
        L.ref_decode_sum.restype = ctypes.c_uint64
        L.ref_decode_sum.argtypes = [_u32p, ctypes.c_uint, ctypes.c_uint64, ctypes.c_int]
        L.ref_pack_column.restype = None
        L.ref_pack_column.argtypes = [_u32p, ctypes.c_uint64, ctypes.c_uint, _u32p, ctypes.c_int]
        L.ref_decode.restype = ctypes.c_uint64
        L.ref_decode.argtypes = [_u32p, ctypes.c_uint, ctypes.c_uint64, _u32p, ctypes.c_int]

    def helper_arr(self, bw: int) -> np.ndarray:
        ptr = self.L.ref_helper_arr(bw)
        return np.ctypeslib.as_array(ptr, shape=(1024,)).copy()

    def pack(self, vec, bw):
        vec = np.ascontiguousarray(vec, dtype=np.uint32)
        out = np.zeros(max(32 * bw, 1), dtype=np.uint32)
        self.L.ref_pack_u32(_p(vec, _u32p), _p(out, _u32p), ctypes.c_uint(bw))
        return out[:32 * bw]

    def _unary(self, fn, vec):
        vec = np.ascontiguousarray(vec, dtype=np.uint32)
        out = np.zeros(1024, dtype=np.uint32)
        fn(_p(vec, _u32p), _p(out, _u32p))
        return out

    def transpose_i(self, vec):
        return self._unary(self.L.ref_transpose_i_u32, vec)

    def transpose_o(self, vec):
        return self._unary(self.L.ref_transpose_o_u32, vec)

    def unrsum(self, vec):
        return self._unary(self.L.ref_unrsum_u32, vec)

    def unpack(self, packed, bw, fused=False):
        buf = np.zeros(32 * 33, dtype=np.uint32)
        buf[:packed.size] = packed
        out = np.zeros(1024, dtype=np.uint32)
        fn = self.L.ref_unpack_fused_u32 if fused else self.L.ref_unpack_u32
        assert fn(_p(buf, _u32p), _p(out, _u32p), ctypes.c_uint(bw)) == 0
        return out

    def unpack_quarter(self, packed_q, bw):
        buf = np.zeros(32 * 33, dtype=np.uint32)
        buf[:packed_q.size] = packed_q
        out = np.zeros(256, dtype=np.uint32)
        rc = self.L.ref_unpack8_u32(_p(buf, _u32p), _p(out, _u32p), ctypes.c_uint(bw))
        return None if rc != 0 else out

    def unpack_h16(self, packed, bw):
        buf = np.zeros(32 * 33, dtype=np.uint32)
        buf[:packed.size] = packed
        out = np.zeros(1024, dtype=np.uint16)
        rc = self.L.ref_unpack_h16(_p(buf, _u32p), _p(out, _u16p), ctypes.c_uint(bw))
        return None if rc != 0 else out

    def rsum(self, deltas, base):
        deltas = np.ascontiguousarray(deltas, dtype=np.uint32)
        base = np.ascontiguousarray(base, dtype=np.uint32)
        out = np.zeros(1024, dtype=np.uint32)
        self.L.ref_rsum_u32(_p(deltas, _u32p), _p(out, _u32p), _p(base, _u32p))
        return out

    def vector_rle(self, vec):
        vec = np.ascontiguousarray(vec, dtype=np.int32)
        idx = np.zeros(1024, np.uint8)
        dic = np.zeros(1024, np.int32)
        d4 = np.zeros(4, np.uint16)
        n = self.L.ref_vector_rle(_p(vec, _i32p), _p(idx, _u8p), _p(dic, _i32p), _p(d4, _u16p))
        return n, idx, dic[:n].copy(), d4

    def rfor_encode(self, values):
        """The reference's rleBinPack (tile_based/src/rlebinpack.cpp) on values
        padded to whole tiles with the last value, as its main pads them."""
        v = np.ascontiguousarray(values).view(np.uint32)
        n = (v.size + 511) // 512 * 512
        x = np.concatenate([v, np.full(n - v.size, v[-1], np.uint32)])
        bound = 4 + (n // 512) * 515
        val, rl = np.zeros(bound, np.uint32), np.zeros(bound, np.uint32)
        vo, ro = np.zeros(n // 512 + 1, np.uint32), np.zeros(n // 512 + 1, np.uint32)
        sz = np.zeros(2, np.uint32)
        self.L.ref_rfor_encode(_p(x, _u32p), n, _p(val, _u32p), _p(rl, _u32p), _p(vo, _u32p), _p(ro, _u32p),
                               _p(sz, _u32p))
        return val[:sz[0]].copy(), rl[:sz[1]].copy(), vo, ro

    def q11_sum(self, cols, bws, n_rows, date_lo, date_hi, disc_lo, disc_hi, qty_lt, threads):
        args = []
        for c, b in zip(cols, bws):
            args += [_p(c, _u32p), b]
        return int(self.L.ref_q11_sum(*args, n_rows, date_lo, date_hi, disc_lo, disc_hi, qty_lt, threads))

    def q21_groupby(self, cols, bws, n_rows, ht_s, ht_p, ht_d, d_keys_min, threads):
        args = []
        for c, b in zip(cols, bws):
            args += [_p(c, _u32p), b]
        res = np.zeros(4 * N_GROUPS, np.int32)
        self.L.ref_q21_groupby(*args, n_rows, _p(ht_s, _i32p), ht_s.size, _p(ht_p, _i32p), ht_p.size // 2,
                               _p(ht_d, _i32p), ht_d.size // 2, d_keys_min, _p(res, _i32p), threads)
        return res

    def q31_groupby(self, cols, bws, n_rows, ht_s, ht_c, ht_d, d_keys_min, threads):
        args = []
        for c, b in zip(cols, bws):
            args += [_p(c, _u32p), b]
        res = np.zeros(6 * 4375, np.int32)
        self.L.ref_q31_groupby(*args, n_rows, _p(ht_s, _i32p), ht_s.size // 2, _p(ht_c, _i32p), ht_c.size // 2,
                               _p(ht_d, _i32p), ht_d.size // 2, d_keys_min, _p(res, _i32p), threads)
        return res

    def q41_groupby(self, cols, bws, n_rows, ht_s, ht_c, ht_p, ht_d, d_keys_min, threads):
        args = []
        for c, b in zip(cols, bws):
            args += [_p(c, _u32p), b]
        res = np.zeros(4 * 175, np.int32)
        self.L.ref_q41_groupby(*args, n_rows, _p(ht_s, _i32p), ht_s.size, _p(ht_c, _i32p), ht_c.size // 2,
                               _p(ht_p, _i32p), ht_p.size, _p(ht_d, _i32p), ht_d.size // 2, d_keys_min,
                               _p(res, _i32p), threads)
        return res

    def pack_column(self, values, bw, threads):
        v = np.ascontiguousarray(values).view(np.uint32)
        out = np.zeros(((v.size + 1023) // 1024) * 32 * bw + 4, dtype=np.uint32)
        self.L.ref_pack_column(_p(v, _u32p), v.size, bw, _p(out, _u32p), threads)
        return out

    def decode_sum(self, packed, bw, n_vec, threads):
        return int(self.L.ref_decode_sum(_p(packed, _u32p), bw, n_vec, threads))
