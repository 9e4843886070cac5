"""The drop-in device API proven on the reference's own kernels: the query
kernels of fastlanes/src/ssb/fls_q21.cu (Q2.1: hash-table builds with
BlockLoad / BlockPredEQ / BlockBuildSelectivePHT_1/_2; probe_v1 decoding with
unpack_device into 32 registers, probe_v2 with
unpack_8_at_a_time::unpack_device + BlockLoad, probe_v3 with BlockPredLoad)
and of compress_ssb.cu (Q4.1 over per-vector bit widths, bases and offsets
through unpack_8_at_a_time, builds with BlockPredOrEQ), compiled unchanged
against include/fls_crystal.cuh via include/compat (oracle/Makefile, target
dropin), run on the GPU.  Their hash tables must equal the oracle's builds and
their group records the oracle's loop and the library's own join operator."""
import ctypes
import os

import numpy as np
import pytest

from fastlanesgpu_b200 import LAYOUT_TRANSPOSED, SCHEME_DELTA, EncodedColumn, datagen, ops

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DATE_MIN, DATE_SLOTS = 19920101, 19981230 - 19920101 + 1


def _lib(name):
    path = os.path.join(ROOT, "oracle", "_ref", f"libdropin_{name}.so")
    if not os.path.exists(path):
        pytest.skip(f"{path} not built (make -C oracle dropin needs the reference sources)")
    return ctypes.CDLL(path)


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def _dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.int32)).cuda()


def _packed(values, bw):
    """Uniform FastLanes bit-packing (the reference's pack.cpp layout) on the device."""
    c = EncodedColumn.uniform(np.asarray(values, np.int32), bw=bw)
    return _dev(c.words.view(np.int32)), c


def _dates():
    days = np.datetime64("1992-01-01") + np.arange(datagen.N_DAYS)
    ymd = days.astype(object)
    key = np.array([d.year * 10000 + d.month * 100 + d.day for d in ymd], np.int32)
    return key, np.array([d.year for d in ymd], np.int32)


def _no_decoder_error(L, name):
    bits = ctypes.c_uint32(99)
    assert getattr(L, f"dropin_{name}_take_error")(ctypes.byref(bits)) == 0
    assert bits.value == 0


def _records(res, stride, key_words, sum_slot):
    rec = res.reshape(-1, stride)
    s = rec[:, sum_slot:sum_slot + 2].copy().view(np.int64)[:, 0]
    return sorted([int(x) for x in r[:key_words]] + [int(v)] for r, v in zip(rec, s) if v != 0)


def test_reference_q21_kernels_on_dropin_headers(cuda, oracle):
    import torch
    L = _lib("q21")
    w = (ctypes.c_int * 4)()
    L.dropin_q21_widths(w)
    bw_od, bw_pk, bw_sk, bw_rev = list(w)
    g = np.random.default_rng(2121)
    s_len, p_len, n = 2000, 200000, 300 * 1024 + 77
    s_key = np.arange(1, s_len + 1, dtype=np.int32)
    s_region = g.integers(0, 5, s_len).astype(np.int32)
    p_key = np.arange(1, p_len + 1, dtype=np.int32)
    p_cat = g.integers(0, 25, p_len).astype(np.int32)
    p_brand = (p_cat * 40 + g.integers(0, 40, p_len)).astype(np.int32)
    d_key, d_year = _dates()
    lo_sk = g.integers(1, s_len + 1, n).astype(np.int32)
    lo_pk = g.integers(1, p_len + 1, n).astype(np.int32)
    lo_od = d_key[g.integers(0, d_key.size, n)]
    lo_rev = g.integers(81360, 10474951, n).astype(np.int32)
    # the reference's tables, built by its own kernels
    ht_s = torch.zeros(s_len, dtype=torch.int32, device=cuda)
    ht_p = torch.zeros(2 * p_len, dtype=torch.int32, device=cuda)
    ht_d = torch.zeros(2 * DATE_SLOTS, dtype=torch.int32, device=cuda)
    dims = [_dev(x) for x in (s_region, s_key, p_cat, p_key, p_brand, d_key, d_year)]
    assert L.dropin_q21_build(_ptr(dims[0]), _ptr(dims[1]), s_len, _ptr(dims[2]), _ptr(dims[3]), _ptr(dims[4]), p_len,
                              _ptr(dims[5]), _ptr(dims[6]), d_key.size, _ptr(ht_s), _ptr(ht_p), _ptr(ht_d),
                              DATE_SLOTS) == 0
    o_s = oracle.pht_build_ranges(s_region, [(1, 1)], s_key, None, s_len)
    o_p = oracle.pht_build_ranges(p_cat, [(1, 1)], p_key, p_brand, p_len)
    o_d = oracle.pht_build_ranges(None, [(0, -1)], d_key, d_year, DATE_SLOTS, DATE_MIN)
    assert np.array_equal(ht_s.cpu().numpy(), o_s) and np.array_equal(ht_p.cpu().numpy(), o_p)
    assert np.array_equal(ht_d.cpu().numpy(), o_d)
    # the oracle's Q2.1 loop (fls_q21.cu:50-77 semantics)
    q = datagen.SSB_QUERIES["q21"]
    want = oracle.join_groupby([(lo_sk, o_s, s_len, 0, 1), (lo_pk, o_p, p_len, 0, 2),
                                (lo_od, o_d, DATE_SLOTS, DATE_MIN, 2)], lo_rev, q["keys"], q["sub"], q["groups"],
                               q["stride"], q["sum_slot"])
    assert len(_records(want, 4, 2, 2)) > 200
    # the columns as fls_q21.cu packs them: orderdate - 19920101 and the keys
    # at the file's widths, revenue packed (probe_v1) or plain (v2, v3)
    od, _ = _packed(lo_od - DATE_MIN, bw_od)
    pk, _ = _packed(lo_pk, bw_pk)
    sk, _ = _packed(lo_sk, bw_sk)
    rev_p, _ = _packed(lo_rev, bw_rev)
    rev = _dev(lo_rev)
    for version in (1, 2, 3):
        res = torch.zeros(4 * 7000, dtype=torch.int32, device=cuda)
        assert L.dropin_q21_probe(version, _ptr(od), _ptr(pk), _ptr(sk), _ptr(rev_p if version == 1 else rev), n,
                                  _ptr(ht_s), s_len, _ptr(ht_p), p_len, _ptr(ht_d), DATE_SLOTS, _ptr(res)) == 0
        assert np.array_equal(res.cpu().numpy(), want), version
    _no_decoder_error(L, "q21")
    # the library's own operator on the same data gives the same records
    cols = {"lo_suppkey": lo_sk, "lo_partkey": lo_pk, "lo_orderdate": lo_od, "lo_revenue": lo_rev}
    dcols = [EncodedColumn.uniform(cols[k], base=int(cols[k].min())).to_device() for k in q["cols"]]
    probes = [(0, ht_s, s_len, 0, 1), (1, ht_p, p_len, 0, 2), (2, ht_d, DATE_SLOTS, DATE_MIN, 2)]
    got = ops.join_groupby(dcols, probes, agg_col=3, keys=q["keys"], group_sub=q["sub"], n_groups=q["groups"],
                           res_stride=4, sum_slot=2).cpu().numpy()
    ops.check_device_error()
    assert np.array_equal(got, want)


def _find_bw(x):
    """The reference's per-vector width: bit width of the maximum rounded up to
    a multiple of 4 (fastlanes/src/include/ssb_utils.h:222-239)."""
    b = int(x.max()).bit_length()
    return 0 if b == 0 else -(-b // 4) * 4


def _per_vector(values):
    """compress_ssb.cu:400-447: per vector, the minimum as base, the width of
    the rest, and the word offset of the packed vector."""
    n = values.size
    nv = -(-n // 1024)
    v = np.concatenate([values, np.full(nv * 1024 - n, values[-1], np.int32)]).reshape(nv, 1024)
    words, bws, bases, offs, off = [], [], [], [], 0
    for vec in v:
        base = int(vec.min())
        bw = _find_bw(vec - base)
        words.append(ops.pack((vec - base).astype(np.int32), bw).view(np.int32))
        bws.append(bw)
        bases.append(base)
        offs.append(off)
        off += 32 * bw
    words.append(np.zeros(32 * 32, np.int32))  # slack after the last vector
    return (_dev(np.concatenate(words)), _dev(np.array(bws)), _dev(np.array(bases)), _dev(np.array(offs)),
            np.array(bws))


def test_reference_q41_per_vector_kernel_on_dropin_headers(cuda, oracle):
    import torch
    L = _lib("q41")
    w = (ctypes.c_int * 3)()
    L.dropin_q41_widths(w)
    bw_sk, bw_pk, bw_sc = list(w)
    g = np.random.default_rng(4141)
    s_len, p_len, c_len, n = 2000, 200000, 30000, 200 * 1024 + 333
    s_key, p_key, c_key = (np.arange(1, k + 1, dtype=np.int32) for k in (s_len, p_len, c_len))
    s_region = g.integers(0, 5, s_len).astype(np.int32)
    p_mfgr = g.integers(0, 5, p_len).astype(np.int32)
    c_region = g.integers(0, 5, c_len).astype(np.int32)
    c_nation = (c_region * 5 + g.integers(0, 5, c_len)).astype(np.int32)
    d_key, d_year = _dates()
    lo_sk = g.integers(1, s_len + 1, n).astype(np.int32)
    lo_pk = g.integers(1, p_len + 1, n).astype(np.int32)
    # custkey and orderdate vary in range from vector to vector, so their
    # per-vector widths differ
    nv = -(-n // 1024)
    spans = g.choice([1, 16, 300, 5000, c_len], nv)
    starts = np.array([g.integers(1, c_len - s + 2) for s in spans])
    lo_ck = (np.repeat(starts, 1024)[:n] + g.integers(0, np.repeat(spans, 1024)[:n])).astype(np.int32)
    assert lo_ck.min() >= 1 and lo_ck.max() <= c_len
    lo_od = d_key[g.integers(0, d_key.size, n)]
    lo_rev = g.integers(81360, 10474951, n).astype(np.int32)
    lo_sc = g.integers(54060, 125940, n).astype(np.int32)
    ht_s = torch.zeros(2 * s_len, dtype=torch.int32, device=cuda)
    ht_p = torch.zeros(2 * p_len, dtype=torch.int32, device=cuda)
    ht_c = torch.zeros(2 * c_len, dtype=torch.int32, device=cuda)
    ht_d = torch.zeros(2 * DATE_SLOTS, dtype=torch.int32, device=cuda)
    dims = [_dev(x) for x in (s_region, s_key, p_mfgr, p_key, c_region, c_key, c_nation, d_key, d_year)]
    assert L.dropin_q41_build(_ptr(dims[0]), _ptr(dims[1]), s_len, _ptr(dims[2]), _ptr(dims[3]), p_len, _ptr(dims[4]),
                              _ptr(dims[5]), _ptr(dims[6]), c_len, _ptr(dims[7]), _ptr(dims[8]), d_key.size,
                              _ptr(ht_s), _ptr(ht_p), _ptr(ht_c), _ptr(ht_d), DATE_SLOTS) == 0
    o_s = oracle.pht_build_ranges(s_region, [(1, 1)], s_key, None, s_len)
    o_p = oracle.pht_build_ranges(p_mfgr, [(0, 1)], p_key, None, p_len)
    o_c = oracle.pht_build_ranges(c_region, [(1, 1)], c_key, c_nation, c_len)
    o_d = oracle.pht_build_ranges(None, [(0, -1)], d_key, d_year, DATE_SLOTS, DATE_MIN)
    assert np.array_equal(ht_s.cpu().numpy()[:s_len], o_s) and np.array_equal(ht_p.cpu().numpy()[:p_len], o_p)
    assert np.array_equal(ht_c.cpu().numpy(), o_c) and np.array_equal(ht_d.cpu().numpy(), o_d)
    q = datagen.SSB_QUERIES["q41"]
    want = oracle.join_groupby([(lo_sk, o_s, s_len, 0, 1), (lo_ck, o_c, c_len, 0, 2), (lo_pk, o_p, p_len, 0, 1),
                                (lo_od, o_d, DATE_SLOTS, DATE_MIN, 2)], lo_rev, q["keys"], q["sub"], q["groups"],
                               q["stride"], q["sum_slot"], agg_sub=lo_sc)
    assert len(_records(want, 4, 2, 2)) > 20
    od, od_bw, od_base, od_off, od_bws = _per_vector(lo_od - DATE_MIN)
    ck, ck_bw, ck_base, ck_off, ck_bws = _per_vector(lo_ck)
    assert len(set(ck_bws.tolist())) >= 3  # several widths among the vectors
    sk, _ = _packed(lo_sk, bw_sk)
    pk, _ = _packed(lo_pk, bw_pk)
    sc, _ = _packed(lo_sc, bw_sc)
    rev = _dev(lo_rev)
    res = torch.zeros(4 * 175, dtype=torch.int32, device=cuda)
    assert L.dropin_q41_probe(_ptr(od), _ptr(od_bw), _ptr(od_base), _ptr(od_off), _ptr(pk), _ptr(ck), _ptr(ck_bw),
                              _ptr(ck_base), _ptr(ck_off), _ptr(sk), _ptr(rev), _ptr(sc), n, _ptr(ht_p), p_len,
                              _ptr(ht_s), s_len, _ptr(ht_c), c_len, _ptr(ht_d), DATE_SLOTS, _ptr(res)) == 0
    assert np.array_equal(res.cpu().numpy(), want)
    _no_decoder_error(L, "q41")


def test_reference_q31_kernels_on_dropin_headers(cuda, oracle):
    """fls_q31.cu: the normal-form unpack_device into shared memory + BlockLoad
    (probe_v1), BlockProbeAndPHT_2_R_S into shared tiles (probe_v2) and
    unpack_8_at_a_time with BlockLoad / BlockPredLoad (probe_v3 / v4)."""
    import torch
    L = _lib("q31")
    w = (ctypes.c_int * 4)()
    L.dropin_q31_widths(w)
    bw_od, bw_ck, bw_sk, bw_rev = list(w)
    g = np.random.default_rng(3131)
    s_len, c_len, n = 2000, 30000, 250 * 1024 + 5
    s_key, c_key = np.arange(1, s_len + 1, dtype=np.int32), np.arange(1, c_len + 1, dtype=np.int32)
    s_region, c_region = g.integers(0, 5, s_len).astype(np.int32), g.integers(0, 5, c_len).astype(np.int32)
    s_nation = (s_region * 5 + g.integers(0, 5, s_len)).astype(np.int32)
    c_nation = (c_region * 5 + g.integers(0, 5, c_len)).astype(np.int32)
    d_key, d_year = _dates()
    lo_sk = g.integers(1, s_len + 1, n).astype(np.int32)
    lo_ck = g.integers(1, c_len + 1, n).astype(np.int32)
    lo_od = d_key[g.integers(0, d_key.size, n)]
    lo_rev = g.integers(81360, 10474951, n).astype(np.int32)
    ht_s = torch.zeros(2 * s_len, dtype=torch.int32, device=cuda)
    ht_c = torch.zeros(2 * c_len, dtype=torch.int32, device=cuda)
    ht_d = torch.zeros(2 * DATE_SLOTS, dtype=torch.int32, device=cuda)
    # fls_q31.cu's builds select region 2 (ASIA) and years 1992-1997
    dims = [_dev(x) for x in (s_region, s_key, s_nation, c_region, c_key, c_nation, d_key, d_year)]
    assert L.dropin_q31_build(_ptr(dims[0]), _ptr(dims[1]), _ptr(dims[2]), s_len, _ptr(dims[3]), _ptr(dims[4]),
                              _ptr(dims[5]), c_len, _ptr(dims[6]), _ptr(dims[7]), d_key.size, _ptr(ht_s), _ptr(ht_c),
                              _ptr(ht_d), DATE_SLOTS) == 0
    o_s = oracle.pht_build_ranges(s_region, [(2, 2)], s_key, s_nation, s_len)
    o_c = oracle.pht_build_ranges(c_region, [(2, 2)], c_key, c_nation, c_len)
    o_d = oracle.pht_build_ranges(d_year, [(1992, 1997)], d_key, d_year, DATE_SLOTS, DATE_MIN)
    assert np.array_equal(ht_s.cpu().numpy(), o_s) and np.array_equal(ht_c.cpu().numpy(), o_c)
    assert np.array_equal(ht_d.cpu().numpy(), o_d)
    q = datagen.SSB_QUERIES["q31"]
    want = oracle.join_groupby([(lo_sk, o_s, s_len, 0, 2), (lo_ck, o_c, c_len, 0, 2),
                                (lo_od, o_d, DATE_SLOTS, DATE_MIN, 2)], lo_rev, q["keys"], q["sub"], q["groups"],
                               q["stride"], q["sum_slot"])
    assert len(_records(want, 6, 3, 4)) > 100
    od, _ = _packed(lo_od - DATE_MIN, bw_od)
    ck, _ = _packed(lo_ck, bw_ck)
    sk, _ = _packed(lo_sk, bw_sk)
    rev_p, _ = _packed(lo_rev, bw_rev)
    rev = _dev(lo_rev)
    for version in (1, 2, 3, 4):
        res = torch.zeros(6 * 4375, dtype=torch.int32, device=cuda)
        assert L.dropin_q31_probe(version, _ptr(od), _ptr(ck), _ptr(sk), _ptr(rev_p if version <= 2 else rev), n,
                                  _ptr(ht_s), s_len, _ptr(ht_c), c_len, _ptr(ht_d), DATE_SLOTS, _ptr(res)) == 0
        assert np.array_equal(res.cpu().numpy(), want), version
    _no_decoder_error(L, "q31")


@pytest.mark.parametrize("bw_seed", [(0.3, 1), (0.05, 2)])
def test_reference_delta_kernel_on_dropin_headers(cuda, bw_seed):
    """delta_shared_memory.cu's decode + sum: the normal-form unpack_device,
    d_rsum_32 over the transposed rows with the vector's lane bases, BlockLoad
    and BlockSum, over the library's own uniform DELTA encoding (32 lane bases
    + 32*bw packed deltas per vector, split into the kernel's two arrays)."""
    import torch
    L = _lib("delta")
    p, seed = bw_seed
    n = 500 * 1024
    vals = datagen.sorted_geometric(n, p=p, seed=seed)
    col = EncodedColumn.uniform(vals, SCHEME_DELTA, layout=LAYOUT_TRANSPOSED)
    nv, bw = col.n_vec, col.bw
    words = col.words[: nv * (32 + 32 * bw)].reshape(nv, 32 + 32 * bw)
    bases = _dev(words[:, :32].reshape(-1).view(np.int32))
    packed = _dev(np.concatenate([words[:, 32:].reshape(-1), np.zeros(32 * 32, np.uint32)]).view(np.int32))
    s = torch.zeros(1, dtype=torch.int64, device=cuda)
    assert L.dropin_delta_sum(_ptr(bases), _ptr(packed), ctypes.c_uint64(nv), ctypes.c_uint32(bw), ctypes.c_uint64(n),
                              _ptr(s)) == 0
    want = int(vals.view(np.uint32).astype(np.uint64).sum()) & ((1 << 64) - 1)
    assert int(s.cpu()[0]) & ((1 << 64) - 1) == want
    _no_decoder_error(L, "delta")
