"""The oracle's generic join + group-by loop and range-filtered builds (the
SSB query suite's checker) pinned on the CPU against its per-query loops,
which are themselves pinned against the reference's CPU arm."""
import numpy as np

from fastlanesgpu_b200 import datagen


def test_range_build_equals_equality_build(oracle):
    t = datagen.q31_tables(20000, seed=4)
    a = oracle.pht2_build(t["s_region"], 1, t["s_suppkey"], t["s_nation"], t["s_suppkey"].size)
    b = oracle.pht_build_ranges(t["s_region"], [(1, 1)], t["s_suppkey"], t["s_nation"], t["s_suppkey"].size)
    assert np.array_equal(a, b)
    a = oracle.pht1_build(t["c_region"], 3, t["c_custkey"], t["c_custkey"].size)
    b = oracle.pht_build_ranges(t["c_region"], [(3, 3)], t["c_custkey"], None, t["c_custkey"].size)
    assert np.array_equal(a, b)
    both = oracle.pht_build_ranges(t["c_nation"], [(0, 2), (20, 20)], t["c_custkey"], t["c_nation"],
                                   t["c_custkey"].size)
    keep = ((t["c_nation"] <= 2) | (t["c_nation"] == 20)) & (t["c_custkey"] > 0)
    got = both.reshape(-1, 2)
    assert np.array_equal(got[:, 0] != 0, keep)
    assert np.array_equal(got[keep, 1], t["c_nation"][keep])


def test_generic_loop_equals_q31_and_q41_loops(oracle):
    t = datagen.q31_tables(60000, seed=5)
    hs = oracle.pht2_build(t["s_region"], 1, t["s_suppkey"], t["s_nation"], t["s_suppkey"].size)
    hc = oracle.pht2_build(t["c_region"], 1, t["c_custkey"], t["c_nation"], t["c_custkey"].size)
    hd = oracle.pht2_build(t["d_in_range"], 1, t["d_datekey"], t["d_year"], datagen.N_DAYS)
    want = oracle.q31_groupby(t["lo_suppkey"], t["lo_custkey"], t["lo_orderdate"], t["lo_revenue"], hs, hc, hd)
    got = oracle.join_groupby([(t["lo_suppkey"], hs, hs.size // 2, 0, 2), (t["lo_custkey"], hc, hc.size // 2, 0, 2),
                               (t["lo_orderdate"], hd, hd.size // 2, 0, 2)], t["lo_revenue"],
                              [(0, 175, 2), (1, 7, 1), (2, 1, 0)], 1992, 4375, 6, 4)
    assert (want != 0).sum() > 100 and np.array_equal(got, want)
    t = datagen.q41_tables(60000, seed=6)
    hs = oracle.pht1_build(t["s_region"], 1, t["s_suppkey"], t["s_suppkey"].size)
    hc = oracle.pht2_build(t["c_region"], 1, t["c_custkey"], t["c_nation"], t["c_custkey"].size)
    hp = oracle.pht1_build(t["p_mfgr_low"], 1, t["p_partkey"], t["p_partkey"].size)
    hd = oracle.pht2_build(None, 0, t["d_datekey"], t["d_year"], datagen.N_DAYS)
    want = oracle.q41_groupby(t["lo_suppkey"], t["lo_custkey"], t["lo_partkey"], t["lo_orderdate"],
                              t["lo_revenue"], t["lo_supplycost"], hs, hc, hp, hd)
    got = oracle.join_groupby([(t["lo_suppkey"], hs, hs.size, 0, 1), (t["lo_custkey"], hc, hc.size // 2, 0, 2),
                               (t["lo_partkey"], hp, hp.size, 0, 1), (t["lo_orderdate"], hd, hd.size // 2, 0, 2)],
                              t["lo_revenue"], [(1, 7, 1), (3, 1, 0)], 1992, 175, 4, 2, agg_sub=t["lo_supplycost"])
    assert (want != 0).sum() > 50 and np.array_equal(got, want)


def test_generic_loop_32bit_sums_wrap(oracle):
    """sum_bits 32 keeps the low 32 bits of the int64 sum (the wrapping int32
    atomicAdd of crystal-opt q32.cu:101)."""
    t = datagen.q31_tables(60000, seed=7)
    hs = oracle.pht2_build(t["s_region"], 1, t["s_suppkey"], t["s_nation"], t["s_suppkey"].size)
    hd = oracle.pht2_build(None, 0, t["d_datekey"], t["d_year"], datagen.N_DAYS)
    probes = [(t["lo_suppkey"], hs, hs.size // 2, 0, 2), (t["lo_orderdate"], hd, hd.size // 2, 0, 2)]
    r64 = oracle.join_groupby(probes, t["lo_revenue"], [(0, 0, 1), (1, 1, 0)], 1992, 7, 4, 2)
    r32 = oracle.join_groupby(probes, t["lo_revenue"], [(0, 0, 1), (1, 1, 0)], 1992, 7, 4, 3, sum_bits=32)
    s64 = r64.reshape(-1, 4)[:, 2:].copy().view(np.int64)[:, 0]
    assert (np.abs(s64) > 2**31).any()
    assert np.array_equal(r32.reshape(-1, 4)[:, 3], s64.astype(np.uint64).astype(np.uint32).view(np.int32))
    assert np.array_equal(r32.reshape(-1, 4)[:, :2], r64.reshape(-1, 4)[:, :2])


def test_ssb_schema_and_predicates():
    """The synthetic schema keeps dbgen's hierarchy and every SSB predicate
    selects something."""
    t = datagen.ssb_tables(1 << 16, seed=8)
    assert np.array_equal(t["s_nation"], t["s_city"] // 10) and np.array_equal(t["s_region"], t["s_nation"] // 5)
    assert np.array_equal(t["p_category"], t["p_brand1"] // 40) and np.array_equal(t["p_mfgr"], t["p_category"] // 5)
    assert t["d_yearmonthnum"][datagen.day_id(1997, 12, 5)] == 199712
    assert datagen.year_of_day(np.array([datagen.day_id(1995, 7, 1)]))[0] == 1995
    for name, q in datagen.SSB_QUERIES.items():
        if q["kind"] == "filter":
            continue
        for col, dim, payload, filt, ranges in q["probes"]:
            if filt is None:
                continue
            f = t[filt]
            sel = np.zeros(f.size, bool)
            for lo, hi in ranges:
                sel |= (f >= lo) & (f <= hi)
            assert sel.any(), (name, filt)
