"""The oracle (CPU restatement) pinned against the reference: its golden
unpack-test arrays, fixtures made by the reference's own functions, and (where
the reference sources were available to build oracle/_ref) the reference
library itself on random inputs."""
import hashlib
import json
import os

import numpy as np
import pytest

from conftest import GOLDEN
from fastlanesgpu_b200 import datagen


@pytest.mark.parametrize("bw", range(33))
def test_pack_matches_reference_fixture(oracle, golden, bw):
    x = datagen.uniform_bits(1024, bw, seed=1000 + bw).view(np.uint32)
    assert np.array_equal(oracle.pack(x, bw), golden[f"pack_{bw}"])
    assert np.array_equal(oracle.unpack(golden[f"pack_{bw}"], bw), x)


def test_delta_matches_reference_fixture(oracle, golden):
    s = datagen.sorted_geometric(1024, seed=77).view(np.uint32)
    t = oracle.transpose_i(s)
    assert np.array_equal(t, golden["delta_transposed"])
    d = oracle.unrsum(t)
    assert np.array_equal(d, golden["delta_deltas"])
    bw = int(golden["delta_bw"][0])
    assert np.array_equal(oracle.pack(d, bw), golden["delta_packed"])
    r = oracle.rsum(oracle.unpack(golden["delta_packed"], bw), t[:32].copy())
    assert np.array_equal(r, golden["delta_rsum"])
    assert np.array_equal(oracle.untranspose(r), s)


def test_rle_matches_reference_fixture(oracle, golden):
    r = datagen.geometric_runs(1024, seed=78)
    n, idx, dic, d4 = oracle.vector_rle(r)
    assert n == int(golden["rle_n"][0])
    assert np.array_equal(idx, golden["rle_idx"])
    assert np.array_equal(dic, golden["rle_dict"])
    assert np.array_equal(d4, golden["rle_dict4"])


@pytest.mark.parametrize("bw", [4, 8, 12, 16, 20])
def test_quarter_unpack_matches_reference_fixture(oracle, golden, bw):
    x = datagen.uniform_bits(1024, bw, seed=2000 + bw).view(np.uint32)
    p = oracle.pack(x, bw)
    pad = np.concatenate([p, np.zeros(64, np.uint32)])
    got = np.concatenate([oracle.unpack_quarter(pad[q * bw * 8:], bw) for q in range(4)])
    assert np.array_equal(got, golden[f"quarter_{bw}"])


def test_helper_arrays_digest(oracle, reference):
    """The reference's golden arrays (rand_arr_*), read from the built
    reference library, round-trip through the oracle and hash to the
    committed digests."""
    with open(os.path.join(GOLDEN, "reference_helper_digest.json")) as f:
        dig = json.load(f)
    for bw in range(33):
        a = reference.helper_arr(bw)
        assert hashlib.sha256(a.tobytes()).hexdigest() == dig[str(bw)]["array_sha256"]
        p = oracle.pack(a, bw)
        assert hashlib.sha256(p.tobytes()).hexdigest() == dig[str(bw)]["packed_sha256"]
        assert np.array_equal(oracle.unpack(p, bw), a)
        assert np.array_equal(reference.unpack(p, bw), a)
        assert np.array_equal(reference.unpack(p, bw, fused=True), a)


def test_transpose_matches_reference(oracle, reference):
    x = np.arange(1024, dtype=np.uint32)
    assert np.array_equal(oracle.transpose_i(x), reference.transpose_i(x))
    # The reference's transpose_o applies the same permutation as transpose_i
    # (it is not the inverse); the oracle's untranspose is the inverse.
    assert np.array_equal(reference.transpose_o(x), reference.transpose_i(x))
    assert np.array_equal(oracle.untranspose(oracle.transpose_i(x)), x)
    pos = oracle.tpos()
    assert np.array_equal(np.sort(pos), np.arange(1024))


def test_random_vectors_match_reference(oracle, reference):
    g = np.random.default_rng(123)
    for trial in range(40):
        bw = int(g.integers(0, 33))
        x = g.integers(0, 2**32, 1024, dtype=np.uint64).astype(np.uint32)
        assert np.array_equal(oracle.pack(x, bw), reference.pack(x, bw))
        p = reference.pack(x, bw)
        assert np.array_equal(oracle.unpack(p, bw), reference.unpack(p, bw))
        s = (np.sort(g.integers(0, 2**31, 1024)) if trial % 2 else g.integers(0, 2**32, 1024)).astype(np.uint32)
        t = reference.transpose_i(s)
        d = reference.unrsum(t)
        assert np.array_equal(oracle.unrsum(t), d)
        assert np.array_equal(oracle.rsum(d, t[:32].copy()), reference.rsum(d, t[:32].copy()))
        runs = np.repeat(g.integers(-5, 5, 300), g.geometric(0.1, 300))[:1024].astype(np.int32)
        if runs.size == 1024:
            a, b = oracle.vector_rle(runs), reference.vector_rle(runs)
            assert a[0] == b[0] and all(np.array_equal(u, v) for u, v in zip(a[1:], b[1:]))


def test_reference_quarter_bw24_not_used(reference):
    # hardcoded_16.cuh's 8-at-a-time routine only covers bw 0,4,...,20 (bw 24
    # writes past its 8-entry output); the wrapper refuses other widths.
    assert reference.unpack_quarter(np.zeros(1024, np.uint32), 24) is None
    assert reference.unpack_quarter(np.zeros(1024, np.uint32), 5) is None


@pytest.mark.parametrize("scheme", range(5))
@pytest.mark.parametrize("kind", ["uniform", "sorted", "runs", "zipf", "const", "extremes"])
def test_scheme_roundtrip(oracle, scheme, kind):
    g = np.random.default_rng(hash((scheme, kind)) % 2**32)
    v = {"uniform": lambda: g.integers(-2**31, 2**31, 1024),
         "sorted": lambda: np.cumsum(g.geometric(0.3, 1024)),
         "runs": lambda: datagen.geometric_runs(1024, seed=int(g.integers(1 << 30))),
         "zipf": lambda: datagen.zipf_values(1024, seed=int(g.integers(1 << 30))),
         "const": lambda: np.full(1024, -7),
         "extremes": lambda: g.choice(np.array([-2**31, 2**31 - 1, 0, -1]), 1024)}[kind]().astype(np.int32)
    for transposed in (True, False):
        if scheme in (1, 2) and not transposed:
            continue
        p, m = oracle.encode_vec(v, scheme, transposed=transposed)
        if p is None:
            assert scheme == 3 and kind != "const"
            continue
        assert m.n_words % 4 == 0
        assert np.array_equal(oracle.decode_vec(p, m, transposed=transposed), v)


@pytest.mark.parametrize("query", ["q21", "q31", "q41"])
def test_join_loops_match_reference(oracle, reference, query):
    """The oracle's restated join + group-by loops (fls_q21/q31/q41.cu) equal the
    reference's CPU arm (its own decoders of the packed columns)."""
    from fastlanesgpu_b200 import datagen
    n = 200_000 + 17
    if query == "q21":
        t = datagen.q21_tables(n, seed=9, part_ids=1 << 14, supp_ids=1 << 12)
        hs = oracle.pht1_build(t["s_region"], 1, t["s_suppkey"], 1 << 12)
        hp = oracle.pht2_build(t["p_category"], 1, t["p_partkey"], t["p_brand1"], 1 << 14)
        hd = oracle.pht2_build(None, 0, t["d_datekey"], t["d_year"], datagen.N_DAYS)
        names, bits = ["lo_suppkey", "lo_partkey", "lo_orderdate", "lo_revenue"], datagen.Q21_BITS
        want = oracle.probe_groupby(*[t[k] for k in names], hs, hp, hd)
        words = [reference.pack_column(t[k], bits[k], 4) for k in names]
        got = reference.q21_groupby(words, [bits[k] for k in names], n, hs, hp, hd, 0, 4)
    elif query == "q31":
        t = datagen.q31_tables(n, seed=9, cust_ids=1 << 14, supp_ids=1 << 12)
        hs = oracle.pht2_build(t["s_region"], 1, t["s_suppkey"], t["s_nation"], 1 << 12)
        hc = oracle.pht2_build(t["c_region"], 1, t["c_custkey"], t["c_nation"], 1 << 14)
        hd = oracle.pht2_build(t["d_in_range"], 1, t["d_datekey"], t["d_year"], datagen.N_DAYS)
        names, bits = ["lo_suppkey", "lo_custkey", "lo_orderdate", "lo_revenue"], datagen.Q31_BITS
        want = oracle.q31_groupby(*[t[k] for k in names], hs, hc, hd)
        words = [reference.pack_column(t[k], bits[k], 4) for k in names]
        got = reference.q31_groupby(words, [bits[k] for k in names], n, hs, hc, hd, 0, 4)
    else:
        t = datagen.q41_tables(n, seed=9, cust_ids=1 << 14, supp_ids=1 << 12, part_ids=1 << 15)
        hs = oracle.pht1_build(t["s_region"], 1, t["s_suppkey"], 1 << 12)
        hc = oracle.pht2_build(t["c_region"], 1, t["c_custkey"], t["c_nation"], 1 << 14)
        hp = oracle.pht1_build(t["p_mfgr_low"], 1, t["p_partkey"], 1 << 15)
        hd = oracle.pht2_build(None, 0, t["d_datekey"], t["d_year"], datagen.N_DAYS)
        names = ["lo_suppkey", "lo_custkey", "lo_partkey", "lo_orderdate", "lo_revenue", "lo_supplycost"]
        bits = datagen.Q41_BITS
        want = oracle.q41_groupby(*[t[k] for k in names], hs, hc, hp, hd)
        words = [reference.pack_column(t[k], bits[k], 4) for k in names]
        got = reference.q41_groupby(words, [bits[k] for k in names], n, hs, hc, hp, hd, 0, 4)
    assert (want != 0).sum() > 10
    assert np.array_equal(got, want)
