"""Parity at the workloads' full sizes: the Q1.1 filter-aggregate and the Q2.1
probe + group-by over 2^27 rows against the oracle (specialised and general
kernels), and decode of 2^28 values (FOR at three widths, to HBM and fused
with a sum) and of 2^27 delta / RLE values against the input, through
size-independent checks (sums and element-wise equality)."""
import numpy as np
import pytest

from fastlanesgpu_b200 import (LAYOUT_TRANSPOSED, ORDER_ORIGINAL, SCHEME_DELTA, SCHEME_RLE, EncodedColumn, datagen,
                               ops)
from fastlanesgpu_b200._lib import TUNE_JIT

pytestmark = pytest.mark.gpu


@pytest.fixture
def both_paths(cuda):
    yield (1, 0)
    ops.set_tuning(TUNE_JIT, 1)


def test_q11_full_size(both_paths, oracle):
    n = 1 << 27
    t = datagen.lineorder_q11(n, seed=2027)
    names = ["date", "discount", "quantity", "price"]
    cols = [EncodedColumn.uniform(t[k], bw=datagen.Q11_BITS[k]).to_device() for k in names]
    f = datagen.Q11_FILTER
    want = oracle.filter_agg(t["date"], t["discount"], t["quantity"], t["price"], *f["date"], *f["discount"],
                             f["quantity"][1] + 1)
    assert want > 0
    for jit in both_paths:
        ops.set_tuning(TUNE_JIT, jit)
        got = int(ops.query_filter_agg(cols, [(0, *f["date"]), (1, *f["discount"]), (2, *f["quantity"])],
                                       agg_a=3, agg_b=1).cpu()[0])
        ops.check_device_error()
        assert got == want, jit


def test_q21_full_size(both_paths, oracle):
    import torch
    n = 1 << 27
    t = datagen.q21_tables(n, seed=2121)
    dev = {k: torch.from_numpy(v).cuda() for k, v in t.items() if not k.startswith("lo_")}
    ht_s = ops.build_pht(dev["s_suppkey"], dev["s_suppkey"].numel(), filt=dev["s_region"], filter_eq=1)
    ht_p = ops.build_pht(dev["p_partkey"], dev["p_partkey"].numel(), vals=dev["p_brand1"], filt=dev["p_category"],
                         filter_eq=1)
    ht_d = ops.build_pht(dev["d_datekey"], datagen.N_DAYS, vals=dev["d_year"])
    names = ["lo_suppkey", "lo_partkey", "lo_orderdate", "lo_revenue"]
    cols = [EncodedColumn.uniform(t[k], bw=datagen.Q21_BITS[k]).to_device() for k in names]
    probes = [(0, ht_s, ht_s.numel(), 0, 1), (1, ht_p, ht_p.numel() // 2, 0, 2), (2, ht_d, ht_d.numel() // 2, 0, 2)]
    want = oracle.probe_groupby(t["lo_suppkey"], t["lo_partkey"], t["lo_orderdate"], t["lo_revenue"],
                                ht_s.cpu().numpy(), ht_p.cpu().numpy(), ht_d.cpu().numpy())
    assert (want[0::4] != 0).sum() > 6000
    for jit in both_paths:
        ops.set_tuning(TUNE_JIT, jit)
        got = ops.probe_groupby(cols, probes, 3, 1, 2, 7, 1992, datagen.N_GROUPS).cpu().numpy()
        ops.check_device_error()
        assert np.array_equal(got, want), jit


@pytest.mark.parametrize("bw", [3, 17, 32])
def test_decode_for_2p28(cuda, bw):
    import torch
    n = 1 << 28
    vals = datagen.uniform_bits(n, bw, seed=2800 + bw)
    want = int(vals.view(np.uint32).astype(np.uint64).sum())
    col = EncodedColumn.uniform(vals, bw=bw).to_device()
    raw = torch.from_numpy(vals).cuda()
    del vals
    assert int(ops.query_aggregate(col).cpu()[0]) & 0xFFFFFFFFFFFFFFFF == want
    assert torch.equal(ops.unpack_global(col)[:n], raw)
    ops.check_device_error()


@pytest.mark.parametrize("scheme", [SCHEME_DELTA, SCHEME_RLE])
def test_decode_delta_rle_2p27(cuda, scheme):
    import torch
    n = 1 << 27
    vals = (datagen.sorted_geometric(n, p=0.3, seed=2701) if scheme == SCHEME_DELTA
            else datagen.geometric_runs(n, mean_run=16.0, value_bits=16, seed=2702))
    want = int(vals.view(np.uint32).astype(np.uint64).sum())
    col = EncodedColumn.encode(vals, scheme, layout=LAYOUT_TRANSPOSED).to_device()
    raw = torch.from_numpy(vals).cuda()
    del vals
    assert int(ops.query_aggregate(col).cpu()[0]) & 0xFFFFFFFFFFFFFFFF == want
    assert torch.equal(ops.unpack_global(col, order=ORDER_ORIGINAL)[:n], raw)
    ops.check_device_error()


@pytest.mark.parametrize("query", ["q31", "q41"])
def test_ssb_joins_full_size(both_paths, oracle, query):
    n = 1 << 27
    t, tables, hcols, dcols, probes, kw = datagen.ssb_join(query, n, seed=3141)
    ht = {k: v.cpu().numpy() for k, v in tables.items()}
    if query == "q31":
        want = oracle.q31_groupby(t["lo_suppkey"], t["lo_custkey"], t["lo_orderdate"], t["lo_revenue"], ht["ht_s"],
                                  ht["ht_c"], ht["ht_d"])
    else:
        want = oracle.q41_groupby(t["lo_suppkey"], t["lo_custkey"], t["lo_partkey"], t["lo_orderdate"],
                                  t["lo_revenue"], t["lo_supplycost"], ht["ht_s"], ht["ht_c"], ht["ht_p"], ht["ht_d"])
    for jit in both_paths:
        ops.set_tuning(TUNE_JIT, jit)
        got = ops.join_groupby(dcols, probes, **kw).cpu().numpy()
        ops.check_device_error()
        assert np.array_equal(got, want), (query, jit)


def test_ssb_suite_full_size(cuda, oracle):
    """All thirteen SSB queries over one 2^27-row lineorder table against the
    oracle (specialised kernels)."""
    from test_gpu_ssb_suite import ssb_run, ssb_want
    n = 1 << 27
    t = datagen.ssb_tables(n, seed=2727)
    dcols = {k: EncodedColumn.uniform(t[k], bw=b).to_device() for k, b in datagen.SSB_BITS.items()}
    for name in datagen.SSB_QUERIES:
        want, _ = ssb_want(oracle, name, t)
        got, _ = ssb_run(name, t, dcols)
        if isinstance(want, int):
            assert got == want, name
        else:
            assert np.array_equal(got, want), name
