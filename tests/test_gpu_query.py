"""GPU parity of the fused decode + query operators against the oracle and the
reference's CPU arm (reference decoders + restated query loops)."""
import numpy as np
import pytest

from fastlanesgpu_b200 import LAYOUT_NORMAL, LAYOUT_TRANSPOSED, EncodedColumn, FlsError, datagen, ops

pytestmark = pytest.mark.gpu

N_GROUPS = datagen.N_GROUPS


def _q11_cols(t, layout=LAYOUT_NORMAL, per_vector=False):
    order = ["date", "discount", "quantity", "price"]
    cols = []
    for k in order:
        if per_vector:
            cols.append(EncodedColumn.encode(t[k], 0, layout=layout))
        else:
            cols.append(EncodedColumn.uniform(t[k], bw=datagen.Q11_BITS[k], layout=layout))
    return cols


def _q11(cols_dev, f=datagen.Q11_FILTER):
    return ops.query_filter_agg(cols_dev, [(0, *f["date"]), (1, *f["discount"]), (2, *f["quantity"])],
                                agg_a=3, agg_b=1)


@pytest.mark.parametrize("n", [1, 1000, 1 << 20, (1 << 20) + 333])
def test_filter_agg_q11_shape(cuda, oracle, reference, n):
    t = datagen.lineorder_q11(n, seed=n)
    cols = _q11_cols(t)
    got = int(_q11([c.to_device() for c in cols]).cpu()[0])
    f = datagen.Q11_FILTER
    want = oracle.filter_agg(t["date"], t["discount"], t["quantity"], t["price"], *f["date"], *f["discount"],
                             f["quantity"][1] + 1)
    assert got == want
    ref = reference.q11_sum([c.words for c in cols], [c.bw for c in cols], n, *f["date"], *f["discount"],
                            f["quantity"][1] + 1, 4)
    assert got == ref
    ops.check_device_error()


@pytest.mark.parametrize("layout", [LAYOUT_NORMAL, LAYOUT_TRANSPOSED])
def test_filter_agg_per_vector_columns(cuda, oracle, layout):
    n = 300 * 1024 + 17
    t = datagen.lineorder_q11(n, seed=5)
    cols = [c.to_device() for c in _q11_cols(t, layout=layout, per_vector=True)]
    f = datagen.Q11_FILTER
    want = oracle.filter_agg(t["date"], t["discount"], t["quantity"], t["price"], *f["date"], *f["discount"],
                             f["quantity"][1] + 1)
    assert int(_q11(cols).cpu()[0]) == want


def test_filter_agg_variants_and_schemes(cuda):
    n = 200 * 1024 + 9
    a = datagen.sorted_geometric(n, seed=3)
    b = datagen.geometric_runs(n, seed=4)
    c = datagen.zipf_values(n, seed=5)
    cols = [EncodedColumn.encode(a, 1).to_device(), EncodedColumn.encode(b, 2).to_device(),
            EncodedColumn.encode(c, 4).to_device()]
    lo, hi = int(np.quantile(a, 0.2)), int(np.quantile(a, 0.7))
    sel = (a >= lo) & (a <= hi) & (b >= 100) & (b <= 40000)
    assert int(ops.query_filter_agg(cols, [(0, lo, hi), (1, 100, 40000)], agg_a=2).cpu()[0]) == int(
        c[sel].astype(np.int64).sum())
    assert int(ops.query_filter_agg(cols, [(0, lo, hi), (1, 100, 40000)]).cpu()[0]) == int(sel.sum())
    assert int(ops.query_filter_agg(cols, [(2, 0, 10)], agg_a=0, agg_b=1).cpu()[0]) == int(
        (a.astype(np.int64) * b)[(c >= 0) & (c <= 10)].sum())
    assert int(ops.query_filter_agg(cols, [(0, 5, 4)], agg_a=2).cpu()[0]) == 0  # empty range
    assert int(ops.query_filter_agg(cols, [], agg_a=2).cpu()[0]) == int(c.astype(np.int64).sum())


def test_filter_agg_negative_values(cuda):
    g = np.random.default_rng(3)
    n = 50 * 1024
    a = g.integers(-2**31, 2**31, n).astype(np.int32)
    b = g.integers(-1000, 1000, n).astype(np.int32)
    cols = [EncodedColumn.encode(a, 0).to_device(), EncodedColumn.encode(b, 0).to_device()]
    sel = (a >= -2**30) & (a <= 2**29)
    want = int((a[sel].astype(np.int64) * b[sel]).sum())
    assert int(ops.query_filter_agg(cols, [(0, -2**30, 2**29)], agg_a=0, agg_b=1).cpu()[0]) == want


def test_mixed_layouts_rejected(cuda):
    t = datagen.lineorder_q11(4096)
    c0 = EncodedColumn.uniform(t["date"], layout=LAYOUT_NORMAL).to_device()
    c1 = EncodedColumn.encode(t["price"], 0, layout=LAYOUT_TRANSPOSED).to_device()
    with pytest.raises(FlsError):
        ops.query_filter_agg([c0, c1], [(0, 0, 10)], agg_a=1)


def _q21(n, seed, part_ids, supp_ids):
    import torch
    t = datagen.q21_tables(n, seed=seed, part_ids=part_ids, supp_ids=supp_ids)
    dev = {k: torch.from_numpy(v).cuda() for k, v in t.items()}
    ht_s = ops.build_pht(dev["s_suppkey"], supp_ids, filt=dev["s_region"], filter_eq=1)
    ht_p = ops.build_pht(dev["p_partkey"], part_ids, vals=dev["p_brand1"], filt=dev["p_category"], filter_eq=1)
    ht_d = ops.build_pht(dev["d_datekey"], datagen.N_DAYS, vals=dev["d_year"])
    return t, ht_s, ht_p, ht_d


def _q21_run(t, hts, layout=LAYOUT_NORMAL, per_vector=False):
    ht_s, ht_p, ht_d = hts
    names = ["lo_suppkey", "lo_partkey", "lo_orderdate", "lo_revenue"]
    if per_vector:
        cols = [EncodedColumn.encode(t[k], 0, layout=layout) for k in names]
    else:
        cols = [EncodedColumn.uniform(t[k], bw=datagen.Q21_BITS[k], layout=layout) for k in names]
    dcols = [c.to_device() for c in cols]
    probes = [(0, ht_s, ht_s.numel(), 0, 1), (1, ht_p, ht_p.numel() // 2, 0, 2), (2, ht_d, ht_d.numel() // 2, 0, 2)]
    res = ops.probe_groupby(dcols, probes, agg_col=3, key_a=1, key_b=2, group_mul=7, group_sub=1992,
                            n_groups=N_GROUPS)
    return cols, res.cpu().numpy()


@pytest.mark.parametrize("n,part_ids,supp_ids", [(1 << 20, 1 << 16, 1 << 14), (123457, 1 << 19, 1 << 17)])
def test_pht_build_and_probe_groupby(cuda, oracle, reference, n, part_ids, supp_ids):
    t, ht_s, ht_p, ht_d = _q21(n, 21, part_ids, supp_ids)
    o_s = oracle.pht1_build(t["s_region"], 1, t["s_suppkey"], supp_ids)
    o_p = oracle.pht2_build(t["p_category"], 1, t["p_partkey"], t["p_brand1"], part_ids)
    o_d = oracle.pht2_build(None, 0, t["d_datekey"], t["d_year"], datagen.N_DAYS)
    assert np.array_equal(ht_s.cpu().numpy(), o_s)
    assert np.array_equal(ht_p.cpu().numpy(), o_p)
    assert np.array_equal(ht_d.cpu().numpy(), o_d)
    cols, got = _q21_run(t, (ht_s, ht_p, ht_d))
    want = oracle.probe_groupby(t["lo_suppkey"], t["lo_partkey"], t["lo_orderdate"], t["lo_revenue"], o_s, o_p, o_d)
    assert np.array_equal(got, want)
    assert (want[0::4] != 0).sum() > 0
    ref = reference.q21_groupby([c.words for c in cols], [c.bw for c in cols], n, o_s, o_p, o_d, 0, 4)
    assert np.array_equal(got, ref)
    ops.check_device_error()


@pytest.mark.parametrize("layout", [LAYOUT_NORMAL, LAYOUT_TRANSPOSED])
def test_probe_groupby_per_vector_columns(cuda, oracle, layout):
    n = 200 * 1024 + 3
    t, ht_s, ht_p, ht_d = _q21(n, 22, 1 << 16, 1 << 12)
    _, got = _q21_run(t, (ht_s, ht_p, ht_d), layout=layout, per_vector=True)
    want = oracle.probe_groupby(t["lo_suppkey"], t["lo_partkey"], t["lo_orderdate"], t["lo_revenue"],
                                ht_s.cpu().numpy(), ht_p.cpu().numpy(), ht_d.cpu().numpy())
    assert np.array_equal(got, want)


def test_probe_global_tables(cuda, oracle):
    """Tables too large for shared memory are probed in global memory."""
    n = 64 * 1024
    t, ht_s, ht_p, ht_d = _q21(n, 23, 1 << 19, 1 << 20)  # supplier bitmap 128 KB > smem budget
    _, got = _q21_run(t, (ht_s, ht_p, ht_d), per_vector=True)
    want = oracle.probe_groupby(t["lo_suppkey"], t["lo_partkey"], t["lo_orderdate"], t["lo_revenue"],
                                ht_s.cpu().numpy(), ht_p.cpu().numpy(), ht_d.cpu().numpy())
    assert np.array_equal(got, want)


def test_probe_out_of_range_keys_flagged(cuda, oracle):
    """Keys below keys_min hash to a negative slot: the reference reads out of
    bounds there; here the row is dropped and the device error word is set."""
    import torch
    n = 8 * 1024
    t, ht_s, ht_p, ht_d = _q21(n, 24, 1 << 12, 1 << 10)
    t["lo_orderdate"][::97] = -5
    names = ["lo_suppkey", "lo_partkey", "lo_orderdate", "lo_revenue"]
    cols = [EncodedColumn.encode(t[k], 0).to_device() for k in names]
    probes = [(0, ht_s, ht_s.numel(), 0, 1), (1, ht_p, ht_p.numel() // 2, 0, 2), (2, ht_d, ht_d.numel() // 2, 0, 2)]
    ops.probe_groupby(cols, probes, 3, 1, 2, 7, 1992, N_GROUPS)
    with pytest.raises(FlsError):
        ops.check_device_error()
    torch.cuda.synchronize()


@pytest.mark.parametrize("sparse_rows", [1, 4, 8, 32])
def test_sparse_threshold_does_not_change_results(cuda, oracle, sparse_rows):
    """Dense and row-at-a-time evaluation give identical answers."""
    n = 100 * 1024 + 1
    t = datagen.lineorder_q11(n, seed=9)
    f = datagen.Q11_FILTER
    want = oracle.filter_agg(t["date"], t["discount"], t["quantity"], t["price"], *f["date"], *f["discount"],
                             f["quantity"][1] + 1)
    tq, ht_s, ht_p, ht_d = _q21(n, 25, 1 << 14, 1 << 10)
    want21 = oracle.probe_groupby(tq["lo_suppkey"], tq["lo_partkey"], tq["lo_orderdate"], tq["lo_revenue"],
                                  ht_s.cpu().numpy(), ht_p.cpu().numpy(), ht_d.cpu().numpy())
    try:
        ops.set_tuning(0, sparse_rows)
        for per_vector in (False, True):
            cols = [c.to_device() for c in _q11_cols(t, per_vector=per_vector)]
            assert int(_q11(cols).cpu()[0]) == want
            _, got = _q21_run(tq, (ht_s, ht_p, ht_d), per_vector=per_vector)
            assert np.array_equal(got, want21)
    finally:
        ops.set_tuning(0, 0)


@pytest.mark.parametrize("n", [1000, (1 << 20) + 77])
def test_crystal_api_kernels(cuda, oracle, n):
    """Kernels written against the drop-in primitive API (fls_crystal.cuh),
    launched one CTA per vector like the reference, match the oracle."""
    t = datagen.lineorder_q11(n, seed=31)
    cols = [c.to_device() for c in _q11_cols(t)]
    f = datagen.Q11_FILTER
    got = int(ops.crystal_q11(cols, n, f["date"][0] - 1, f["date"][1] + 1, f["quantity"][1] + 1, *f["discount"]).cpu()[0])
    want = oracle.filter_agg(t["date"], t["discount"], t["quantity"], t["price"], *f["date"], *f["discount"],
                             f["quantity"][1] + 1)
    assert got == want
    tq, ht_s, ht_p, ht_d = _q21(n, 32, 1 << 16, 1 << 14)
    names = ["lo_suppkey", "lo_partkey", "lo_orderdate", "lo_revenue"]
    qcols = [EncodedColumn.uniform(tq[k], bw=datagen.Q21_BITS[k]).to_device() for k in names]
    got21 = ops.crystal_q21_probe(qcols, n, ht_s, ht_p, ht_d).cpu().numpy()
    want21 = oracle.probe_groupby(tq["lo_suppkey"], tq["lo_partkey"], tq["lo_orderdate"], tq["lo_revenue"],
                                  ht_s.cpu().numpy(), ht_p.cpu().numpy(), ht_d.cpu().numpy())
    assert np.array_equal(got21, want21)
