"""The Q3.1 and Q4.1 join + group-by shapes (fastlanes/src/ssb/fls_q31.cu and
fls_q41.cu probe_v1) through the general join + group-by operator: against the
oracle's restatement of those loops and the reference's CPU arm (its own
decoders), with the specialised and the general kernels, on uniform and
per-vector columns; the Q2.1 call as a special case; descriptor validation."""
import numpy as np
import pytest

from fastlanesgpu_b200 import EncodedColumn, FlsError, datagen, ops
from fastlanesgpu_b200._lib import TUNE_JIT

pytestmark = pytest.mark.gpu


def _want(oracle, query, t, tables):
    ht = {k: v.cpu().numpy() for k, v in tables.items()}
    if query == "q31":
        return oracle.q31_groupby(t["lo_suppkey"], t["lo_custkey"], t["lo_orderdate"], t["lo_revenue"], ht["ht_s"],
                                  ht["ht_c"], ht["ht_d"])
    return oracle.q41_groupby(t["lo_suppkey"], t["lo_custkey"], t["lo_partkey"], t["lo_orderdate"], t["lo_revenue"],
                              t["lo_supplycost"], ht["ht_s"], ht["ht_c"], ht["ht_p"], ht["ht_d"])


def _ref(reference, query, hcols, n, tables):
    ht = {k: v.cpu().numpy() for k, v in tables.items()}
    words, bws = [c.words for c in hcols], [c.bw for c in hcols]
    if query == "q31":
        return reference.q31_groupby(words, bws, n, ht["ht_s"], ht["ht_c"], ht["ht_d"], 0, 4)
    return reference.q41_groupby(words, bws, n, ht["ht_s"], ht["ht_c"], ht["ht_p"], ht["ht_d"], 0, 4)


@pytest.mark.parametrize("query", ["q31", "q41"])
@pytest.mark.parametrize("n", [1, 3000, (1 << 20) + 11])
def test_join_groupby_against_oracle_and_reference(cuda, oracle, reference, query, n):
    t, tables, hcols, dcols, probes, kw = datagen.ssb_join(query, n, seed=n + 7)
    want = _want(oracle, query, t, tables)
    if n > 1000:
        assert (want != 0).sum() > 10
    assert np.array_equal(_ref(reference, query, hcols, n, tables), want)
    try:
        for jit in (1, 0):
            ops.set_tuning(TUNE_JIT, jit)
            before = ops.jit_stats()["launches"]
            got = ops.join_groupby(dcols, probes, **kw).cpu().numpy()
            ops.check_device_error()
            assert ops.jit_stats()["launches"] - before == jit
            assert np.array_equal(got, want), (query, n, jit)
    finally:
        ops.set_tuning(TUNE_JIT, 1)


@pytest.mark.parametrize("query", ["q31", "q41"])
@pytest.mark.parametrize("scheme", [0, 1])
def test_join_groupby_per_vector_columns(cuda, oracle, query, scheme):
    """Per-vector FOR columns take the general row-at-a-time kernel; a DELTA
    foreign key takes the general whole-vector kernel."""
    n = 100 * 1024 + 5
    t, tables, hcols, _, probes, kw = datagen.ssb_join(query, n, seed=77)
    names = (["lo_suppkey", "lo_custkey", "lo_orderdate", "lo_revenue"] if query == "q31" else
             ["lo_suppkey", "lo_custkey", "lo_partkey", "lo_orderdate", "lo_revenue", "lo_supplycost"])
    dcols = [EncodedColumn.encode(t[c], scheme if i == 0 else 0).to_device() for i, c in enumerate(names)]
    got = ops.join_groupby(dcols, probes, **kw).cpu().numpy()
    ops.check_device_error()
    assert np.array_equal(got, _want(oracle, query, t, tables))


def test_q21_call_is_the_general_form(cuda, oracle):
    import torch
    n = 200 * 1024 + 3
    t = datagen.q21_tables(n, seed=5, part_ids=1 << 14, supp_ids=1 << 12)
    dev = {k: torch.from_numpy(v).cuda() for k, v in t.items() if not k.startswith("lo_")}
    ht_s = ops.build_pht(dev["s_suppkey"], 1 << 12, filt=dev["s_region"])
    ht_p = ops.build_pht(dev["p_partkey"], 1 << 14, vals=dev["p_brand1"], filt=dev["p_category"])
    ht_d = ops.build_pht(dev["d_datekey"], datagen.N_DAYS, vals=dev["d_year"])
    names = ["lo_suppkey", "lo_partkey", "lo_orderdate", "lo_revenue"]
    cols = [EncodedColumn.uniform(t[k], bw=datagen.Q21_BITS[k]).to_device() for k in names]
    probes = [(0, ht_s, ht_s.numel(), 0, 1), (1, ht_p, ht_p.numel() // 2, 0, 2), (2, ht_d, ht_d.numel() // 2, 0, 2)]
    a = ops.probe_groupby(cols, probes, 3, 1, 2, 7, 1992, datagen.N_GROUPS).cpu().numpy()
    b = ops.join_groupby(cols, probes, 3, [(1, 7, 1), (2, 1, 0)], 1992, datagen.N_GROUPS, 4, 2).cpu().numpy()
    want = oracle.probe_groupby(t["lo_suppkey"], t["lo_partkey"], t["lo_orderdate"], t["lo_revenue"],
                                ht_s.cpu().numpy(), ht_p.cpu().numpy(), ht_d.cpu().numpy())
    assert np.array_equal(a, want) and np.array_equal(b, want)


def test_join_groupby_descriptor_validation(cuda):
    t, tables, hcols, dcols, probes, kw = datagen.ssb_join("q41", 4096, seed=3)
    bad = [dict(kw, keys=[(0, 7, 1)]),            # a key on a PHT_1 probe
           dict(kw, res_stride=5),                 # odd record
           dict(kw, sum_slot=3),                   # odd sum word
           dict(kw, keys=[(1, 7, 2), (3, 1, 0)]),  # key word on the sum
           dict(kw, agg_sub_col=9),                # no such column
           dict(kw, keys=[])]                      # no key
    for b in bad:
        with pytest.raises((FlsError, ValueError)):
            ops.join_groupby(dcols, probes, **b)


@pytest.mark.parametrize("query", ["q31", "q41"])
def test_join_groupby_workspace_forms(cuda, oracle, query):
    """The presence bitmaps built once per call into a workspace, or per CTA
    without one, give the same result; a workspace smaller than
    fls_join_workspace_bytes is refused before anything runs."""
    import torch
    n = 300 * 1024 + 17
    t, tables, hcols, dcols, probes, kw = datagen.ssb_join(query, n, seed=n)
    want = _want(oracle, query, t, tables)
    need = ops.join_workspace_bytes(dcols, probes, **kw)
    assert need > 0
    big = torch.zeros(need + 4096, dtype=torch.uint8, device="cuda")
    for ws in (None, "auto", big):
        got = ops.join_groupby(dcols, probes, workspace=ws, **kw).cpu().numpy()
        ops.check_device_error()
        assert np.array_equal(got, want), ws if ws is None or isinstance(ws, str) else "tensor"
    with pytest.raises(FlsError) as e:
        ops.join_groupby(dcols, probes, workspace=big[:need - 16], **kw)
    assert e.value.status == 8
    ops.check_device_error()


def test_q21_workspace_forms(cuda, oracle):
    import torch
    n = 200 * 1024 + 9
    t = datagen.q21_tables(n, seed=9)
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
    for ws in (None, "auto"):
        got = ops.probe_groupby(cols, probes, 3, 1, 2, 7, 1992, datagen.N_GROUPS, workspace=ws).cpu().numpy()
        ops.check_device_error()
        assert np.array_equal(got, want), ws
