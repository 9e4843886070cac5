"""All thirteen SSB queries (crystal-opt src/ssb q11.cu .. q43.cu) on the
seeded SSB-shaped schema, through the library's two query operators: the
hash tables built on the device with the queries' dimension predicates equal
the oracle's builds, and every result equals the oracle's loop, with the
specialised and the general kernels, with measures staged or read late and
with the default and the largest shared-memory budget for the tables."""
import numpy as np
import pytest

from fastlanesgpu_b200 import EncodedColumn, datagen, ops
from fastlanesgpu_b200._lib import TUNE_HALF_VECTORS, TUNE_JIT, TUNE_LATE_MEASURE, TUNE_TABLE_KB

pytestmark = pytest.mark.gpu

QUERIES = list(datagen.SSB_QUERIES)


def _dim_key(dim):
    return {"d": ("d_datekey", datagen.N_DAYS), "s": ("s_suppkey", datagen.SSB_SUPP),
            "c": ("c_custkey", datagen.SSB_CUST), "p": ("p_partkey", datagen.SSB_PART)}[dim]


def ssb_want(oracle, name, t):
    """The oracle's answer to SSB query `name` and its hash tables."""
    q = datagen.SSB_QUERIES[name]
    cols = [t[c] for c in q["cols"]]
    if q["kind"] == "filter":
        return oracle.filter_agg_ranges(cols, q["filters"], 3, 1), []
    tables, probes = [], []
    for col, dim, payload, filt, ranges in q["probes"]:
        key, length = _dim_key(dim)
        ht = oracle.pht_build_ranges(None if filt is None else t[filt], ranges or [(0, -1)], t[key],
                                     None if payload is None else t[payload], length)
        tables.append(ht)
        probes.append((cols[col], ht, length, 0, 1 if payload is None else 2))
    res = oracle.join_groupby(probes, cols[q["agg"]], q["keys"], q["sub"], q["groups"], q["stride"], q["sum_slot"],
                              agg_sub=None if q["agg_sub"] is None else cols[q["agg_sub"]], sum_bits=q["sum_bits"])
    return res, tables


def ssb_run(name, t, dcols):
    dq = datagen.ssb_device_query(name, t, dcols)
    if dq["kind"] == "filter":
        got = int(ops.query_filter_agg(dq["cols"], dq["filters"], agg_a=3, agg_b=1).cpu()[0])
    else:
        got = ops.join_groupby(dq["cols"], dq["probes"], **dq["kw"]).cpu().numpy()
    ops.check_device_error()
    return got, dq


@pytest.fixture(scope="module")
def ssb_data(cuda):
    n = (1 << 20) + 11
    t = datagen.ssb_tables(n, seed=1313)
    dcols = {k: EncodedColumn.uniform(t[k], bw=b).to_device() for k, b in datagen.SSB_BITS.items()}
    return t, dcols


@pytest.mark.parametrize("name", QUERIES)
def test_ssb_query_against_oracle(ssb_data, oracle, name):
    t, dcols = ssb_data
    want, tables = ssb_want(oracle, name, t)
    try:
        for jit, late, table_kb, half in ((1, 0, 0, 0), (1, 1, 0, 0), (1, 0, 144, 0), (1, 1, 144, 0), (1, 0, 0, 1),
                                          (1, 1, 0, 1), (1, 0, 144, 1), (0, 0, 0, 0)):
            ops.set_tuning(TUNE_JIT, jit)
            ops.set_tuning(TUNE_LATE_MEASURE, late)
            ops.set_tuning(TUNE_TABLE_KB, table_kb)
            ops.set_tuning(TUNE_HALF_VECTORS, half)
            before = ops.jit_stats()["launches"]
            got, dq = ssb_run(name, t, dcols)
            assert ops.jit_stats()["launches"] - before == jit, (name, jit)
            if dq["kind"] == "filter":
                assert want > 0 and got == want, (name, jit)
            else:
                for a, b in zip(dq["tables"], tables):
                    assert np.array_equal(a.cpu().numpy(), b), name
                assert (want != 0).any() and np.array_equal(got, want), (name, jit)
    finally:
        ops.set_tuning(TUNE_JIT, 1)
        ops.set_tuning(TUNE_LATE_MEASURE, 1)  # the default
        ops.set_tuning(TUNE_TABLE_KB, 0)
        ops.set_tuning(TUNE_HALF_VECTORS, 0)
    assert ops.jit_stats()["failures"] == 0, ops.jit_last_log()
