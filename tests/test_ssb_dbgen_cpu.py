"""The Star Schema Benchmark data path without a GPU: dbgen compiled from the
reference's sources and the loader (oracle/ssb_data.py) reproduce the tables
the reference's answers were computed on -- the oracle's filter-aggregate
loop (crystal-opt src/ssb q11/q12/q13 predicates on yyyymmdd dates) gives
Q1.1 at scale factors 0.1 and 1 and Q1.2 and Q1.3 at 1 exactly as
fastlanes/src/include/ssb_utils.h:178-183 holds them -- and the dimension
codes follow the reference loader (data/ssb/loader/convert.py)."""
import json
import os

import numpy as np
import pytest

from fastlanesgpu_b200 import datagen

HERE = os.path.dirname(os.path.abspath(__file__))
ANSWERS = json.load(open(os.path.join(HERE, "golden", "ssb_answers.json")))


def _load(sf):
    import ssb_data
    if not ssb_data.available():
        pytest.skip("dbgen not built (make -C oracle dbgen needs the reference sources)")
    t = ssb_data.load(ssb_data.generate(sf))
    assert t["lo_orderdate"].size == ssb_data.LINEORDER_ROWS[sf]
    return t


@pytest.mark.parametrize("sf,names", [(0.1, ["q11"]), (1, ["q11", "q12", "q13"])])
def test_filter_queries_equal_reference_answers(oracle, sf, names):
    t = _load(sf)
    for name in names:
        q = datagen.SSB_QUERIES[name]
        cols = [t[c] for c in q["cols"]]
        filters = [(0, *datagen.SSB_DBGEN_DATE_FILTER[name])] + list(q["filters"][1:])
        assert oracle.filter_agg_ranges(cols, filters, 3, 1) == ANSWERS["scalar"][name][f"{sf:g}"], (sf, name)


def test_dimension_codes():
    t = _load(1)
    assert t["s_suppkey"].size == 2000 and t["c_custkey"].size == 30000 and t["p_partkey"].size == 200000
    assert t["d_datekey"].size == 2556 and t["d_datekey"][0] == 19920101 and t["d_datekey"][-1] == 19981230
    for k in ("s_suppkey", "c_custkey", "p_partkey"):
        assert np.array_equal(t[k], np.arange(1, t[k].size + 1))
    for p in ("s", "c"):
        assert np.array_equal(t[f"{p}_city"] // 10, t[f"{p}_nation"])
        assert t[f"{p}_nation"].max() == 24 and t[f"{p}_region"].max() == 4
    assert np.array_equal(t["p_brand1"] // 40, t["p_category"]) and np.array_equal(t["p_category"] // 5, t["p_mfgr"])
    assert t["p_brand1"].max() == 999 and t["p_mfgr"].max() == 4
    dims = datagen.ssb_dbgen_dims(t)
    assert dims["d"] == ("d_datekey", 61130, 19920101)
    # the date table's slots cover every day key
    assert (t["d_datekey"] - 19920101).max() < 61130
