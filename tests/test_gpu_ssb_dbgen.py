"""The thirteen SSB queries (crystal-opt src/ssb q11..q43) on the Star Schema
Benchmark's own data -- dbgen compiled from the reference's sources, loaded
with the reference loader's integer encoding (oracle/ssb_data.py) -- encoded as
uniform FastLanes FOR columns and run through the library's operators:

  * against the answers the reference holds: Q1.1, Q1.2 and Q1.3 at scale
    factor 1 and Q1.1 at 10 (fastlanes/src/include/ssb_utils.h:178-183), and
    every group of Q2.1, Q3.1 and Q4.1 at scale factor 10
    (data/result_of_queries/q21,q31,q41), committed in
    tests/golden/ssb_answers.json;
  * and all thirteen against the oracle's loops on the same tables.

Scale factor 10 (60 M rows) is generated on the machine that runs the test
(about two minutes of one core; cached under FLS_SSB_DIR or the temporary
directory)."""
import json
import os

import numpy as np
import pytest

from fastlanesgpu_b200 import datagen, ops

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
ANSWERS = json.load(open(os.path.join(HERE, "golden", "ssb_answers.json")))
QUERIES = list(datagen.SSB_QUERIES)


def _tables(sf):
    import ssb_data as ssb
    if not ssb.available():
        pytest.skip("dbgen not built (make -C oracle dbgen needs the reference sources)")
    t = ssb.load(ssb.generate(sf))
    assert t["lo_orderdate"].size == ssb.LINEORDER_ROWS[sf]
    dcols = {k: c.to_device() for k, c in datagen.ssb_dbgen_columns(t).items()}
    return t, dcols


@pytest.fixture(scope="module")
def sf1(cuda):
    return _tables(1)


@pytest.fixture(scope="module")
def sf10(cuda):
    return _tables(10)


def run(name, t, dcols):
    dq = datagen.ssb_dbgen_query(name, t, dcols)
    if dq["kind"] == "filter":
        got = int(ops.query_filter_agg(dq["cols"], dq["filters"], agg_a=3, agg_b=1).cpu()[0])
    else:
        got = ops.join_groupby(dq["cols"], dq["probes"], **dq["kw"]).cpu().numpy()
    ops.check_device_error()
    return got, dq


def want(oracle, name, t):
    """The oracle's answer on dbgen's tables (its filter and join loops)."""
    q = datagen.SSB_QUERIES[name]
    cols = [t[c] for c in q["cols"]]
    if q["kind"] == "filter":
        filters = [(0, *datagen.SSB_DBGEN_DATE_FILTER[name])] + list(q["filters"][1:])
        return oracle.filter_agg_ranges(cols, filters, 3, 1)
    dims = datagen.ssb_dbgen_dims(t)
    probes = []
    for col, dim, payload, filt, ranges in q["probes"]:
        key, length, kmin = dims[dim]
        ht = oracle.pht_build_ranges(None if filt is None else t[filt], ranges or [(0, -1)], t[key],
                                     None if payload is None else t[payload], length, kmin)
        probes.append((cols[col], ht, length, kmin, 1 if payload is None else 2))
    return oracle.join_groupby(probes, cols[q["agg"]], q["keys"], q["sub"], q["groups"], q["stride"], q["sum_slot"],
                               agg_sub=None if q["agg_sub"] is None else cols[q["agg_sub"]], sum_bits=q["sum_bits"])


def groups(res, stride, key_words, sum_slot):
    """Non-empty group records as sorted rows [key words..., int64 sum]."""
    rec = res.reshape(-1, stride)
    sums = rec[:, sum_slot:sum_slot + 2].copy().view(np.int64)[:, 0]
    rows = [[int(x) for x in r[:key_words]] + [int(s)] for r, s in zip(rec, sums) if s != 0]
    return sorted(rows)


def test_sf1_filter_queries_equal_reference_answers(sf1):
    t, dcols = sf1
    for name in ("q11", "q12", "q13"):
        got, _ = run(name, t, dcols)
        assert got == ANSWERS["scalar"][name]["1"], name


@pytest.mark.parametrize("name", QUERIES)
def test_sf1_query_against_oracle(sf1, oracle, name):
    t, dcols = sf1
    got, dq = run(name, t, dcols)
    w = want(oracle, name, t)
    if dq["kind"] == "filter":
        assert got == w and w > 0
    else:
        assert (w != 0).any() and np.array_equal(got, w), name


def test_sf10_equals_reference_answers(sf10):
    t, dcols = sf10
    got, _ = run("q11", t, dcols)
    assert got == ANSWERS["scalar"]["q11"]["10"] == ANSWERS["q11_file"]
    for name, key_words, stride, sum_slot in (("q21", 2, 4, 2), ("q31", 3, 6, 4), ("q41", 2, 4, 2)):
        res, _ = run(name, t, dcols)
        assert groups(res, stride, key_words, sum_slot) == sorted(ANSWERS["groups_sf10"][name]), name


@pytest.mark.parametrize("name", QUERIES)
def test_sf10_query_against_oracle(sf10, oracle, name):
    t, dcols = sf10
    got, dq = run(name, t, dcols)
    w = want(oracle, name, t)
    if dq["kind"] == "filter":
        assert got == w and w > 0
    else:
        assert (w != 0).any() and np.array_equal(got, w), name
