"""Failure detection without a GPU fault: a bounded device wait on a barrier
that nothing arrives on gives up, the host reads FLS_ERR_TIMEOUT from the
device error word, the word is cleared, and the context keeps working (a
query on the same stream returns the right answer afterwards)."""
import numpy as np
import pytest

from fastlanesgpu_b200 import EncodedColumn, FlsError, datagen, ops

pytestmark = pytest.mark.gpu


def test_bounded_wait_times_out_and_context_survives(cuda, oracle):
    ops.check_device_error()  # start clean
    for polls in (1, 64):
        ops.selftest_bounded_wait(polls)
        with pytest.raises(FlsError) as e:
            ops.check_device_error()
        assert e.value.status == 6 and "wait-timeout" in str(e.value)
        ops.check_device_error()  # the error word was cleared
    t = datagen.lineorder_q11(200 * 1024 + 3, seed=4)
    cols = [EncodedColumn.uniform(t[k], bw=datagen.Q11_BITS[k]).to_device() for k in ("date", "discount",
                                                                                          "quantity", "price")]
    f = datagen.Q11_FILTER
    got = int(ops.query_filter_agg(cols, [(0, *f["date"]), (1, *f["discount"]), (2, *f["quantity"])], agg_a=3,
                                   agg_b=1).cpu()[0])
    ops.check_device_error()
    want = oracle.filter_agg(t["date"], t["discount"], t["quantity"], t["price"], *f["date"], *f["discount"],
                             f["quantity"][1] + 1)
    assert got == want


def test_selftest_arguments(cuda):
    for polls in (0, 1025):
        with pytest.raises(FlsError) as e:
            ops.selftest_bounded_wait(polls)
        assert e.value.status == 1
