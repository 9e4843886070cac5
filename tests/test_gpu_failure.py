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


def test_error_words_are_per_stream(cuda, oracle):
    """Two streams with words of their own (fls_bind_error_word): a query over
    bad vector metadata on one and an exact query on the other run at the
    same time; each check reports only its own stream's error, and the
    default word of unbound streams stays clean."""
    import torch
    ops.check_device_error()
    s_bad, s_good = torch.cuda.Stream(), torch.cuda.Stream()
    w_bad = torch.zeros(2, dtype=torch.int32, device=cuda)
    w_good = torch.zeros(2, dtype=torch.int32, device=cuda)
    vals = datagen.uniform_bits(64 * 1024, 9, seed=2)
    col = EncodedColumn.encode(vals, 0)
    col.meta["offset"][5] = col.words.size  # outside the buffer: skipped and reported
    bad = col.to_device()
    t = datagen.lineorder_q11(300 * 1024 + 7, seed=5)
    cols = [EncodedColumn.uniform(t[k], bw=datagen.Q11_BITS[k]).to_device() for k in ("date", "discount",
                                                                                          "quantity", "price")]
    f = datagen.Q11_FILTER
    filters = [(0, *f["date"]), (1, *f["discount"]), (2, *f["quantity"])]
    want = oracle.filter_agg(t["date"], t["discount"], t["quantity"], t["price"], *f["date"], *f["discount"],
                             f["quantity"][1] + 1)
    torch.cuda.synchronize()
    try:
        ops.bind_error_word(w_bad, s_bad)
        ops.bind_error_word(w_good, s_good)
        for _ in range(3):
            with torch.cuda.stream(s_bad):
                ops.query_aggregate(bad)
            with torch.cuda.stream(s_good):
                res = ops.query_filter_agg(cols, filters, agg_a=3, agg_b=1)
        ops.check_device_error(s_good)  # clean, although the other stream's kernels flagged errors
        with torch.cuda.stream(s_good):
            assert int(res.cpu()[0]) == want
        with pytest.raises(FlsError) as e:
            ops.check_device_error(s_bad)
        assert e.value.status == 5 and "bad-vector-metadata" in str(e.value)
        ops.check_device_error(s_bad)   # taken out by the check
        ops.check_device_error()        # the default word never saw either
        # a timeout on the good stream is that stream's alone
        with torch.cuda.stream(s_good):
            ops.selftest_bounded_wait(1)
        ops.check_device_error(s_bad)
        with pytest.raises(FlsError) as e:
            ops.check_device_error(s_good)
        assert e.value.status == 6
        assert int(w_bad.cpu()[0]) == 0 and int(w_good.cpu()[0]) == 0
    finally:
        ops.bind_error_word(None, s_bad)
        ops.bind_error_word(None, s_good)
    # unbound again: errors go to the default word
    with torch.cuda.stream(s_bad):
        ops.query_aggregate(bad)
    with pytest.raises(FlsError):
        ops.check_device_error(s_bad)
    ops.check_device_error()


def test_bind_error_word_arguments(cuda):
    import torch
    w = torch.zeros(4, dtype=torch.int32, device=cuda)
    with pytest.raises(FlsError) as e:
        ops.bind_error_word(w[1:])  # 4-byte offset: not 8-byte aligned
    assert e.value.status == 3
    ops.bind_error_word(None)       # unbinding an unbound stream is a no-op
