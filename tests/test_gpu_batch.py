"""GPU: batched persistent execution of many filter-aggregate queries over
columns of uneven length, bit width and scheme -- equal to per-query launches
and to the oracle; CUDA-graph replay; autotuner."""
import numpy as np
import pytest

from fastlanesgpu_b200 import EncodedColumn, ops
from fastlanesgpu_b200.batch import Batch, graph_of
from fastlanesgpu_b200.selector import training_corpus

pytestmark = pytest.mark.gpu


def _mixed_columns(n_cols, seed, max_log=18):
    g = np.random.default_rng(seed)
    vals, cols = [], []
    for c in range(n_cols):
        n = int(2 ** g.uniform(10, max_log)) + int(g.integers(0, 1000))
        v = training_corpus((n + 1023) // 1024, seed=seed * 100 + c)[:n]
        sizes, best = ops.encode_exhaustive(v)
        vals.append(v)
        cols.append(EncodedColumn.encode(v, best).to_device())
    return vals, cols


def _queries(vals, n_q, seed):
    g = np.random.default_rng(seed)
    qs = []
    for _ in range(n_q):
        c = int(g.integers(0, len(vals)))
        lo, hi = np.sort(g.choice(vals[c], 2))
        qs.append((c, int(lo), int(hi), c))
    return qs


def _want(vals, q):
    c, lo, hi, a = q
    sel = (vals[c] >= lo) & (vals[c] <= hi)
    return int(vals[a][sel].astype(np.int64).sum()), int(sel.sum())


def test_batch_matches_oracle_and_per_query(cuda):
    vals, cols = _mixed_columns(12, seed=1)
    qs = _queries(vals, 40, seed=2)
    b = Batch(cols, qs, chunk_vectors=8)
    got = b.run().cpu().numpy()
    for i, q in enumerate(qs):
        assert tuple(got[i]) == _want(vals, q)
        c, lo, hi, a = q
        one = int(ops.query_filter_agg([cols[c]], [(0, lo, hi)], agg_a=0).cpu()[0])
        assert one == got[i][0]
    ops.check_device_error()
    b.close()


def test_batch_two_columns_and_empty_ranges(cuda):
    g = np.random.default_rng(5)
    n = 70_000
    a = g.integers(0, 1000, n).astype(np.int32)
    b_ = np.cumsum(g.geometric(0.5, n)).astype(np.int32)
    cols = [EncodedColumn.encode(a, 0).to_device(), EncodedColumn.encode(b_, 1).to_device()]
    qs = [(0, 100, 200, 1), (1, 10, 5, 0), (0, -5, 2000, 1), (1, int(b_[100]), int(b_[60000]), 0)]
    got = Batch(cols, qs, chunk_vectors=4).run().cpu().numpy()
    vals = [a, b_]
    for i, q in enumerate(qs):
        c, lo, hi, ag = q
        sel = (vals[c] >= lo) & (vals[c] <= hi)
        assert tuple(got[i]) == (int(vals[ag][sel].astype(np.int64).sum()), int(sel.sum()))


def test_batch_graph_replay(cuda):
    import torch
    vals, cols = _mixed_columns(6, seed=3, max_log=16)
    qs = _queries(vals, 16, seed=4)
    b = Batch(cols, qs)
    g = graph_of(b.run)
    b.results.fill_(-1)
    g.replay()
    torch.cuda.synchronize()
    got = b.results.view(-1, 2).cpu().numpy()
    for i, q in enumerate(qs):
        assert tuple(got[i]) == _want(vals, q)
    del g


def test_autotuner_picks_and_caches(cuda, tmp_path):
    from fastlanesgpu_b200 import autotune, datagen
    t = datagen.lineorder_q11(1 << 18, seed=3)
    cols = [EncodedColumn.uniform(t[k], bw=datagen.Q11_BITS[k]).to_device()
            for k in ("date", "discount", "quantity", "price")]
    f = datagen.Q11_FILTER
    run = lambda: ops.query_filter_agg(cols, [(0, *f["date"]), (1, *f["discount"]), (2, *f["quantity"])], 3, 1)
    want = int(run().cpu()[0])
    space = {"warps": [8, 16], "stages": [2], "tile_bytes": [6144], "sparse_rows": [2, 8]}
    path = str(tmp_path / "tune.json")
    try:
        best = autotune.tune("q11-test", run, space=space, iters=3, path=path)
        assert len(best["candidates"]) == 4 and best["ms"] > 0
        assert int(run().cpu()[0]) == want
        again = autotune.tune("q11-test", run, space=space, iters=3, path=path)
        assert again["config"] == best["config"]
    finally:
        autotune.reset()


def test_autotuner_join_space(cuda, oracle, tmp_path):
    """JOIN_SPACE picks the join kernel's variants for one query (late
    measures, group sums per CTA, table budget) by timing them; every candidate gives the
    oracle's records, and the choice is applied and cached."""
    from fastlanesgpu_b200 import autotune, datagen
    from test_gpu_ssb_suite import ssb_want
    t = datagen.ssb_tables(1 << 20, seed=5)
    dcols = {k: EncodedColumn.uniform(t[k], bw=b).to_device() for k, b in datagen.SSB_BITS.items()}
    dq = datagen.ssb_device_query("q43", t, dcols)
    want, _ = ssb_want(oracle, "q43", t)
    got = []
    run = lambda: got.append(ops.join_groupby(dq["cols"], dq["probes"], **dq["kw"]))  # noqa: E731
    path = str(tmp_path / "tune.json")
    try:
        best = autotune.tune("q43-test", run, space=autotune.JOIN_SPACE, iters=2, path=path)
        assert len(best["candidates"]) == 8 and set(best["config"]) == {"late_measure", "group_smem", "table_kb"}
        assert ops.get_tuning(3) == best["config"]["late_measure"]
        assert ops.get_tuning(4) == best["config"]["table_kb"]
        assert all(np.array_equal(g.cpu().numpy(), want) for g in got)
        again = autotune.tune("q43-test", run, space=autotune.JOIN_SPACE, iters=2, path=path)
        assert again["config"] == best["config"]
        # re-timing the leaders and a preferred configuration no other beats
        # by 100 %: the preferred one is kept and applied
        kept = autotune.tune("q43-keep", run, space=autotune.JOIN_SPACE, iters=2, use_cache=False,
                             prefer=autotune.JOIN_DEFAULT, margin=1.0, retime=2)
        assert kept["config"] == autotune.JOIN_DEFAULT and len(kept["candidates"]) == 8
        assert ops.get_tuning(3) == 1 and ops.get_tuning(2) == 1 and ops.get_tuning(4) == 72
        assert all(np.array_equal(g.cpu().numpy(), want) for g in got)
    finally:
        autotune.reset()
