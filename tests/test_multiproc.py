"""Multi-rank host logic on CPU (gloo, world size 2): row sharding and the
all-reduce of partial aggregates give the single-process answer."""
import os
import socket

import numpy as np
import pytest

from fastlanesgpu_b200.shard import vector_range


def test_vector_ranges_cover_rows():
    for n in (1, 1023, 1024, 5000, 1 << 20):
        for world in (1, 2, 3, 8):
            rs = [vector_range(n, world, r) for r in range(world)]
            assert rs[0][0] == 0 and rs[-1][1] == n
            for (a0, a1), (b0, b1) in zip(rs, rs[1:]):
                assert a1 == b0 and (a0 % 1024 == 0 or a0 == n)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, n, q):
    import sys
    import torch
    import torch.distributed as dist
    here = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, here)
    sys.path.insert(0, os.path.join(here, "oracle"))
    import datetime
    import oracle as orc
    from fastlanesgpu_b200 import datagen
    from fastlanesgpu_b200.shard import allreduce_sum, vector_range
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        t = datagen.lineorder_q11(n, seed=5)
        r0, r1 = vector_range(n, world, rank)
        f = datagen.Q11_FILTER
        part = orc.Oracle().filter_agg(t["date"][r0:r1], t["discount"][r0:r1], t["quantity"][r0:r1],
                                       t["price"][r0:r1], *f["date"], *f["discount"], f["quantity"][1] + 1)
        x = torch.tensor([part], dtype=torch.int64)
        allreduce_sum(x)
        q.put((rank, int(x.item())))
    finally:
        dist.destroy_process_group()


def test_gloo_two_ranks_allreduce_partials(oracle):
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    n = 300_000
    port = _free_port()
    ps = [ctx.Process(target=_worker, args=(r, 2, port, n, q)) for r in range(2)]
    for p in ps:
        p.start()
    for p in ps:
        p.join(timeout=120)
        assert p.exitcode == 0
    got = dict(q.get(timeout=5) for _ in range(2))
    from fastlanesgpu_b200 import datagen
    t = datagen.lineorder_q11(n, seed=5)
    f = datagen.Q11_FILTER
    want = oracle.filter_agg(t["date"], t["discount"], t["quantity"], t["price"], *f["date"], *f["discount"],
                             f["quantity"][1] + 1)
    assert got[0] == got[1] == want


def _ssb_records(oracle, name, t, r0, r1):
    """The oracle's records of SSB join query `name` over rows [r0, r1)."""
    from fastlanesgpu_b200 import datagen
    q = datagen.SSB_QUERIES[name]
    keys = {"d": "d_datekey", "s": "s_suppkey", "c": "c_custkey", "p": "p_partkey"}
    cols = [t[c][r0:r1] for c in q["cols"]]
    probes = []
    for col, dim, payload, filt, ranges in q["probes"]:
        k = t[keys[dim]]
        ht = oracle.pht_build_ranges(None if filt is None else t[filt], ranges or [(0, -1)], k,
                                     None if payload is None else t[payload], k.size)
        probes.append((cols[col], ht, k.size, 0, 1 if payload is None else 2))
    return oracle.join_groupby(probes, cols[q["agg"]], q["keys"], q["sub"], q["groups"], q["stride"],
                               q["sum_slot"], agg_sub=None if q["agg_sub"] is None else cols[q["agg_sub"]],
                               sum_bits=q["sum_bits"])


def _records_worker(rank, world, port, n, names, q):
    import sys
    import torch
    import torch.distributed as dist
    here = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, here)
    sys.path.insert(0, os.path.join(here, "oracle"))
    import datetime
    import oracle as orc
    from fastlanesgpu_b200 import datagen
    from fastlanesgpu_b200.shard import combine_group_records, vector_range
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        t = datagen.ssb_tables(n, seed=9)
        r0, r1 = vector_range(n, world, rank)
        out = {}
        for name in names:
            spec = datagen.SSB_QUERIES[name]
            res = torch.from_numpy(_ssb_records(orc.Oracle(), name, t, r0, r1))
            combine_group_records(res, spec["stride"], spec["sum_slot"], spec["sum_bits"])
            out[name] = res.numpy()
        q.put((rank, out))
    finally:
        dist.destroy_process_group()


def test_gloo_two_ranks_combine_group_records(oracle):
    """Row shards of SSB join queries with int64 sums (Q4.2: 6-word records)
    and wrapping int32 sums (Q3.2, Q4.3) combine into the single-process
    records."""
    import multiprocessing as mp
    from fastlanesgpu_b200 import datagen
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    n, names = 400_000, ["q32", "q42", "q43"]
    port = _free_port()
    ps = [ctx.Process(target=_records_worker, args=(r, 2, port, n, names, q)) for r in range(2)]
    for p in ps:
        p.start()
    got = dict(q.get(timeout=300) for _ in range(2))
    for p in ps:
        p.join(timeout=120)
        assert p.exitcode == 0
    t = datagen.ssb_tables(n, seed=9)
    for name in names:
        want = _ssb_records(oracle, name, t, 0, n)
        assert (want != 0).any()
        assert np.array_equal(got[0][name], want) and np.array_equal(got[1][name], want), name


def _leaving_worker(rank, world, port, q):
    import datetime
    import sys
    import time
    import torch
    import torch.distributed as dist
    here = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, here)
    from fastlanesgpu_b200.shard import allreduce_sum
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=5))
    x = torch.ones(1, dtype=torch.int64)
    allreduce_sum(x)  # one good step on both ranks
    if rank == 1:
        q.put((rank, "left", int(x.item())))
        q.close()
        q.join_thread()  # the message is out before the process ends
        os._exit(0)  # leaves between steps, without its next collective
    t0 = time.time()
    try:
        allreduce_sum(x)
        q.put((rank, "no error", time.time() - t0))
    except Exception as e:  # the peer is gone: the collective ends with an error
        q.put((rank, type(e).__name__, time.time() - t0))
    q.close()
    q.join_thread()
    os._exit(0)


def test_gloo_rank_that_leaves_ends_the_next_collective_with_an_error():
    """Failure detection on the host: after one good step, rank 1 exits
    between steps; rank 0's next all-reduce raises within the process group's
    short timeout instead of waiting for good."""
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_leaving_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    got = {}
    for _ in range(2):
        r, what, val = q.get(timeout=120)
        got[r] = (what, val)
    for p in ps:
        p.join(timeout=60)
    assert got[1] == ("left", 2)
    assert got[0][0] != "no error" and got[0][1] < 60, got
