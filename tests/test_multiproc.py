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
