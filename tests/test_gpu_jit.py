"""GPU parity of the specialised (NVRTC-compiled) filter-aggregate kernel:
against the oracle on Q1.1, and against a numpy evaluation and the general
kernel on seeded random query shapes (bit widths 0..32, both layouts, 0-4
filters, count / sum / sum of products, ragged lengths)."""
import numpy as np
import pytest

from fastlanesgpu_b200 import LAYOUT_NORMAL, LAYOUT_TRANSPOSED, EncodedColumn, datagen, ops
from fastlanesgpu_b200._lib import TUNE_GROUP_SMEM, TUNE_JIT, TUNE_SPARSE_ROWS

pytestmark = pytest.mark.gpu


@pytest.fixture
def jit_on(cuda):
    ops.set_tuning(TUNE_JIT, 1)
    yield
    ops.set_tuning(TUNE_JIT, 1)
    ops.set_tuning(TUNE_SPARSE_ROWS, 0)


def _launches():
    return ops.jit_stats()["launches"]


def _run(cols, filters, a, b, jit):
    ops.set_tuning(TUNE_JIT, 1 if jit else 0)
    before = _launches()
    got = int(ops.query_filter_agg(cols, filters, agg_a=a, agg_b=b).cpu()[0])
    ops.check_device_error()
    return got, _launches() - before


def _numpy(vals, filters, a, b):
    sel = np.ones(vals[0].size, bool)
    for c, lo, hi in filters:
        sel &= (vals[c] >= lo) & (vals[c] <= hi)
    if a < 0:
        return int(sel.sum())
    x = vals[a][sel].astype(np.int64)
    if b >= 0:
        x = x * vals[b][sel].astype(np.int64)
    return int(x.sum())


@pytest.mark.parametrize("n", [1, 1000, 1 << 20, (1 << 20) + 333, 1 << 24])
def test_jit_q11_against_oracle(jit_on, oracle, n):
    t = datagen.lineorder_q11(n, seed=n)
    order = ["date", "discount", "quantity", "price"]
    cols = [EncodedColumn.uniform(t[k], bw=datagen.Q11_BITS[k]).to_device() for k in order]
    f = datagen.Q11_FILTER
    filters = [(0, *f["date"]), (1, *f["discount"]), (2, *f["quantity"])]
    want = oracle.filter_agg(t["date"], t["discount"], t["quantity"], t["price"], *f["date"], *f["discount"],
                             f["quantity"][1] + 1)
    got, used = _run(cols, filters, 3, 1, jit=True)
    assert used == 1 and got == want
    assert ops.jit_stats()["failures"] == 0, ops.jit_last_log()


def _random_case(g, n):
    n_cols = int(g.integers(1, 6))
    layout = LAYOUT_TRANSPOSED if g.random() < 0.3 else LAYOUT_NORMAL
    vals, cols = [], []
    for _ in range(n_cols):
        bw = int(g.choice([0, 1, 2, 3, 4, 6, 7, 8, 10, 12, 14, 16, 17, 24, 31, 32]))
        if bw == 32:
            v = g.integers(-2**31, 2**31, n, dtype=np.int64).astype(np.int32)
            base = 0
        else:
            base = int(g.integers(-(1 << 20), 1 << 20))
            v = (g.integers(0, 1 << bw, n, dtype=np.int64) + base).astype(np.int32) if bw else np.full(n, base, np.int32)
        vals.append(v)
        cols.append(EncodedColumn.uniform(v, bw=bw, base=base, layout=layout).to_device())
    n_f = int(g.integers(0, min(4, n_cols) + 1))
    fcols = g.permutation(n_cols)[:n_f]
    filters = []
    for c in fcols:
        q = np.sort(g.random(2))
        if g.random() < 0.3:  # a selective range
            q[1] = q[0] + (q[1] - q[0]) * 0.05
        lo, hi = (int(x) for x in np.quantile(vals[c], q))
        filters.append((int(c), lo, hi))
    r = g.random()
    if r < 0.2:
        a, b = -1, -1
    elif r < 0.6:
        a, b = int(g.integers(0, n_cols)), -1
    else:
        a, b = int(g.integers(0, n_cols)), int(g.integers(0, n_cols))
    return vals, cols, filters, a, b


@pytest.mark.parametrize("seed", range(24))
def test_jit_random_shapes(jit_on, seed):
    g = np.random.default_rng(1000 + seed)
    n = int(g.choice([1, 17, 1024, 1025, 40 * 1024 + 511, 300 * 1024]))
    vals, cols, filters, a, b = _random_case(g, n)
    want = _numpy(vals, filters, a, b)
    got_jit, used = _run(cols, filters, a, b, jit=True)
    got_gen, used_gen = _run(cols, filters, a, b, jit=False)
    assert used_gen == 0
    assert got_gen == want
    assert got_jit == want, (filters, a, b, [c.desc.bw for c in cols])
    assert ops.jit_stats()["failures"] == 0, ops.jit_last_log()


@pytest.mark.parametrize("bw", [2, 4, 6, 8, 10, 12, 14])
def test_jit_swar_filter_edges(jit_on, bw):
    """Filters that test several packed fields at once (4-bit and even widths
    up to 14): ranges below, across and above the column's domain, empty after
    clamping, single values, negative bases and a base so large that decoded
    values could wrap (then the per-row form runs); sparse_rows 32 forces the
    dense form on every filter."""
    g = np.random.default_rng(bw)
    n = 20 * 1024 + 77
    top = (1 << bw) - 1
    ops.set_tuning(TUNE_SPARSE_ROWS, 32)
    for base in (0, -123456, 2**31 - 1 - top, 2**31 - top // 2):
        f = g.integers(0, top + 1, n)
        vals = (f + base).astype(np.int64)
        vals = ((vals + 2**31) % 2**32 - 2**31).astype(np.int32)  # the decoder's wrap for the last base
        a = g.integers(-1000, 1000, n).astype(np.int32)
        cols = [EncodedColumn.uniform(vals, bw=bw, base=base).to_device(), EncodedColumn.uniform(a, bw=11, base=-1000)
                .to_device()]
        lo_v, hi_v = int(vals.min()), int(vals.max())
        ranges = [(lo_v, hi_v), (lo_v - 50, lo_v), (hi_v, hi_v + 50), (lo_v - 100, lo_v - 1), (hi_v + 1, hi_v + 9),
                  (lo_v + top // 3, lo_v + top // 2), (-2**31, 2**31 - 1), (int(vals[5]), int(vals[5]))]
        for lo, hi in ranges:
            lo, hi = min(max(lo, -2**31), 2**31 - 1), min(max(hi, -2**31), 2**31 - 1)
            for filters in ([(0, lo, hi)], [(0, lo, hi), (1, -500, 400)]):
                got, used = _run(cols, filters, 1, -1, jit=True)
                assert used == (1 if lo <= hi else 0), (bw, base, lo, hi)  # an empty range launches nothing
                sel = np.ones(n, bool)
                for c, l, h in filters:
                    v = [vals, a][c]
                    sel &= (v >= l) & (v <= h)
                assert got == int(a[sel].astype(np.int64).sum()), (bw, base, lo, hi)


@pytest.mark.parametrize("sparse_rows", [1, 4, 12, 32])
def test_jit_sparse_threshold_does_not_change_results(jit_on, sparse_rows):
    n = 500 * 1024 + 3
    t = datagen.lineorder_q11(n, seed=11)
    order = ["date", "discount", "quantity", "price"]
    cols = [EncodedColumn.uniform(t[k], bw=datagen.Q11_BITS[k]).to_device() for k in order]
    vals = [t[k] for k in order]
    for filters in ([(0, 366, 730), (1, 1, 3), (2, -2**31, 24)], [(2, 0, 40)], [(0, 0, 2000), (1, 0, 9)]):
        ops.set_tuning(TUNE_SPARSE_ROWS, sparse_rows)
        got, used = _run(cols, filters, 3, 1, jit=True)
        assert used == 1
        assert got == _numpy(vals, filters, 3, 1)


def test_jit_falls_back_where_it_does_not_apply(jit_on):
    n = 64 * 1024 + 5
    g = np.random.default_rng(7)
    a = g.integers(0, 1000, n).astype(np.int32)
    b = g.integers(0, 50, n).astype(np.int32)
    ua, ub = EncodedColumn.uniform(a, bw=10).to_device(), EncodedColumn.uniform(b, bw=6).to_device()
    # two ranges on one column
    got, used = _run([ua, ub], [(0, 100, 900), (0, 200, 950)], 1, -1, jit=True)
    assert used == 0 and got == _numpy([a, b], [(0, 100, 900), (0, 200, 950)], 1, -1)
    # a per-vector column
    pb = EncodedColumn.encode(b, 0, layout=LAYOUT_NORMAL).to_device()
    got, used = _run([ua, pb], [(0, 100, 900)], 1, 0, jit=True)
    assert used == 0 and got == _numpy([a, b], [(0, 100, 900)], 1, 0)
    # no column read at all
    got, used = _run([ua], [], -1, -1, jit=True)
    assert used == 0 and got == n
    # switched off
    got, used = _run([ua, ub], [(0, 100, 900)], 1, -1, jit=False)
    assert used == 0 and got == _numpy([a, b], [(0, 100, 900)], 1, -1)


def test_jit_unused_columns_are_not_read(jit_on):
    n = 100 * 1024
    g = np.random.default_rng(9)
    a = g.integers(0, 1 << 12, n).astype(np.int32)
    c = g.integers(0, 1 << 20, n).astype(np.int32)
    cols = [EncodedColumn.uniform(a, bw=12).to_device(), EncodedColumn.uniform(c, bw=20).to_device(),
            EncodedColumn.uniform(a, bw=12).to_device()]
    got, used = _run(cols, [(2, 10, 2000)], 1, -1, jit=True)
    assert used == 1 and got == _numpy([a, c, a], [(2, 10, 2000)], 1, -1)


# ------------------------------------------------------------ probe + group-by

def _q21_tables(n, seed, part_ids, supp_ids):
    import torch
    t = datagen.q21_tables(n, seed=seed, part_ids=part_ids, supp_ids=supp_ids)
    dev = {k: torch.from_numpy(v).cuda() for k, v in t.items()}
    ht_s = ops.build_pht(dev["s_suppkey"], supp_ids, filt=dev["s_region"], filter_eq=1)
    ht_p = ops.build_pht(dev["p_partkey"], part_ids, vals=dev["p_brand1"], filt=dev["p_category"], filter_eq=1)
    ht_d = ops.build_pht(dev["d_datekey"], datagen.N_DAYS, vals=dev["d_year"])
    return t, ht_s, ht_p, ht_d


def _probe_run(cols, probes, agg, ka, kb, mul, sub, ng, jit):
    ops.set_tuning(TUNE_JIT, 1 if jit else 0)
    before = _launches()
    res = ops.probe_groupby(cols, probes, agg, ka, kb, mul, sub, ng).cpu().numpy()
    ops.check_device_error()
    return res, _launches() - before


@pytest.mark.parametrize("n,part_ids,supp_ids", [(1, 1 << 10, 1 << 8), (5000, 1 << 12, 1 << 10),
                                                 ((1 << 20) + 77, 1 << 19, 1 << 17), (1 << 23, 1 << 19, 1 << 17)])
def test_jit_q21_against_oracle(jit_on, oracle, n, part_ids, supp_ids):
    t, ht_s, ht_p, ht_d = _q21_tables(n, 31, part_ids, supp_ids)
    names = ["lo_suppkey", "lo_partkey", "lo_orderdate", "lo_revenue"]
    cols = [EncodedColumn.uniform(t[k], bw=datagen.Q21_BITS[k]).to_device() for k in names]
    probes = [(0, ht_s, ht_s.numel(), 0, 1), (1, ht_p, ht_p.numel() // 2, 0, 2), (2, ht_d, ht_d.numel() // 2, 0, 2)]
    got, used = _probe_run(cols, probes, 3, 1, 2, 7, 1992, datagen.N_GROUPS, jit=True)
    assert used == 1
    want = oracle.probe_groupby(t["lo_suppkey"], t["lo_partkey"], t["lo_orderdate"], t["lo_revenue"],
                                ht_s.cpu().numpy(), ht_p.cpu().numpy(), ht_d.cpu().numpy())
    assert np.array_equal(got, want)
    assert ops.jit_stats()["failures"] == 0, ops.jit_last_log()


def _numpy_probe(keys, measure, probes_np, agg_vals, ka, kb, mul, sub, ng):
    """Probe + group-by semantics of fls_q21.cu probe_v1 with crystal-opt/join.cuh
    hashing, restated over numpy arrays (tables as int32 numpy arrays)."""
    n = measure.size
    sel = np.ones(n, bool)
    vals = {}
    for q, (col, ht, ln, kmin, kind) in enumerate(probes_np):
        d = (keys[col].astype(np.int64) - kmin).astype(np.int32).astype(np.int64)
        h = np.where((d >= 0) & (d < ln), d, np.fmod(d, ln))
        ok = h >= 0
        hc = np.where(ok, h, 0)
        if kind == 1:
            hit = ok & (ht[hc] != 0)
            v = np.zeros(n, np.int64)
        else:
            x, y = ht[2 * hc], ht[2 * hc + 1]
            hit = ok & ((x != 0) | (y != 0))
            v = y.astype(np.int64)
        sel &= hit
        vals[q] = v
    a, b = vals[ka][sel], vals[kb][sel]
    key = ((a * mul + (b - sub)) & 0xFFFFFFFF).astype(np.uint32).astype(np.int32).astype(np.int64)
    g = np.where((key >= 0) & (key < ng), key, np.fmod(key, ng))
    assert (g >= 0).all()
    res = np.zeros((ng, 2), np.int64)
    res32 = np.zeros(4 * ng, np.int32)
    m = measure[sel].astype(np.int64)
    np.add.at(res[:, 1], g, m)
    res32[4 * g] = b
    res32[4 * g + 1] = a
    sums = res[:, 1].astype(np.uint64).view(np.uint32).reshape(ng, 2)
    res32[2::4] = sums[:, 0].view(np.int32)
    res32[3::4] = sums[:, 1].view(np.int32)
    return res32


@pytest.fixture(params=[0, 1], ids=["staged", "late"])
def late_measure(request):
    from fastlanesgpu_b200._lib import TUNE_LATE_MEASURE
    ops.set_tuning(TUNE_LATE_MEASURE, request.param)
    yield request.param
    ops.set_tuning(TUNE_LATE_MEASURE, 1)  # the default


@pytest.mark.parametrize("seed", range(12))
def test_jit_probe_random_shapes(jit_on, late_measure, seed):
    import torch
    g = np.random.default_rng(500 + seed)
    n = int(g.choice([17, 1024, 3000, 50 * 1024 + 9, 200 * 1024]))
    n_probes = int(g.integers(1, 5))
    layout = LAYOUT_TRANSPOSED if g.random() < 0.3 else LAYOUT_NORMAL
    keys, cols, probes_np, probes = [], [], [], []
    ka = kb = None
    for q in range(n_probes):
        kind = 2 if (q == n_probes - 1 and ka is None) or g.random() < 0.5 else 1
        ln = int(g.choice([7, 300, 2556, 40000, 1 << 17, 1 << 20]))  # the largest go to global memory
        kmin = int(g.integers(0, 50))
        bw = int(max(1, int(np.ceil(np.log2(ln + kmin + 64)))))
        k = g.integers(kmin, min(kmin + ln + 40, 1 << bw), n).astype(np.int32)  # some keys wrap (modulo path)
        keys.append(k)
        cols.append(EncodedColumn.uniform(k, bw=bw, layout=layout).to_device())
        ht = np.zeros(ln if kind == 1 else 2 * ln, np.int32)
        present = g.random(ln) < g.choice([0.05, 0.3, 0.9])
        if kind == 1:
            ht[present] = 1 + np.nonzero(present)[0]
        else:
            ht[0::2][present] = 1 + np.nonzero(present)[0]
            ht[1::2][present] = g.integers(0, 6, int(present.sum()))
            ka = q if ka is None else ka
            kb = q
        probes_np.append((q, ht, ln, kmin, kind))
        probes.append((q, torch.from_numpy(ht).cuda(), ln, kmin, kind))
    measure = g.integers(-2**20, 2**20, n).astype(np.int32)
    keys.append(measure)
    cols.append(EncodedColumn.uniform(measure, bw=21, base=-2**20, layout=layout).to_device())
    agg = n_probes
    ng = 36
    want = _numpy_probe(keys, measure, probes_np, None, ka, kb, 6, 0, ng)
    got_jit, used = _probe_run(cols, probes, agg, ka, kb, 6, 0, ng, jit=True)
    got_gen, used_gen = _probe_run(cols, probes, agg, ka, kb, 6, 0, ng, jit=False)
    assert used == 1 and used_gen == 0
    assert np.array_equal(got_gen, want)
    assert np.array_equal(got_jit, want)
    assert ops.jit_stats()["failures"] == 0, ops.jit_last_log()


@pytest.mark.parametrize("ng,n", [(3, 300 * 1024 + 5), (8192, 1 << 20), (8193, 50 * 1024)])
def test_jit_probe_group_sums_in_shared_memory(jit_on, ng, n):
    """Per-CTA group-sum slots in shared memory against one global atomic per
    row and against numpy: 3 groups in 4 slots; 8192 and 8193 groups in 2048
    slots, where most groups find their slot held by another and add to
    their records directly.  Measures near +-2^31 make the slots' 32-bit low
    words carry and borrow on most rows."""
    import torch
    g = np.random.default_rng(ng)
    ln = 64 if ng == 3 else 16384
    ht = np.zeros(2 * ln, np.int32)
    present = g.random(ln) < 0.9
    ht[0::2][present] = 1 + np.nonzero(present)[0]
    ht[1::2][present] = g.integers(0, ng, int(present.sum()))
    k = g.integers(0, ln, n).astype(np.int32)
    big = g.integers(2**31 - 4096, 2**31, n)
    measure = np.where(g.random(n) < 0.5, big, -big - 1).astype(np.int64)
    measure = np.where(g.random(n) < 0.2, g.integers(-100, 100, n), measure).astype(np.int32)
    cols = [EncodedColumn.uniform(k, bw=int(np.log2(ln))).to_device(),
            EncodedColumn.uniform(measure, bw=32).to_device()]
    probes = [(0, torch.from_numpy(ht).cuda(), ln, 0, 2)]
    want = _numpy_probe([k, measure], measure, [(0, ht, ln, 0, 2)], None, 0, 0, 0, 0, ng)
    assert np.abs(want.reshape(ng, 4)[:, 2:].copy().view(np.int64)).max() > 2**33
    try:
        for gsm in (1, 0):
            ops.set_tuning(TUNE_GROUP_SMEM, gsm)
            got, used = _probe_run(cols, probes, 1, 0, 0, 0, 0, ng, jit=True)
            assert used == 1 and np.array_equal(got, want), gsm
        got, used = _probe_run(cols, probes, 1, 0, 0, 0, 0, ng, jit=False)
        assert used == 0 and np.array_equal(got, want)
    finally:
        ops.set_tuning(TUNE_GROUP_SMEM, 1)
    assert ops.jit_stats()["failures"] == 0, ops.jit_last_log()


def test_jit_probe_out_of_range_keys_flagged(jit_on):
    """Keys below keys_min hash to a negative slot: the row is dropped and the
    device error word is set, in the specialised kernel as in the general one."""
    import torch
    from fastlanesgpu_b200 import FlsError
    n = 8 * 1024
    t, ht_s, ht_p, ht_d = _q21_tables(n, 24, 1 << 12, 1 << 10)
    names = ["lo_suppkey", "lo_partkey", "lo_orderdate", "lo_revenue"]
    cols = [EncodedColumn.uniform(t[k], bw=datagen.Q21_BITS[k]).to_device() for k in names]
    probes = [(0, ht_s, ht_s.numel(), 5, 1), (1, ht_p, ht_p.numel() // 2, 0, 2), (2, ht_d, ht_d.numel() // 2, 0, 2)]
    before = _launches()
    ops.probe_groupby(cols, probes, 3, 1, 2, 7, 1992, datagen.N_GROUPS)
    assert _launches() - before == 1
    with pytest.raises(FlsError):
        ops.check_device_error()
    torch.cuda.synchronize()


@pytest.mark.parametrize("late", [0, 1])
def test_jit_row_phase_flags_only_rows_that_reach_the_probe(jit_on, late):
    """In the row phase a key with a negative remainder at a later probe sets
    the error word only when its row passed the probes before it, as in the
    reference's probe chain (a rejected row reads no further table).  Probe 0, a PHT_2 of 2^14 slots kept in
    global memory by a 1 KB table budget, rejects every third slot; probe 1's
    keys (keys_min 100) are 50 on exactly the rows probe 0 rejects: no flag and
    the restated records.  The same key on one row that probe 0 accepts: the
    flag is set, and that row is dropped."""
    import torch
    from fastlanesgpu_b200 import FlsError
    from fastlanesgpu_b200._lib import TUNE_LATE_MEASURE, TUNE_TABLE_KB
    g = np.random.default_rng(4242)
    n, l0, l1, ng = 8 * 1024 + 5, 1 << 14, 1000, 36
    slots0 = np.arange(l0)
    ht0 = np.zeros(2 * l0, np.int32)
    present0 = slots0 % 3 != 0
    ht0[0::2][present0] = 1 + slots0[present0]
    ht0[1::2][present0] = slots0[present0] % 5
    slots1 = np.arange(l1)
    ht1 = np.zeros(2 * l1, np.int32)
    present1 = g.random(l1) < 0.6
    ht1[0::2][present1] = 1 + slots1[present1]
    ht1[1::2][present1] = slots1[present1] % 7
    k0 = g.integers(0, l0, n).astype(np.int32)
    hit0 = present0[k0]
    k1 = np.where(hit0, g.integers(100, 1100, n), 50).astype(np.int32)
    measure = g.integers(-2**20, 2**20, n).astype(np.int32)
    probes_np = [(0, ht0, l0, 0, 2), (1, ht1, l1, 100, 2)]
    probes = [(q, torch.from_numpy(ht).cuda(), ln, kmin, kind) for q, ht, ln, kmin, kind in probes_np]
    m_col = EncodedColumn.uniform(measure, bw=21, base=-2**20).to_device()
    try:
        ops.set_tuning(TUNE_TABLE_KB, 1)
        ops.set_tuning(TUNE_LATE_MEASURE, late)
        cols = [EncodedColumn.uniform(k0, bw=14).to_device(), EncodedColumn.uniform(k1, bw=11).to_device(), m_col]
        want = _numpy_probe([k0, k1], measure, probes_np, None, 0, 1, 7, 0, ng)
        got, used = _probe_run(cols, probes, 2, 0, 1, 7, 0, ng, jit=True)
        assert used == 1 and np.array_equal(got, want)
        k1b = k1.copy()
        k1b[int(np.nonzero(hit0)[0][17])] = 50
        cols[1] = EncodedColumn.uniform(k1b, bw=11).to_device()
        want_b = _numpy_probe([k0, k1b], measure, probes_np, None, 0, 1, 7, 0, ng)
        assert not np.array_equal(want_b, want)
        got_b = ops.probe_groupby(cols, probes, 2, 0, 1, 7, 0, ng).cpu().numpy()
        with pytest.raises(FlsError):
            ops.check_device_error()
        assert np.array_equal(got_b, want_b)
    finally:
        ops.set_tuning(TUNE_TABLE_KB, 0)
        ops.set_tuning(TUNE_LATE_MEASURE, 1)  # the default
    assert ops.jit_stats()["failures"] == 0, ops.jit_last_log()


# ------------------------------------------------------------------ decode

@pytest.mark.parametrize("bw", [0, 1, 3, 8, 13, 16, 24, 27, 28, 31, 32])
@pytest.mark.parametrize("base", [0, -7, 2**31 - 5])
def test_jit_decode_sum_and_hbm(jit_on, oracle, bw, base):
    """Specialised decode-sum (32-bit partial sums with the base added once per
    vector when no value can wrap; per-value uint64 adds otherwise) and decode to
    HBM equal the general kernel and the oracle, on full and partial vectors."""
    n = 70 * 1024 + 333
    g = np.random.default_rng(bw * 7 + (base & 0xFF))
    packed = (g.integers(0, 1 << 32, n, dtype=np.uint64) & ((1 << bw) - 1)).astype(np.uint32)
    vals = (packed + np.uint32(base & 0xFFFFFFFF)).view(np.int32)  # wraps like the decoder does
    col = EncodedColumn.uniform(vals, bw=bw, base=base).to_device()
    want_sum = int(vals.view(np.uint32).astype(np.uint64).sum())
    for jit in (1, 0):
        ops.set_tuning(TUNE_JIT, jit)
        before = _launches()
        s = int(ops.query_aggregate(col).cpu()[0]) & 0xFFFFFFFFFFFFFFFF
        out = ops.unpack_global(col).cpu().numpy()[:n]
        ops.check_device_error()
        assert _launches() - before == (2 if jit else 0)
        assert s == want_sum, (jit, bw, base)
        assert np.array_equal(out, vals), (jit, bw, base)
    assert ops.jit_stats()["failures"] == 0, ops.jit_last_log()


def test_jit_decode_transposed_orders(jit_on):
    """Transposed uniform columns: stored order runs specialised, original order
    takes the general kernel; both agree with the host's untransposed values."""
    from fastlanesgpu_b200._lib import ORDER_ORIGINAL
    n = 9 * 1024 + 100
    vals = datagen.uniform_bits(n, 9, seed=77)
    col = EncodedColumn.uniform(vals, bw=9, layout=LAYOUT_TRANSPOSED).to_device()
    before = _launches()
    stored = ops.unpack_global(col).cpu().numpy()
    assert _launches() - before == 1
    orig = ops.unpack_global(col, order=ORDER_ORIGINAL).cpu().numpy()[:n]
    assert _launches() - before == 1
    assert np.array_equal(orig, vals)
    for v in range(n // 1024):
        assert np.array_equal(ops.untranspose(stored[v * 1024:(v + 1) * 1024].view(np.uint32)).view(np.int32),
                              vals[v * 1024:(v + 1) * 1024])
