"""Query specialisation without a GPU: NVRTC compiles the specialised
filter-aggregate kernel for the Q1.1 shape and for edge shapes, and queries
that do not qualify are refused with FLS_ERR_UNSUPPORTED."""
import pytest

from fastlanesgpu_b200 import FlsError, datagen, ops
from fastlanesgpu_b200._lib import LAYOUT_NORMAL, LAYOUT_TRANSPOSED, SCHEME_DELTA, SCHEME_FOR, Column

N = (1 << 20) + 7


def _col(bw, layout=LAYOUT_NORMAL, scheme=SCHEME_FOR, base=0):
    nv = (N + 1023) // 1024
    return Column(data=0x100000, meta=0, n_values=N, n_words=32 * bw * nv + 32 * nv, layout=layout, scheme=scheme,
                  bw=bw, base=base, max_vec_words=0, scheme_mask=1 << scheme)


def test_precompile_q11_shape():
    bits = datagen.Q11_BITS
    f = datagen.Q11_FILTER
    cols = [_col(bits[k]) for k in ("date", "discount", "quantity", "price")]
    before = ops.jit_stats()
    ops.jit_precompile(cols, [(0, *f["date"]), (1, *f["discount"]), (2, *f["quantity"])], 3, 1)
    after = ops.jit_stats()
    assert after["failures"] == before["failures"], ops.jit_last_log()
    assert after["cached"] >= 1


@pytest.mark.parametrize("bws,filters,a,b,layout", [
    ([0, 32], [(0, 0, 0), (1, -5, 5)], 1, 1, LAYOUT_NORMAL),
    ([1, 2, 3, 4, 5], [(0, 0, 0), (1, 0, 1), (2, 0, 2), (3, 0, 3)], 4, 0, LAYOUT_TRANSPOSED),
    ([17], [], 0, -1, LAYOUT_NORMAL),
    ([31, 9], [(1, 3, 300)], -1, -1, LAYOUT_TRANSPOSED),
])
def test_precompile_edge_shapes(bws, filters, a, b, layout):
    ops.jit_precompile([_col(x, layout) for x in bws], filters, a, b)
    assert ops.jit_stats()["failures"] == 0, ops.jit_last_log()


def test_precompile_refuses_unqualified_queries():
    with pytest.raises(FlsError) as e:
        ops.jit_precompile([_col(8, LAYOUT_TRANSPOSED, SCHEME_DELTA)], [(0, 1, 2)], 0, -1)
    assert e.value.status == 7
    with pytest.raises(FlsError) as e:
        ops.jit_precompile([_col(8), _col(9)], [(0, 1, 2), (0, 3, 4)], 1, -1)
    assert e.value.status == 7
    with pytest.raises(FlsError):
        ops.jit_precompile([_col(8)], [(3, 1, 2)], 0, -1)  # filter column out of range


def test_precompile_q21_probe_shape():
    bits = datagen.Q21_BITS
    cols = [_col(bits[k]) for k in ("lo_suppkey", "lo_partkey", "lo_orderdate", "lo_revenue")]
    probes = [(0, 0x200000, 1 << 17, 0, 1), (1, 0x400000, 1 << 19, 0, 2), (2, 0x800000, datagen.N_DAYS, 0, 2)]
    ops.jit_precompile_probe(cols, probes, 3, 1, 2, 7, 1992, datagen.N_GROUPS)
    assert ops.jit_stats()["failures"] == 0, ops.jit_last_log()


@pytest.mark.parametrize("probes,agg", [
    ([(0, 0x200000, 1000, 5, 2)], 0),                                   # measure = probed column
    ([(1, 0x200000, 70000, 0, 1), (0, 0x400000, 3000, 0, 2)], 2),       # global bitmap probe, smem PHT_2
    ([(0, 0x200000, 10, 0, 2), (1, 0x400000, 20, 1, 2), (2, 0x800000, 30, 2, 1), (3, 0xA00000, 40, 3, 2)], 4),
])
@pytest.mark.parametrize("half", [0, 1])
def test_precompile_probe_edge_shapes(probes, agg, half):
    """Probe shapes over bit widths 17, 3, 32, 0 and 9, with whole-vector and
    half-vector tiles (FLS_TUNE_HALF_VECTORS)."""
    from fastlanesgpu_b200._lib import TUNE_HALF_VECTORS
    cols = [_col(bw) for bw in (17, 3, 32, 0, 9)]
    ka = next(i for i, p in enumerate(probes) if p[4] == 2)
    try:
        ops.set_tuning(TUNE_HALF_VECTORS, half)
        ops.jit_precompile_probe(cols, probes, agg, ka, ka, 3, 1, 100)
    finally:
        ops.set_tuning(TUNE_HALF_VECTORS, 0)
    assert ops.jit_stats()["failures"] == 0, ops.jit_last_log()


def test_half_vector_tuning():
    """FLS_TUNE_HALF_VECTORS accepts 0 and 1 only and defaults to 0."""
    from fastlanesgpu_b200._lib import TUNE_HALF_VECTORS
    assert ops.get_tuning(TUNE_HALF_VECTORS) == 0
    for bad in (-1, 2):
        with pytest.raises(FlsError):
            ops.set_tuning(TUNE_HALF_VECTORS, bad)
    assert ops.get_tuning(TUNE_HALF_VECTORS) == 0


@pytest.mark.parametrize("half", [0, 1])
@pytest.mark.parametrize("query", ["q31", "q41"])
def test_precompile_ssb_join_shapes(query, half):
    if query == "q31":
        bits = datagen.Q31_BITS
        cols = [_col(bits[k]) for k in ("lo_suppkey", "lo_custkey", "lo_orderdate", "lo_revenue")]
        probes = [(0, 0x200000, 1 << 17, 0, 2), (1, 0x400000, 1 << 18, 0, 2), (2, 0x800000, datagen.N_DAYS, 0, 2)]
        kw = dict(agg_col=3, keys=[(0, 175, 2), (1, 7, 1), (2, 1, 0)], group_sub=1992, n_groups=4375, res_stride=6,
                  sum_slot=4)
    else:
        bits = datagen.Q41_BITS
        cols = [_col(bits[k]) for k in ("lo_suppkey", "lo_custkey", "lo_partkey", "lo_orderdate", "lo_revenue",
                                        "lo_supplycost")]
        probes = [(0, 0x200000, 1 << 17, 0, 1), (1, 0x400000, 1 << 18, 0, 2), (2, 0x600000, 1 << 19, 0, 1),
                  (3, 0x800000, datagen.N_DAYS, 0, 2)]
        kw = dict(agg_col=4, keys=[(1, 7, 1), (3, 1, 0)], group_sub=1992, n_groups=175, res_stride=4, sum_slot=2,
                  agg_sub_col=5)
    from fastlanesgpu_b200._lib import TUNE_HALF_VECTORS
    try:
        ops.set_tuning(TUNE_HALF_VECTORS, half)
        ops.jit_precompile_join(cols, probes, **kw)
    finally:
        ops.set_tuning(TUNE_HALF_VECTORS, 0)
    assert ops.jit_stats()["failures"] == 0, ops.jit_last_log()


def test_group_smem_tuning_and_shapes():
    """FLS_TUNE_GROUP_SMEM accepts 0 and 1 only; both settings compile their
    own specialised Q3.1 kernel (per-CTA group sums in shared memory or one
    global atomic per row)."""
    from fastlanesgpu_b200._lib import TUNE_GROUP_SMEM
    assert ops.get_tuning(TUNE_GROUP_SMEM) == 1
    with pytest.raises(FlsError):
        ops.set_tuning(TUNE_GROUP_SMEM, 2)
    bits = datagen.Q31_BITS
    cols = [_col(bits[k]) for k in ("lo_suppkey", "lo_custkey", "lo_orderdate", "lo_revenue")]
    probes = [(0, 0x200000, 1 << 17, 0, 2), (1, 0x400000, 1 << 18, 0, 2), (2, 0x800000, datagen.N_DAYS, 0, 2)]
    kw = dict(agg_col=3, keys=[(0, 175, 2), (1, 7, 1), (2, 1, 0)], group_sub=1992, n_groups=4375, res_stride=6,
              sum_slot=4)
    try:
        for gsm in (0, 1):
            ops.set_tuning(TUNE_GROUP_SMEM, gsm)
            before = ops.jit_stats()["cached"]
            ops.jit_precompile_join(cols, probes, **kw)
            assert ops.jit_stats()["failures"] == 0, ops.jit_last_log()
            assert ops.jit_stats()["cached"] >= before
    finally:
        ops.set_tuning(TUNE_GROUP_SMEM, 1)


def test_join_workspace_bytes():
    """The join workspace holds the presence bitmaps the specialised kernel
    stages: Q3.1 stages the supplier (2^17 slots) and customer (2^18) PHT_2
    bitmaps and the date table verbatim, 17400 words in all; a query whose
    tables all fit verbatim, or the general kernel (FLS_TUNE_JIT=0), needs none."""
    from fastlanesgpu_b200._lib import TUNE_JIT
    bits = datagen.Q31_BITS
    cols = [_col(bits[k]) for k in ("lo_suppkey", "lo_custkey", "lo_orderdate", "lo_revenue")]
    probes = [(0, 0x200000, 1 << 17, 0, 2), (1, 0x400000, 1 << 18, 0, 2), (2, 0x800000, datagen.N_DAYS, 0, 2)]
    kw = dict(agg_col=3, keys=[(0, 175, 2), (1, 7, 1), (2, 1, 0)], group_sub=1992, n_groups=4375, res_stride=6,
              sum_slot=4)
    assert ops.join_workspace_bytes(cols, probes, **kw) == 4 * (4096 + 8192 + 5112)
    small = [(0, 0x200000, 1000, 0, 2), (1, 0x400000, 2000, 0, 2), (2, 0x800000, datagen.N_DAYS, 0, 2)]
    assert ops.join_workspace_bytes(cols, small, **kw) == 0
    try:
        ops.set_tuning(TUNE_JIT, 0)
        assert ops.join_workspace_bytes(cols, probes, **kw) == 0
    finally:
        ops.set_tuning(TUNE_JIT, 1)


def test_table_budget_tuning():
    """FLS_TUNE_TABLE_KB bounds the shared memory of the join kernels' tables
    (default 72 KB, at most 144, 0 restores the default).  Q2.1 over the SSB
    schema (supplier PHT_1 of 2^17 slots, part PHT_2 of 2^19, date PHT_2 of
    2556): at 72 KB the supplier bitmap (4096 words) and the date table
    verbatim (5112) sit on chip and the part table stays in global memory; at
    144 KB the part presence bitmap (16384) sits between them, the workspace
    covers all three, and the kernel for that placement compiles."""
    from fastlanesgpu_b200._lib import TUNE_TABLE_KB
    assert ops.get_tuning(TUNE_TABLE_KB) == 72
    for bad in (-1, 145):
        with pytest.raises(FlsError):
            ops.set_tuning(TUNE_TABLE_KB, bad)
    bits = datagen.SSB_BITS
    cols = [_col(bits[k]) for k in ("lo_suppkey", "lo_partkey", "lo_orderdate", "lo_revenue")]
    probes = [(0, 0x200000, 1 << 17, 0, 1), (1, 0x400000, 1 << 19, 0, 2), (2, 0x800000, datagen.N_DAYS, 0, 2)]
    kw = dict(agg_col=3, keys=[(1, 7, 1), (2, 1, 0)], group_sub=1992, n_groups=7000, res_stride=4, sum_slot=2)
    try:
        assert ops.join_workspace_bytes(cols, probes, **kw) == 4 * (4096 + 5112)
        ops.set_tuning(TUNE_TABLE_KB, 144)
        assert ops.get_tuning(TUNE_TABLE_KB) == 144
        assert ops.join_workspace_bytes(cols, probes, **kw) == 4 * (4096 + 16384 + 5112)
        ops.jit_precompile_join(cols, probes, **kw)
        assert ops.jit_stats()["failures"] == 0, ops.jit_last_log()
        ops.set_tuning(TUNE_TABLE_KB, 0)
        assert ops.get_tuning(TUNE_TABLE_KB) == 72
    finally:
        ops.set_tuning(TUNE_TABLE_KB, 0)
