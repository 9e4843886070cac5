"""Decode fused with a sum for columns whose vectors share one scheme (the
scheme-specialised operators of fls_decode_sum_u32): DELTA, RLE and DICT
columns give the exact uint64 sum of their values -- against numpy on the
input and against the general per-vector operator (FLS_TUNE_JIT=0) -- for
ragged tails, negative bases, values above 2^27 (64-bit lane sums) and below
(32-bit lane sums), one-entry dictionaries and 32-bit dictionary values."""
import numpy as np
import pytest

from fastlanesgpu_b200 import LAYOUT_TRANSPOSED, SCHEME_DELTA, SCHEME_DICT, SCHEME_RLE, EncodedColumn, datagen, ops
from fastlanesgpu_b200._lib import TUNE_JIT

pytestmark = pytest.mark.gpu
M64 = (1 << 64) - 1


def _cases():
    g = np.random.default_rng(77)
    n = 37 * 1024 + 411
    yield "delta-sorted", SCHEME_DELTA, datagen.sorted_geometric(n, p=0.3, seed=5)
    yield "delta-big", SCHEME_DELTA, np.sort(g.integers(-2**31, 2**31 - 1, n)).astype(np.int32)
    yield "delta-unsorted", SCHEME_DELTA, g.integers(-2**31, 2**31 - 1, n).astype(np.int32)
    yield "rle-small", SCHEME_RLE, datagen.geometric_runs(n, mean_run=16.0, value_bits=16, seed=6)
    yield "rle-big", SCHEME_RLE, (datagen.geometric_runs(n, mean_run=9.0, value_bits=20, seed=7).astype(np.int64)
                                  * 3000 - 2**31 + 5).astype(np.int32)
    yield "rle-const", SCHEME_RLE, np.full(n, 123456789, np.int32)
    yield "dict-zipf", SCHEME_DICT, datagen.zipf_values(n, s=1.1, domain=1 << 20, seed=8)
    yield "dict-wide", SCHEME_DICT, g.choice(g.integers(-2**31, 2**31 - 1, 900), n).astype(np.int32)
    yield "dict-one", SCHEME_DICT, np.full(n, -7, np.int32)
    full = np.arange(1024, dtype=np.int32) * 4099 + 2**30  # 1024 distinct values in every vector
    yield "dict-1024", SCHEME_DICT, np.concatenate([g.permutation(full) for _ in range(n // 1024 + 1)])[:n]


CASES = list(_cases())


@pytest.mark.parametrize("name,scheme,vals", CASES, ids=[c[0] for c in CASES])
def test_single_scheme_sum(cuda, name, scheme, vals):
    col = EncodedColumn.encode(vals, scheme, layout=LAYOUT_TRANSPOSED)
    assert col.scheme_mask == 1 << scheme
    d = col.to_device()
    want = int(vals.view(np.uint32).astype(np.uint64).sum()) & M64
    try:
        for jit in (1, 0):
            ops.set_tuning(TUNE_JIT, jit)
            got = int(ops.query_aggregate(d).cpu()[0]) & M64
            ops.check_device_error()
            assert got == want, (name, jit)
    finally:
        ops.set_tuning(TUNE_JIT, 1)


@pytest.mark.parametrize("scheme,gen", [(SCHEME_DELTA, lambda n: datagen.sorted_geometric(n, seed=9)),
                                        (SCHEME_RLE, lambda n: datagen.geometric_runs(n, seed=10)),
                                        (SCHEME_DICT, lambda n: datagen.zipf_values(n, seed=11))])
@pytest.mark.parametrize("n", [1, 1023, 1025, 5 * 1024 + 17])
def test_single_scheme_sum_tails(cuda, scheme, gen, n):
    vals = gen(n)
    d = EncodedColumn.encode(vals, scheme, layout=LAYOUT_TRANSPOSED).to_device()
    assert int(ops.query_aggregate(d).cpu()[0]) & M64 == int(vals.view(np.uint32).astype(np.uint64).sum()) & M64
    ops.check_device_error()
