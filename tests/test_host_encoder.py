"""The library's host encoders (C++) against the oracle: every encoded vector
is bit-identical to the oracle's encoding, and the host primitives equal the
reference's."""
import numpy as np
import pytest

from fastlanesgpu_b200 import EncodedColumn, datagen, ops

GENS = {
    "mixed": lambda n: datagen.for_bitpack_mixed(n, seed=9),
    "sorted": lambda n: datagen.sorted_geometric(n, seed=9),
    "runs": lambda n: datagen.geometric_runs(n, seed=9),
    "zipf": lambda n: datagen.zipf_values(n, seed=9),
    "const": lambda n: np.full(n, -3, np.int32),
    "neg": lambda n: np.random.default_rng(9).integers(-2**31, 2**31, n).astype(np.int32),
}


def _vec(vals, vi):
    v = vals[vi * 1024:(vi + 1) * 1024]
    return v if v.size == 1024 else np.concatenate([v, np.full(1024 - v.size, v[-1], np.int32)])


@pytest.mark.parametrize("bw", range(33))
def test_pack_equals_oracle(oracle, bw):
    x = datagen.uniform_bits(1024, bw, seed=bw).view(np.uint32)
    assert np.array_equal(ops.pack(x, bw), oracle.pack(x, bw))


def test_transpose_unrsum_rle_equal_oracle(oracle):
    x = datagen.sorted_geometric(1024).view(np.uint32)
    assert np.array_equal(ops.transpose_i(x), oracle.transpose_i(x))
    assert np.array_equal(ops.untranspose(ops.transpose_i(x)), x)
    assert np.array_equal(ops.unrsum(ops.transpose_i(x)), oracle.unrsum(oracle.transpose_i(x)))
    r = datagen.geometric_runs(1024, seed=3)
    a, b = ops.vector_rle(r), oracle.vector_rle(r)
    assert a[0] == b[0] and all(np.array_equal(u, v) for u, v in zip(a[1:], b[1:]))


@pytest.mark.parametrize("gen", list(GENS))
@pytest.mark.parametrize("scheme", range(5))
@pytest.mark.parametrize("layout", [0, 1])
def test_column_encoding_equals_oracle(oracle, gen, scheme, layout):
    if scheme in (1, 2) and layout == 0:
        return
    vals = GENS[gen](3 * 1024 + 517)
    col = EncodedColumn.encode(vals, scheme, layout=layout)
    assert col.words.size % 4 == 0
    for vi in range(col.n_vec):
        m = col.meta[vi]
        vec = _vec(vals, vi)
        p, om = oracle.encode_vec(vec, int(m["scheme"]), transposed=bool(layout))
        assert om.scheme == m["scheme"] and om.bw == m["bw"] and om.aux == m["aux"] and om.base == m["base"]
        assert int(m["offset"]) % 4 == 0
        assert np.array_equal(col.words[m["offset"]:m["offset"] + om.n_words], p)
        assert np.array_equal(oracle.decode_vec(p, om, transposed=bool(layout)), vec)
    if scheme == 3 and gen != "const":
        assert set(col.meta["scheme"]) <= {0, 3}  # CONST falls back to FOR on non-constant vectors


@pytest.mark.parametrize("gen", list(GENS))
def test_exhaustive_sizes_equal_oracle(oracle, gen):
    vals = GENS[gen](4 * 1024)
    sizes, best = ops.encode_exhaustive(vals)
    for vi in range(sizes.shape[0]):
        s = oracle.scheme_sizes(_vec(vals, vi))
        assert np.array_equal(sizes[vi], s)
        assert sizes[vi][best[vi]] == s.min()
    # the chosen encoding really has that size
    col = EncodedColumn.encode(vals, best)
    assert col.nbytes == int(sizes[np.arange(sizes.shape[0]), best].sum())


@pytest.mark.parametrize("bw", [0, 1, 7, 12, 24, 31, 32])
def test_uniform_encoding_equals_oracle(oracle, bw):
    vals = datagen.uniform_bits(2 * 1024 + 100, bw, seed=bw)
    col = EncodedColumn.uniform(vals, bw=bw)
    assert col.bw == bw
    for vi in range(col.n_vec):
        assert np.array_equal(col.words[vi * 32 * bw:(vi + 1) * 32 * bw], oracle.pack(_vec(vals, vi).view(np.uint32), bw))


def test_uniform_rejects_too_small_bw():
    from fastlanesgpu_b200 import FlsError
    with pytest.raises(FlsError):
        EncodedColumn.uniform(datagen.uniform_bits(1024, 12), bw=11)
