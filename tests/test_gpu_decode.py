"""GPU parity: decode-to-HBM and decode-fused-sum through the C ABI against the
oracle and the reference's own decoders, for every scheme, bit width, layout
and edge case."""
import numpy as np
import pytest

from fastlanesgpu_b200 import (LAYOUT_NORMAL, LAYOUT_TRANSPOSED, ORDER_ORIGINAL, ORDER_STORED, EncodedColumn,
                               FlsError, datagen, ops)

pytestmark = pytest.mark.gpu


def _dev(col):
    return col.to_device()


def _pad(vals):
    n = vals.size
    nv = (n + 1023) // 1024
    out = np.empty(nv * 1024, np.int32)
    out[:n] = vals
    out[n:] = vals[-1]
    return out


def _np(t):
    return t.cpu().numpy()


@pytest.mark.parametrize("bw", range(33))
def test_uniform_for_every_bw(cuda, oracle, bw):
    n = 37 * 1024 + 123
    vals = datagen.uniform_bits(n, bw, seed=500 + bw)
    col = EncodedColumn.uniform(vals, bw=bw)
    d = _dev(col)
    out = _np(ops.unpack_global(d))
    assert np.array_equal(out, _pad(vals))
    # vector by vector, the oracle's unpack of the same words
    for vi in (0, 17, col.n_vec - 1):
        w = col.words[vi * 32 * bw:(vi + 1) * 32 * bw]
        assert np.array_equal(out[vi * 1024:(vi + 1) * 1024].view(np.uint32), oracle.unpack(w, bw))
    s = int(_np(ops.query_aggregate(d))[0])
    assert s == int(vals.view(np.uint32).astype(np.uint64).sum())
    ops.check_device_error()


@pytest.mark.parametrize("bw", range(33))
def test_reference_packed_fixture(cuda, golden, bw):
    """Words packed by the reference's pack.cpp decode to the seeded input."""
    x = datagen.uniform_bits(1024, bw, seed=1000 + bw)
    words = golden[f"pack_{bw}"]
    col = EncodedColumn(words=np.concatenate([words, np.zeros(4, np.uint32)]), meta=None, n_values=1024,
                        layout=LAYOUT_NORMAL, bw=bw)
    assert np.array_equal(_np(ops.unpack_global(col.to_device())), x)


def test_reference_delta_fixture(cuda, golden):
    """The reference's transposed delta vector (bases + packed deltas) decodes
    to its d_rsum_32 output (stored order) and to the input (original order)."""
    bw = int(golden["delta_bw"][0])
    words = np.concatenate([golden["delta_transposed"][:32], golden["delta_packed"]]).astype(np.uint32)
    col = EncodedColumn(words=words, meta=None, n_values=1024, layout=LAYOUT_TRANSPOSED, scheme=1, bw=bw)
    d = col.to_device()
    assert np.array_equal(_np(ops.unpack_global(d, ORDER_STORED)).view(np.uint32), golden["delta_rsum"])
    assert np.array_equal(_np(ops.unpack_global(d, ORDER_ORIGINAL)), datagen.sorted_geometric(1024, seed=77))


def test_config1_mixed_width_roundtrip(cuda, oracle):
    """2^20 values, per vector w in {3,7,11,16,21}, base U[0,2^20): unpack,
    un-FOR and sum; array and checksum bit-exact against the oracle."""
    vals = datagen.for_bitpack_mixed(1 << 20, seed=1)
    col = EncodedColumn.encode(vals, 0, layout=LAYOUT_NORMAL)
    d = col.to_device()
    out = _np(ops.unpack_global(d))
    ref = np.concatenate([oracle.decode_vec(col.words[m["offset"]:], _meta(oracle, m), transposed=False)
                          for m in col.meta])
    assert np.array_equal(out, ref)
    assert np.array_equal(out, vals)
    s = int(_np(ops.query_aggregate(d))[0]) & 0xFFFFFFFFFFFFFFFF
    assert s == int(vals.astype(np.int64).sum()) & 0xFFFFFFFFFFFFFFFF


def _meta(oracle, m):
    import oracle as orc
    om = orc.OrcVec()
    om.scheme, om.bw, om.aux, om.base = int(m["scheme"]), int(m["bw"]), int(m["aux"]), int(m["base"])
    return om


GENS = {
    "mixed": lambda n: datagen.for_bitpack_mixed(n, seed=31),
    "sorted": lambda n: datagen.sorted_geometric(n, seed=31),
    "runs": lambda n: datagen.geometric_runs(n, seed=31),
    "zipf": lambda n: datagen.zipf_values(n, seed=31),
    "neg": lambda n: np.random.default_rng(31).integers(-2**31, 2**31, n).astype(np.int32),
    "const": lambda n: np.full(n, -9, np.int32),
}


@pytest.mark.parametrize("gen", list(GENS))
@pytest.mark.parametrize("scheme", range(5))
@pytest.mark.parametrize("layout", [LAYOUT_NORMAL, LAYOUT_TRANSPOSED])
def test_schemes_decode(cuda, oracle, gen, scheme, layout):
    if scheme in (1, 2) and layout == LAYOUT_NORMAL:
        return
    n = 20 * 1024 + 77
    vals = GENS[gen](n)
    col = EncodedColumn.encode(vals, scheme, layout=layout)
    d = col.to_device()
    orig = _np(ops.unpack_global(d, ORDER_ORIGINAL))
    assert np.array_equal(orig, _pad(vals))
    stored = _np(ops.unpack_global(d, ORDER_STORED))
    if layout == LAYOUT_TRANSPOSED:
        pos = oracle.tpos()
        for vi in range(col.n_vec):
            want = np.empty(1024, np.int32)
            want[pos] = _pad(vals)[vi * 1024:(vi + 1) * 1024]
            assert np.array_equal(stored[vi * 1024:(vi + 1) * 1024], want)
    else:
        assert np.array_equal(stored, orig)
    s = int(_np(ops.query_aggregate(d))[0]) & 0xFFFFFFFFFFFFFFFF
    assert s == int(vals.view(np.uint32).astype(np.uint64).sum()) & 0xFFFFFFFFFFFFFFFF
    ops.check_device_error()


def test_mixed_schemes_in_one_column(cuda):
    parts = [datagen.sorted_geometric(4096, seed=1), datagen.geometric_runs(4096, seed=2),
             datagen.uniform_bits(4096, 13, seed=3), np.full(4096, 42, np.int32), datagen.zipf_values(4096, seed=4)]
    vals = np.concatenate(parts)
    schemes, _ = ops.encode_exhaustive(vals)[1], None
    col = EncodedColumn.encode(vals, schemes)
    assert len(set(col.meta["scheme"])) >= 4
    d = col.to_device()
    assert np.array_equal(_np(ops.unpack_global(d, ORDER_ORIGINAL)), vals)
    assert int(_np(ops.query_aggregate(d))[0]) == int(vals.view(np.uint32).astype(np.uint64).sum())


@pytest.mark.parametrize("n", [1, 31, 1023, 1024, 1025, 4096 * 37])
def test_sizes_and_tails(cuda, n):
    vals = datagen.uniform_bits(n, 11, seed=n)
    for col in (EncodedColumn.uniform(vals), EncodedColumn.encode(vals, 0),
                EncodedColumn.encode(vals, 4, layout=LAYOUT_TRANSPOSED)):
        d = col.to_device()
        assert np.array_equal(_np(ops.unpack_global(d, ORDER_ORIGINAL))[:n], vals)
        assert int(_np(ops.query_aggregate(d))[0]) == int(vals.view(np.uint32).astype(np.uint64).sum())


@pytest.mark.parametrize("cfg", [(1, 2, 1, 0), (2, 2, 2, 512), (4, 3, 1, 0), (8, 4, 1, 4096), (16, 2, 1, 16384), (16, 3, 1, 65536), (8, 2, 2, 2048)])
def test_launch_configs_agree(cuda, cfg):
    vals = datagen.for_bitpack_mixed(300 * 1024 + 5, seed=8)
    d = EncodedColumn.encode(vals, 0).to_device()
    try:
        ops.set_launch_config(*cfg)
        assert np.array_equal(_np(ops.unpack_global(d, ORDER_ORIGINAL))[:vals.size], vals)
        assert int(_np(ops.query_aggregate(d))[0]) == int(vals.view(np.uint32).astype(np.uint64).sum())
    finally:
        ops.set_launch_config(0, 0, 0, 0)


def test_bad_metadata_is_reported_not_read(cuda):
    """A vector whose metadata points past the data buffer is skipped and
    reported through the device error word (no out-of-bounds read)."""
    vals = datagen.uniform_bits(8 * 1024, 9, seed=2)
    col = EncodedColumn.encode(vals, 0)
    col.meta["offset"][5] = col.words.size  # outside the buffer
    col.meta["bw"][6] = 40                  # invalid bit width
    d = col.to_device()
    ops.query_aggregate(d)
    with pytest.raises(FlsError) as e:
        ops.check_device_error()
    assert "bad-vector-metadata" in str(e.value)
    ops.check_device_error()  # cleared


def test_argument_validation(cuda):
    vals = datagen.uniform_bits(2048, 9, seed=2)
    d = EncodedColumn.uniform(vals).to_device()
    d.desc.bw = 33
    with pytest.raises(FlsError):
        ops.unpack_global(d)
    d.desc.bw = 31  # larger than the data buffer allows
    with pytest.raises(FlsError):
        ops.query_aggregate(d)
