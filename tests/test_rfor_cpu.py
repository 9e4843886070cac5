"""The tile-based run-length format (RFOR, tile_based/src/rlebinpack.cpp) on
the host: the library's encoder, the oracle's restatement and the
reference's own rleBinPack (compiled from its source) write identical value
and run-length streams and tile offsets; the oracle's decoder restores the
input; 32-bit fields (where the reference shifts by 32) round-trip."""
import numpy as np
import pytest

from fastlanesgpu_b200 import datagen
from fastlanesgpu_b200.column import RforColumn


def _cases():
    g = np.random.default_rng(5)
    yield "geometric-runs", datagen.geometric_runs(100 * 512 + 37, seed=3)
    # the reference benchmark's pattern: runs of 8 alternating 200 / 300
    # (tile_based_bench_rle_all_memory.cu:237-251)
    yield "alternating", np.tile(np.repeat(np.array([200, 300], np.int32), 8), 2048)
    yield "short-runs", g.integers(0, 1000, 20 * 512).astype(np.int32)
    yield "constant", np.full(3000, 7, np.int32)
    yield "one-value", np.array([42], np.int32)
    yield "wide-values", g.integers(0, 2**30, 7 * 512 + 1).astype(np.int32)
    yield "negative", (datagen.geometric_runs(9 * 512, seed=4) - 100000).astype(np.int32)  # all below 0
    yield "sorted-keys", datagen.sorted_geometric(30 * 512, p=0.3, seed=5)


CASES = list(_cases())


@pytest.mark.parametrize("name,vals", CASES, ids=[c[0] for c in CASES])
def test_library_and_oracle_encoders_agree_and_round_trip(oracle, name, vals):
    want = oracle.rfor_encode(vals)
    col = RforColumn.encode(vals)
    for a, b in zip(want, (col.values, col.run_lengths, col.val_offsets, col.rl_offsets)):
        assert np.array_equal(a, b), name
    assert np.array_equal(oracle.rfor_decode(*want, vals.size), vals.view(np.uint32))


@pytest.mark.parametrize("name,vals", CASES, ids=[c[0] for c in CASES])
def test_oracle_encoder_equals_reference_rlebinpack(oracle, reference, name, vals):
    if not hasattr(reference.L, "ref_rfor_encode"):
        pytest.skip("reference library built without the RFOR encoder")
    for a, b in zip(oracle.rfor_encode(vals), reference.rfor_encode(vals)):
        assert np.array_equal(a, b), name


def test_header_and_block_layout(oracle):
    vals = np.repeat(np.array([5, 9, 5, 7], np.int32), [100, 300, 100, 12])  # one tile, 4 runs
    val, rl, vo, ro = oracle.rfor_encode(vals)
    assert list(val[:4]) == [512, 4, 512, 5] and list(rl[:4]) == [512, 4, 512, 5]
    assert vo[0] == 4 and ro[0] == 4
    # values: min 5, width 3 (9 - 5 = 4), count 4, fields 0, 4, 0, 2
    assert list(val[4:7]) == [5, 3 * 0x01010101, 4] and val[7] == (0 | 4 << 3 | 0 << 6 | 2 << 9)
    # lengths: min 12, width 9 (300 - 12 = 288), fields 88, 288, 88, 0
    assert list(rl[4:7]) == [12, 9 * 0x01010101, 4]
    assert vo[1] == val.size and ro[1] == rl.size


def test_full_width_fields_round_trip(oracle):
    """A tile whose values span more than 2^31 needs 32-bit fields (the
    reference's encoder shifts a 32-bit value by 32 there, which C++ leaves
    undefined); the library packs them as the format defines and decodes
    them back."""
    g = np.random.default_rng(9)
    vals = g.integers(-2**31, 2**31 - 1, 3 * 512).astype(np.int32)
    want = oracle.rfor_encode(vals)
    assert want[0][5] & 255 == 32
    col = RforColumn.encode(vals)
    assert np.array_equal(col.values, want[0]) and np.array_equal(col.run_lengths, want[1])
    assert np.array_equal(oracle.rfor_decode(*want, vals.size), vals.view(np.uint32))
