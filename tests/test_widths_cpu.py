"""FastLanes packing of 8-, 16- and 64-bit lanes on the host
(fls_pack_u8/u16/u64, fls_unpack_*, fls_pack_column) against the oracle's
restatement and the reference's own packer (pack.cpp:29521, 29552, 29710,
compiled from its sources), for every bit width."""
import numpy as np
import pytest

from fastlanesgpu_b200 import FlsError, ops

WIDTHS = [(8, np.uint8), (16, np.uint16), (64, np.uint64)]


def _vec(g, dt):
    return g.integers(0, 2**63, 1024, dtype=np.uint64).astype(dt)


@pytest.mark.parametrize("bits,dt", WIDTHS)
def test_pack_equals_oracle_and_reference(oracle, reference, bits, dt):
    g = np.random.default_rng(bits)
    for bw in range(bits + 1):
        v = _vec(g, dt)
        got = ops.pack_vector(v, bw)
        want = np.zeros(1024 // bits * bw + 1, dt)
        getattr(oracle.L, f"orc_pack_{bits}")(v.ctypes.data, want.ctypes.data, bw)
        ref = np.zeros_like(want)
        getattr(reference.L, f"ref_pack_u{bits}")(v.ctypes.data, ref.ctypes.data, bw)
        assert np.array_equal(ref, want), bw
        assert np.array_equal(got, want[: got.size]), bw
        m = dt(~dt(0)) if bw == bits else dt((1 << bw) - 1)
        assert np.array_equal(ops.unpack_vector(got, bw), v & m), bw


@pytest.mark.parametrize("bits,dt", WIDTHS + [(32, np.uint32)])
def test_pack_column(bits, dt):
    g = np.random.default_rng(bits + 1)
    n, bw, base = 5 * 1024 + 77, min(bits - 1, 13), 3
    v = (g.integers(0, 1 << bw, n, dtype=np.uint64).astype(dt) + dt(base)).astype(dt)
    packed = ops.pack_column_width(v, bw, base)
    per = 1024 // bits * bw
    for k in range(6):
        vec = v[k * 1024:(k + 1) * 1024]
        if vec.size < 1024:
            vec = np.concatenate([vec, np.full(1024 - vec.size, v[-1], dt)])
        if bits == 32:
            continue
        assert np.array_equal(packed[k * per:(k + 1) * per], ops.pack_vector((vec - dt(base)).astype(dt), bw))
    with pytest.raises(FlsError):
        ops.pack_column_width(v, bw - 1, base)  # values need bw bits
    with pytest.raises(FlsError):
        ops.pack_vector(_vec(g, dt), bits + 1) if bits != 32 else ops.pack_column_width(v, 33)
