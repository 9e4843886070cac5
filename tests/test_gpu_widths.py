"""GPU decode of FastLanes columns of 8-, 16- and 64-bit lanes
(fls_decode_u8/u16/u64): every bit width, ragged tails, bases that wrap
modulo 2^T, decode to HBM and decode fused with a sum, against numpy on the
same values; a 2^26-value column per width for the full-size sums."""
import numpy as np
import pytest

from fastlanesgpu_b200 import ops

pytestmark = pytest.mark.gpu

WIDTHS = [(8, np.uint8), (16, np.uint16), (64, np.uint64)]


def _column(g, dt, bits, bw, n, base):
    hi = (1 << bw) if bw < 64 else 1 << 64
    raw = g.integers(0, 2**64 - 1, n, dtype=np.uint64, endpoint=True)
    if bw < 64:
        raw &= np.uint64(hi - 1)
    return (raw.astype(dt) + dt(base & ((1 << bits) - 1))).astype(dt)


def _run(v, dt, bits, bw, base, want_out=True, want_sum=True):
    import torch
    packed = ops.pack_column_width(v, bw, base)
    dev = torch.from_numpy(packed.view(np.uint8).copy()).cuda()
    out, total = ops.decode_width(dev, v.size, bits, bw, base, out=None if want_out else False, want_sum=want_sum)
    ops.check_device_error()
    return out, total


@pytest.mark.parametrize("bits,dt", WIDTHS)
def test_decode_every_bit_width(cuda, bits, dt):
    g = np.random.default_rng(bits)
    n = 7 * 1024 + 333
    for bw in sorted({0, 1, 2, 3, bits // 2 - 1, bits // 2, bits - 3, bits - 1, bits}):
        base = int(g.integers(0, 1 << min(bits, 62)))
        v = _column(g, dt, bits, bw, n, base)
        out, total = _run(v, dt, bits, bw, base)
        pad = np.concatenate([v, np.full((-n) % 1024, v[-1], dt)])
        assert np.array_equal(out.cpu().numpy().view(dt), pad), bw
        assert total == int(v.astype(np.uint64).sum(dtype=np.uint64)), bw


@pytest.mark.parametrize("bits,dt", WIDTHS)
def test_decode_only_and_sum_only(cuda, bits, dt):
    g = np.random.default_rng(100 + bits)
    v = _column(g, dt, bits, bits - 2, 3000, 7)
    out, total = _run(v, dt, bits, bits - 2, 7, want_sum=False)
    assert total is None and np.array_equal(out.cpu().numpy().view(dt)[:3000], v)
    out, total = _run(v, dt, bits, bits - 2, 7, want_out=False)
    assert out is None and total == int(v.astype(np.uint64).sum(dtype=np.uint64))


@pytest.mark.parametrize("bits,dt", WIDTHS)
def test_full_size_sums(cuda, bits, dt):
    g = np.random.default_rng(200 + bits)
    n = 1 << 26
    bw = {8: 5, 16: 11, 64: 37}[bits]
    v = _column(g, dt, bits, bw, n, 1)
    _, total = _run(v, dt, bits, bw, 1, want_out=False)
    assert total == int(v.astype(np.uint64).sum(dtype=np.uint64))


@pytest.mark.parametrize("bits,dt", WIDTHS[:2])
def test_sum_only_every_bit_width(cuda, bits, dt):
    """The sum alone, at every bit width, with a base whose values do not wrap
    (summed without the per-value base) and one whose values do."""
    g = np.random.default_rng(300 + bits)
    n = 5 * 1024 + 77
    for bw in range(0, bits + 1):
        top = (1 << bits) - (1 << bw)  # the largest base with no wrap
        for base in sorted({0, top, min(top + 1, (1 << bits) - 1), int(g.integers(0, 1 << bits))}):
            v = _column(g, dt, bits, bw, n, base)
            _, total = _run(v, dt, bits, bw, base, want_out=False)
            assert total == int(v.astype(np.uint64).sum(dtype=np.uint64)), (bw, base)
