"""GPU decode of the tile-based run-length format (RFOR): decode to HBM
restores the input and decode fused with a sum gives its exact uint64 sum, for
ragged tails, 32-bit fields and the reference benchmark's pattern; a tile
whose block was damaged is skipped and reported through the error word while
the other tiles decode."""
import numpy as np
import pytest

from fastlanesgpu_b200 import FlsError, datagen, ops
from fastlanesgpu_b200.column import RforColumn

pytestmark = pytest.mark.gpu
M64 = (1 << 64) - 1


def _cases():
    g = np.random.default_rng(15)
    yield "geometric-runs", datagen.geometric_runs(300 * 512 + 77, seed=13)
    yield "alternating", np.tile(np.repeat(np.array([200, 300], np.int32), 8), 4096)
    yield "short-runs", g.integers(0, 3, 64 * 512).astype(np.int32)
    yield "all-distinct", g.integers(-2**31, 2**31 - 1, 40 * 512 + 3).astype(np.int32)
    yield "constant", np.full(5000, -3, np.int32)
    yield "one-value", np.array([42], np.int32)
    yield "sorted-keys", datagen.sorted_geometric(200 * 512, p=0.3, seed=14)


CASES = list(_cases())


@pytest.mark.parametrize("name,vals", CASES, ids=[c[0] for c in CASES])
def test_rfor_decode_and_sum(cuda, name, vals):
    d = RforColumn.encode(vals).to_device()
    out = ops.rfor_decode(d).cpu().numpy()
    ops.check_device_error()
    assert np.array_equal(out, vals), name
    s = int(ops.rfor_decode_sum(d).cpu()[0]) & M64
    ops.check_device_error()
    assert s == int(vals.view(np.uint32).astype(np.uint64).sum()) & M64, name


def test_damaged_block_is_flagged_and_skipped(cuda):
    vals = datagen.geometric_runs(20 * 512, seed=16)
    col = RforColumn.encode(vals)
    bad = 7
    col.values[col.val_offsets[bad] + 2] = 600  # run count above the tile's 512 values
    d = col.to_device()
    import torch
    out = torch.full((vals.size,), -1, dtype=torch.int32, device=cuda)
    ops.rfor_decode(d, out=out)
    with pytest.raises(FlsError) as e:
        ops.check_device_error()
    assert "bad-vector-metadata" in str(e.value)
    got = out.cpu().numpy()
    keep = np.ones(vals.size, bool)
    keep[bad * 512:(bad + 1) * 512] = False
    assert np.array_equal(got[keep], vals[keep]) and (got[~keep] == -1).all()


def _ref_gpu():
    import ctypes
    import os
    path = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref",
                        "libref_rfor_gpu.so")
    if not os.path.exists(path):
        pytest.skip("libref_rfor_gpu.so not built (make -C oracle dropin needs the reference sources)")
    return ctypes.CDLL(path)


@pytest.mark.parametrize("name", ["geometric-runs", "alternating", "short-runs", "constant", "sorted-keys"])
def test_reference_gpu_decoder_reads_the_same_streams(cuda, name):
    """The reference's own GPU decoder (LoadRBinPack) decodes the library's
    streams to the input, as the library's decoder does.  (Tiles whose value
    block exceeds 512 words -- 512 runs of 32-bit values -- are outside what
    the reference loader copies, rlebinpack_kernel.cuh:52-61, and are not used
    here.)"""
    import ctypes

    import torch
    L = _ref_gpu()
    vals = dict(CASES)[name]
    col = RforColumn.encode(vals)
    d = col.to_device()
    out = torch.zeros(vals.size, dtype=torch.int32, device=cuda)
    p = lambda t: ctypes.c_void_p(t.data_ptr())  # noqa: E731
    assert L.ref_rfor_decode_gpu(p(d.values), p(d.val_offsets), p(d.run_lengths), p(d.rl_offsets),
                                 ctypes.c_uint32(vals.size), p(out)) == 0
    assert np.array_equal(out.cpu().numpy(), vals), name
    assert np.array_equal(ops.rfor_decode(d).cpu().numpy(), vals)


def test_decode_time_against_reference_gpu_decoder(cuda):
    """Both decoders on 2^26 values of geometric runs (mean 16) of values in
    [0, 2^16): each result equals the input, and the CUDA-event time of each
    (20 launches after 5, on the default stream) is printed."""
    import ctypes

    import torch
    L = _ref_gpu()
    n = 1 << 26
    vals = datagen.geometric_runs(n, mean_run=16.0, value_bits=16, seed=2804)
    d = RforColumn.encode(vals).to_device()
    out = torch.empty(n, dtype=torch.int32, device=cuda)
    p = lambda t: ctypes.c_void_p(t.data_ptr())  # noqa: E731

    def ref():
        assert L.ref_rfor_decode_gpu_launch(p(d.values), p(d.val_offsets), p(d.run_lengths), p(d.rl_offsets),
                                            ctypes.c_uint32(n), p(out)) == 0

    def ours():
        ops.rfor_decode(d, out=out)
    ms = {}
    for name, f in (("reference LoadRBinPack", ref), ("fls_rfor_decode_u32", ours)):
        out.fill_(-1)
        for _ in range(5):
            f()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(20):
            f()
        e1.record()
        torch.cuda.synchronize()
        ms[name] = e0.elapsed_time(e1) / 20
        ops.check_device_error()
        assert torch.equal(out.cpu(), torch.from_numpy(vals)), name
    print("\nRFOR decode of 2^26 values to HBM, ms per launch:",
          ", ".join(f"{k} {v:.4f}" for k, v in ms.items()))
