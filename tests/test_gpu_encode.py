"""GPU encoder (fls_encode_column_gpu) against the host encoder: identical
payload words and metadata for every scheme, layout, tail length, per-vector
scheme arrays and round-to-4 widths; the encoded column decodes back to the
input."""
import numpy as np
import pytest

from fastlanesgpu_b200 import LAYOUT_NORMAL, LAYOUT_TRANSPOSED, ORDER_ORIGINAL, EncodedColumn, FlsError, datagen, ops
from fastlanesgpu_b200.column import encode_column_gpu

pytestmark = pytest.mark.gpu


def _families(n, seed):
    g = np.random.default_rng(seed)
    return {
        "uniform": datagen.uniform_bits(n, int(g.integers(1, 33)), seed=seed),
        "negative": g.integers(-2**31, 2**31, n, dtype=np.int64).astype(np.int32),
        "zipf": datagen.zipf_values(n, s=1.1, domain=1 << 20, seed=seed),
        "sorted": datagen.sorted_geometric(n, p=0.3, seed=seed),
        "runs": datagen.geometric_runs(n, mean_run=16.0, value_bits=16, seed=seed),
        "few_distinct": g.integers(-3, 4, n).astype(np.int32),
        "constant": np.full(n, -77, np.int32),
    }


def _compare(vals, schemes, layout, round4=False):
    import torch
    host = EncodedColumn.encode(vals, schemes, layout=layout, round4=round4)
    sch = schemes if isinstance(schemes, int) else torch.from_numpy(np.ascontiguousarray(schemes, np.uint8)).cuda()
    dcol = encode_column_gpu(torch.from_numpy(vals).cuda(), sch, layout=layout, round4=round4)
    gpu = dcol.to_host()
    ops.check_device_error()
    assert gpu.payload_words == host.payload_words
    assert np.array_equal(gpu.words[:host.payload_words], host.words[:host.payload_words])
    assert np.array_equal(gpu.meta, host.meta)
    assert gpu.max_vec_words == host.max_vec_words and gpu.scheme_mask == host.scheme_mask
    order = ORDER_ORIGINAL if layout == LAYOUT_TRANSPOSED else 0
    assert np.array_equal(ops.unpack_global(dcol, order=order).cpu().numpy()[:vals.size], vals)


@pytest.mark.parametrize("n", [1, 1000, 1025, 20 * 1024 + 5])
@pytest.mark.parametrize("scheme", [0, 1, 2, 3, 4])
def test_gpu_encoder_every_scheme(cuda, n, scheme):
    for name, vals in _families(n, 1000 + n + scheme).items():
        _compare(vals, scheme, LAYOUT_TRANSPOSED)
        if scheme in (0, 3, 4):  # bit-packed codes exist in both row orders
            _compare(vals, scheme, LAYOUT_NORMAL)


@pytest.mark.parametrize("seed", range(4))
def test_gpu_encoder_per_vector_schemes(cuda, seed):
    g = np.random.default_rng(seed)
    parts = list(_families(4096, seed).values())
    vals = np.concatenate([parts[i] for i in g.integers(0, len(parts), 24)] + [parts[0][:333]])
    nv = (vals.size + 1023) // 1024
    _compare(vals, g.integers(0, 5, nv).astype(np.uint8), LAYOUT_TRANSPOSED)
    _, best = ops.encode_exhaustive(vals)
    _compare(vals, best, LAYOUT_TRANSPOSED)


def test_gpu_encoder_round4(cuda):
    vals = datagen.uniform_bits(9 * 1024 + 9, 13, seed=5)
    _compare(vals, 0, LAYOUT_NORMAL, round4=True)
    _compare(vals, 0, LAYOUT_TRANSPOSED, round4=True)


def test_gpu_encoder_bad_scheme_is_flagged(cuda):
    """An out-of-range per-vector scheme is encoded as FOR and reported in the
    device error word (no fault)."""
    import torch
    vals = datagen.uniform_bits(3 * 1024, 9, seed=6)
    sch = torch.tensor([0, 7, 0], dtype=torch.uint8, device="cuda")
    dcol = encode_column_gpu(torch.from_numpy(vals).cuda(), sch, layout=LAYOUT_TRANSPOSED)
    with pytest.raises(FlsError):
        ops.check_device_error()
    host = EncodedColumn.encode(vals, 0, layout=LAYOUT_TRANSPOSED)
    got = dcol.to_host()
    assert np.array_equal(got.words[:host.payload_words], host.words[:host.payload_words])


def test_container_columns_decode_on_gpu(cuda, tmp_path):
    """Columns written to an encoded-column container and read back (host
    encoder through a file; GPU encoder through bytes) decode to the original
    values on the GPU."""
    import torch
    from fastlanesgpu_b200.column import encode_column_gpu
    from fastlanesgpu_b200.selector import training_corpus
    vals = training_corpus(300, seed=21)[: 300 * 1024 - 17]
    _, best = ops.encode_exhaustive(vals)
    col = EncodedColumn.encode(vals, best, layout=LAYOUT_TRANSPOSED)
    p = tmp_path / "col.flsc"
    col.save(str(p))
    back = EncodedColumn.load(str(p))
    out = ops.unpack_global(back.to_device(), ORDER_ORIGINAL).cpu().numpy()[: vals.size]
    assert np.array_equal(out, vals)
    g = encode_column_gpu(torch.from_numpy(vals).cuda(), torch.from_numpy(best).cuda()).to_host()
    g2 = EncodedColumn.from_bytes(g.to_bytes())
    want = int(vals.view(np.uint32).astype(np.uint64).sum())
    assert int(ops.query_aggregate(g2.to_device()).cpu()[0]) & 0xFFFFFFFFFFFFFFFF == want
    ops.check_device_error()
