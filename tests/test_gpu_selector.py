"""GPU: selector statistics, MLP gradients against the double-precision
oracle, training, regret against the exhaustive encoder, and the gain over the
method without the network."""
import numpy as np
import pytest

from fastlanesgpu_b200 import EncodedColumn, ORDER_ORIGINAL, ops
from fastlanesgpu_b200.selector import LearnedSelector, gpu_features, regret, training_corpus

pytestmark = pytest.mark.gpu


def test_gpu_stats_bit_exact(cuda):
    import torch
    vals = training_corpus(300, seed=5)[: 300 * 1024 - 77]
    got = gpu_features(torch.from_numpy(vals).cuda()).cpu().numpy()
    assert np.array_equal(got, ops.vector_stats(vals))


def test_mlp_gradients_match_oracle(cuda, oracle):
    import torch
    sel = LearnedSelector(seed=7)
    g = np.random.default_rng(0)
    x = g.random((256, 16), dtype=np.float32)
    y = g.integers(0, 5, 256).astype(np.uint8)
    loss, grads = sel.gradients(torch.from_numpy(x).cuda(), torch.from_numpy(y).cuda())
    want_loss, want = oracle.mlp_loss_grad(sel.state(), x, y)
    assert abs(float(loss.item()) - want_loss) < 1e-4 * max(1.0, abs(want_loss))
    got = grads.cpu().numpy().astype(np.float64)
    # FP32 sums over 256 samples vs FP64: relative error on the gradient vector
    assert np.linalg.norm(got - want) <= 1e-4 * np.linalg.norm(want)
    assert np.max(np.abs(got - want)) <= 1e-5 + 1e-3 * np.max(np.abs(want))


@pytest.fixture(scope="module")
def trained(cuda):
    import torch
    train = training_corpus(1 << 15, seed=11)
    sizes, labels = ops.encode_exhaustive(train)
    sel = LearnedSelector(seed=1)
    feats = gpu_features(torch.from_numpy(train).cuda())
    losses = sel.train(feats, torch.from_numpy(labels).cuda(), epochs=30, batch=2048, lr=3e-3)
    return sel, losses


def test_training_reduces_loss(trained):
    _, losses = trained
    assert losses[-1] < 0.5 * losses[0]


def test_learned_selection_regret_and_gain(trained):
    """Held-out columns: the network's picks (with the exhaustive fallback for
    low-confidence vectors) stay within 2% of the exhaustive size; without the
    network -- bit-packing everything (the reference's choice) or an untrained
    network -- the encoding is far larger."""
    import torch
    sel, _ = trained
    test = training_corpus(1 << 13, seed=99)
    sizes, best = ops.encode_exhaustive(test)
    schemes, info = sel.select(test, threshold=0.9)
    pure, conf = sel.predict(gpu_features(torch.from_numpy(test).cuda()))
    pure = pure.cpu().numpy()
    r_learned = regret(sizes, schemes)
    r_pure = regret(sizes, pure)
    r_for = regret(sizes, np.zeros_like(best))
    r_untrained = regret(sizes, LearnedSelector(seed=2).predict(gpu_features(torch.from_numpy(test).cuda()))[0]
                         .cpu().numpy())
    assert r_learned <= 0.02, (r_learned, info)
    assert info["fallback_vectors"] <= 0.25 * info["vectors"]
    assert r_pure < r_for and r_pure < r_untrained
    assert r_for > 0.10
    assert (pure == best).mean() > 0.85


def test_learned_encoding_is_lossless(trained):
    sel, _ = trained
    vals = training_corpus(200, seed=123)
    schemes, _ = sel.select(vals, threshold=0.0)
    col = EncodedColumn.encode(vals, schemes)
    out = ops.unpack_global(col.to_device(), ORDER_ORIGINAL).cpu().numpy()
    assert np.array_equal(out, vals)


@pytest.mark.parametrize("kappa", [0.0, 0.03])
def test_device_exhaustive_choice_equals_host(cuda, kappa):
    """fls_encode_learned_gpu with every vector below the confidence
    threshold: the device's exhaustive choice equals the host exhaustive
    encoder's sizes under the selector's label rule, on a ragged column of every
    family (constant vectors included), and the column decodes losslessly."""
    import torch
    from fastlanesgpu_b200.column import encode_column_learned_gpu
    from fastlanesgpu_b200.selector import decode_aware_labels
    vals = training_corpus(3000, seed=31)[: 3000 * 1024 - 333]
    sizes, _ = ops.encode_exhaustive(vals)
    want = decode_aware_labels(sizes, kappa)
    assert {0, 1, 2, 4} <= set(want.tolist())  # constant vectors tie FOR at 16 B and take FOR
    params = LearnedSelector(seed=3).params
    col, schemes, n_fb = encode_column_learned_gpu(torch.from_numpy(vals).cuda(), params, threshold=2.0, kappa=kappa)
    ops.check_device_error()
    assert n_fb == want.size
    assert np.array_equal(schemes.cpu().numpy(), want)
    out = ops.unpack_global(col, ORDER_ORIGINAL).cpu().numpy()[: vals.size]
    assert np.array_equal(out, vals)


def test_device_learned_encoder_equals_select_device(trained):
    """The one-call device encoder gives the same schemes and the same encoded
    column as the selector's device path (network picks, host exhaustive
    fallback) followed by the GPU encoder; threshold 0 keeps every pick."""
    import torch
    from fastlanesgpu_b200.column import encode_column_gpu, encode_column_learned_gpu
    sel, _ = trained
    vals = training_corpus(1500, seed=77)[: 1500 * 1024 - 5]
    dv = torch.from_numpy(vals).cuda()
    want, info = sel.select_device(dv, vals, threshold=0.9, kappa=0.03)
    col, schemes, n_fb = encode_column_learned_gpu(dv, sel.params, threshold=0.9, kappa=0.03)
    ops.check_device_error()
    assert n_fb == info["fallback_vectors"] > 0
    assert torch.equal(schemes, want)
    ref = encode_column_gpu(dv, want)
    assert col.payload_words == ref.payload_words
    assert torch.equal(col.data[: col.payload_words], ref.data[: ref.payload_words])
    assert torch.equal(col.meta, ref.meta)
    picks, _ = sel.predict(gpu_features(dv))
    _, schemes0, n0 = encode_column_learned_gpu(dv, sel.params, threshold=0.0)
    assert n0 == 0 and torch.equal(schemes0, picks)
