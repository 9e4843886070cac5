"""Selector statistics: the library's host statistics equal the oracle's."""
import numpy as np

from fastlanesgpu_b200 import datagen, ops
from fastlanesgpu_b200.selector import regret, training_corpus


def test_host_stats_equal_oracle(oracle):
    vals = training_corpus(64, seed=3)
    got = ops.vector_stats(vals)
    for v in range(64):
        assert np.array_equal(got[v], oracle.vector_stats(vals[v * 1024:(v + 1) * 1024])), v


def test_stats_edge_vectors(oracle):
    for vec in (np.full(1024, -2**31, np.int32), np.arange(1024, dtype=np.int32) * 2**20,
                np.random.default_rng(1).integers(-2**31, 2**31, 1024).astype(np.int32)):
        assert np.array_equal(ops.vector_stats(vec)[0], oracle.vector_stats(vec))


def test_regret_definition():
    sizes = np.array([[100, 50, 80, 0xFFFFFFFF, 90], [20, 40, 60, 16, 30]], np.uint32)
    assert regret(sizes, np.array([1, 3])) == 0.0
    assert abs(regret(sizes, np.array([0, 0])) - (120 / 66 - 1)) < 1e-12
    assert abs(regret(sizes, np.array([3, 3])) - (116 / 66 - 1)) < 1e-12  # CONST on a non-constant vector -> FOR
