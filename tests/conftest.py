"""Test configuration: the `gpu` marker, and fixtures for the oracle (the CPU
restatement in oracle/) and the reference's own code (oracle/_ref)."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA sm_100 device (B200)")


@pytest.fixture(scope="session")
def oracle():
    import oracle as orc
    if not os.path.exists(orc.ORACLE_SO):
        orc.build(with_reference=False)
    return orc.Oracle()


@pytest.fixture(scope="session")
def reference():
    import oracle as orc
    if not os.path.exists(orc.REF_SO):
        try:
            orc.build(with_reference=True)
        except Exception:
            pass
    if not os.path.exists(orc.REF_SO):
        pytest.skip("reference library oracle/_ref/libflsref.so not built (needs the reference sources)")
    return orc.Reference()


@pytest.fixture(scope="session")
def golden():
    import numpy as np
    return dict(np.load(os.path.join(GOLDEN, "reference_pack.npz")))


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from fastlanesgpu_b200 import _lib, build
    if not os.path.exists(_lib.LIB_PATH):
        build.build()
    return torch.device("cuda:0")
