"""The C-ABI library loads, exports every entry point include/fls_gpu.h
declares, and reports argument errors as status codes (no GPU needed)."""
import ctypes
import os
import re

import numpy as np
import pytest

from conftest import ROOT
from fastlanesgpu_b200 import _lib


def _declared():
    src = open(os.path.join(ROOT, "include", "fls_gpu.h")).read()
    return sorted(set(re.findall(r"^\s*(?:[\w\s\*]+?)\b(fls_\w+)\(", src, re.M)))


def test_header_declarations_exported():
    L = _lib.lib()
    names = _declared()
    assert len(names) >= 20
    for n in names:
        assert hasattr(L, n), n
    assert set(names) <= set(_lib.declared_symbols()) | {"fls_last_error"}


def test_argument_errors_are_status_codes():
    L = _lib.lib()
    x = np.zeros(1024, np.uint32)
    out = np.zeros(32 * 33, np.uint32)
    assert L.fls_pack_u32(x.ctypes.data, out.ctypes.data, 33) == 2
    assert b"bit width" in L.fls_last_error()
    assert L.fls_pack_u32(None, out.ctypes.data, 3) == 1
    assert L.fls_set_launch_config(99, 3, 1, 0) == 1
    assert L.fls_decode_u32(None, None, 0, None) == 1


def test_device_calls_without_device_fail_cleanly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is present")
    L = _lib.lib()
    col = _lib.Column(data=0, meta=0, n_values=1024, n_words=0, layout=0, scheme=0, bw=0, base=0)
    st = L.fls_decode_sum_u32(ctypes.byref(col), ctypes.c_void_p(16), None)
    assert st == 9  # FLS_ERR_NO_DEVICE
