"""fls_mlp_gradients_static: the MLP gradient entry point for callers that
cannot allocate device memory themselves (a host engine that owns all device
memory through its own pool, or a loop that must not pay cudaMalloc's
device-wide synchronisation).  Its scratch is a fixed static device array of
the library, so the caller passes only parameters, inputs and outputs.

Checked through the C ABI against fls_mlp_gradients (which takes a caller
workspace) on two calls in a row, so a second call that reuses the shared
array still gives the same answer.  This file is named to be collected last."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MAX_BATCH = 2048  # FLS_MLP_STATIC_MAX_BATCH


def _stream():
    import torch
    return torch.cuda.current_stream().cuda_stream


def _with_workspace(L, params, x, y, b):
    import torch
    ws_bytes = int(L.fls_mlp_workspace_bytes(b))
    ws = torch.empty(ws_bytes, dtype=torch.uint8, device="cuda")
    grads = torch.empty(params.numel(), dtype=torch.float32, device="cuda")
    loss = torch.empty(1, dtype=torch.float32, device="cuda")
    assert L.fls_mlp_gradients(params.data_ptr(), x.data_ptr(), y.data_ptr(), b, ws.data_ptr(), ws_bytes,
                               grads.data_ptr(), loss.data_ptr(), _stream()) == 0
    return grads.cpu().numpy(), float(loss.item())


def _static(L, params, x, y, b):
    import torch
    grads = torch.empty(params.numel(), dtype=torch.float32, device="cuda")
    loss = torch.empty(1, dtype=torch.float32, device="cuda")
    st = L.fls_mlp_gradients_static(params.data_ptr(), x.data_ptr(), y.data_ptr(), b, grads.data_ptr(),
                                    loss.data_ptr(), _stream())
    assert st == 0, L.fls_last_error()
    return grads.cpu().numpy(), float(loss.item())


def test_static_scratch_gradients_match_workspace_version(cuda):
    import torch
    from fastlanesgpu_b200 import _lib
    L = _lib.lib()
    params = torch.empty(_lib.MLP_N_PARAMS, dtype=torch.float32, device="cuda")
    assert L.fls_mlp_init(params.data_ptr(), 5, _stream()) == 0
    g = np.random.default_rng(4)
    for call, b in enumerate((MAX_BATCH, 333)):  # two calls in a row; the second is smaller
        x = torch.from_numpy(g.random((b, 16), dtype=np.float32)).cuda()
        y = torch.from_numpy(g.integers(0, 5, b).astype(np.uint8)).cuda()
        want, want_loss = _with_workspace(L, params, x, y, b)
        got, got_loss = _static(L, params, x, y, b)
        # same tolerance as the gradient check against the oracle
        assert abs(got_loss - want_loss) <= 1e-4 * max(1.0, abs(want_loss)), call
        assert np.linalg.norm(got - want) <= 1e-4 * np.linalg.norm(want), call
        assert np.max(np.abs(got - want)) <= 1e-5 + 1e-3 * np.max(np.abs(want)), call


def test_static_scratch_rejects_oversized_batch(cuda):
    import torch
    from fastlanesgpu_b200 import _lib
    L = _lib.lib()
    params = torch.zeros(_lib.MLP_N_PARAMS, dtype=torch.float32, device="cuda")
    b = MAX_BATCH + 1
    x = torch.zeros((b, 16), dtype=torch.float32, device="cuda")
    y = torch.zeros(b, dtype=torch.uint8, device="cuda")
    grads = torch.empty(_lib.MLP_N_PARAMS, dtype=torch.float32, device="cuda")
    st = L.fls_mlp_gradients_static(params.data_ptr(), x.data_ptr(), y.data_ptr(), b, grads.data_ptr(), None,
                                    _stream())
    assert st == 8  # FLS_ERR_CAPACITY
    assert b"FLS_MLP_STATIC_MAX_BATCH" in L.fls_last_error()
