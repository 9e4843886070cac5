"""Learned encoding selection.

A 16-64-64-5 FP32 MLP, trained on the GPU by the library's own kernels
(fls_mlp_gradients / fls_mlp_adam_step), reads 16 per-vector statistics
(fls_vector_stats_gpu) and picks one of the five schemes for each 1024-value
vector.  The exhaustive encoder (fls_encode_exhaustive: exact size of every
scheme) produces the training labels, measures the selector's regret and is the
fallback for vectors whose top softmax probability is below a threshold.  The
encoder recomputes bit widths exactly for whatever scheme is picked, so the
encoded data is lossless regardless of the pick.
"""
from __future__ import annotations

import ctypes
import time

import numpy as np

from . import datagen
from ._lib import MLP_IN, MLP_N_PARAMS, check, lib
from .ops import encode_exhaustive

N_SCHEMES = 5

# Relative decode time per value of each scheme (FOR, DELTA, RLE, CONST, DICT),
# measured for decode fused with a sum over 2^28 values on B200: FOR 0.086 ms,
# DELTA 0.129 ms, RLE 0.168 ms, DICT 0.382 ms; CONST has no payload.
DECODE_COST = np.array([1.0, 1.5, 2.0, 1.0, 4.5])


def decode_aware_labels(sizes: np.ndarray, kappa: float = 0.0) -> np.ndarray:
    """Training labels from the exhaustive encoder's exact sizes (n x 5):
    argmin over schemes of size * (1 + kappa * (decode cost - 1)); kappa = 0
    is the smallest encoding (ties broken by decode cost)."""
    cost = sizes.astype(np.float64) * (1.0 + kappa * (DECODE_COST - 1.0))[None, :]
    cost[sizes == 0xFFFFFFFF] = np.inf
    order = np.argsort(DECODE_COST, kind="stable")  # cheapest decode first wins ties
    return order[np.argmin(cost[:, order], axis=1)].astype(np.uint8)


def _stream():
    import torch
    return torch.cuda.current_stream().cuda_stream


def gpu_features(values_dev) -> "torch.Tensor":
    """16 statistics per vector of a device int32 column (n_vec x 16 float32)."""
    import torch
    n = values_dev.numel()
    out = torch.empty(((n + 1023) // 1024, MLP_IN), dtype=torch.float32, device=values_dev.device)
    check(lib().fls_vector_stats_gpu(values_dev.data_ptr(), n, out.data_ptr(), _stream()), "fls_vector_stats_gpu")
    return out


def training_corpus(n_vectors: int, seed: int = 0) -> np.ndarray:
    """Vectors drawn from the four families of the mixed workload (uniform,
    Zipf, sorted-with-gaps, geometric runs) with randomised parameters, plus a
    few constant vectors, in segments of 1-16 vectors of one family."""
    g = np.random.default_rng(seed)
    parts, total = [], 0
    while total < n_vectors:
        k = int(min(g.integers(1, 17), n_vectors - total))
        n = k * 1024
        fam = int(g.integers(0, 5))
        s = int(g.integers(1 << 30))
        if fam == 0:
            bw = int(g.integers(1, 32))
            base = int(g.integers(-(1 << 20), 1 << 20))
            v = datagen.uniform_bits(n, bw, seed=s).astype(np.int64) % (1 << bw) + base
        elif fam == 1:
            v = datagen.zipf_values(n, s=float(g.uniform(1.05, 2.5)), domain=1 << int(g.integers(6, 24)), seed=s)
        elif fam == 2:
            v = datagen.sorted_geometric(n, p=float(g.uniform(0.02, 0.95)), seed=s).astype(np.int64)
            v = v + int(g.integers(-(1 << 20), 1 << 20))
        elif fam == 3:
            v = datagen.geometric_runs(n, mean_run=float(g.uniform(2.0, 96.0)), value_bits=int(g.integers(2, 25)),
                                       seed=s)
        else:
            v = np.full(n, int(g.integers(-1000, 1000)))
        parts.append(np.clip(np.asarray(v, dtype=np.int64), -2**31, 2**31 - 1).astype(np.int32))
        total += k
    return np.concatenate(parts)[: n_vectors * 1024]


def _zipf_cdf(s_values, n_ranks: int, device):
    """float64 CDFs of Zipf(s) truncated to ranks 1..n_ranks, one row per s."""
    import torch
    k = torch.arange(1, n_ranks + 1, dtype=torch.float64, device=device)
    w = k[None, :] ** (-torch.as_tensor(s_values, dtype=torch.float64, device=device)[:, None])
    c = torch.cumsum(w, dim=1)
    return c / c[:, -1:]


def corpus_device(n_vectors: int, seed: int = 0, device="cuda"):
    """Training vectors of the mixed workload's four families plus constant
    vectors, generated on `device` (int32 tensor of n_vectors * 1024 values,
    vectors shuffled): uniform values in [base, base + 2^w) with w in [1, 31];
    Zipf(s in [1.05, 2.5], truncated to 2^20 ranks) folded into [0, 2^[6, 24));
    sorted keys with geometric gaps (p in [0.02, 0.95]) from a random start;
    runs of geometric length (mean in [2, 96]) of values in [0, 2^[2, 25))."""
    import torch
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    dev = torch.device(device)

    def rnd(*shape):
        return torch.rand(*shape, generator=g, device=dev, dtype=torch.float64)

    def ints(lo, hi, *shape):
        return torch.randint(lo, hi, shape, generator=g, device=dev, dtype=torch.int64)

    fam = ints(0, 20, n_vectors)
    fam = torch.where(fam < 19, fam % 4, torch.full_like(fam, 4))  # 1 in 20 vectors constant
    out = torch.empty((n_vectors, 1024), dtype=torch.int32, device=dev)
    s_grid = torch.linspace(1.05, 2.5, 16, dtype=torch.float64)
    cdf = _zipf_cdf(s_grid, 1 << 20, dev)
    for f in range(5):
        idx = torch.nonzero(fam == f).flatten()
        k = int(idx.numel())
        if k == 0:
            continue
        if f == 0:
            w = ints(1, 32, k, 1)
            v = (ints(0, 1 << 32, k, 1024) & ((1 << w) - 1)) + ints(-(1 << 20), 1 << 20, k, 1)
        elif f == 1:
            which = ints(0, 16, k)
            u = rnd(k, 1024)
            v = torch.empty((k, 1024), dtype=torch.int64, device=dev)
            for j in range(16):
                rows = torch.nonzero(which == j).flatten()
                if rows.numel():
                    v[rows] = torch.searchsorted(cdf[j], u[rows].contiguous())
            v = v % (1 << ints(6, 24, k, 1))
        elif f == 2:
            p = 0.02 + 0.93 * rnd(k, 1)
            gaps = torch.floor(torch.log1p(-rnd(k, 1024)) / torch.log1p(-p)).to(torch.int64) + 1
            v = torch.cumsum(gaps, dim=1) + ints(-(1 << 20), 1 << 20, k, 1)
        elif f == 3:
            mean = 2.0 + 94.0 * rnd(k, 1)
            starts = rnd(k, 1024) < 1.0 / mean
            starts[:, 0] = True
            run = torch.cumsum(starts.to(torch.int64), dim=1) - 1
            vals = ints(0, 1 << 32, k, 1024) & ((1 << ints(2, 25, k, 1)) - 1)
            v = torch.gather(vals, 1, run)
        else:
            v = ints(-1000, 1000, k, 1).expand(k, 1024)
        out[idx] = torch.clamp(v, -2**31, 2**31 - 1).to(torch.int32)
    return out.reshape(-1)


class LearnedSelector:
    """The MLP parameters on a device plus training / selection."""

    def __init__(self, device=None, seed: int = 0):
        import torch
        self.device = torch.device("cuda") if device is None else torch.device(device)
        self.params = torch.empty(MLP_N_PARAMS, dtype=torch.float32, device=self.device)
        check(lib().fls_mlp_init(self.params.data_ptr(), seed, _stream()), "fls_mlp_init")

    # ------------------------------------------------------------- training
    def gradients(self, x, y):
        """(loss, grads) of one batch, both on the device."""
        import torch
        b = int(y.numel())
        ws_bytes = int(lib().fls_mlp_workspace_bytes(b))
        ws = torch.empty(ws_bytes, dtype=torch.uint8, device=self.device)
        grads = torch.empty(MLP_N_PARAMS, dtype=torch.float32, device=self.device)
        loss = torch.empty(1, dtype=torch.float32, device=self.device)
        check(lib().fls_mlp_gradients(self.params.data_ptr(), x.data_ptr(), y.data_ptr(), b, ws.data_ptr(), ws_bytes,
                                      grads.data_ptr(), loss.data_ptr(), _stream()), "fls_mlp_gradients")
        return loss, grads

    def train(self, feats, labels, epochs: int = 8, batch: int = 4096, lr: float = 3e-3, seed: int = 0):
        """Adam on device features (n x 16 float32) and labels (n uint8)."""
        import torch
        n = int(labels.numel())
        batch = min(batch, n)
        ws_bytes = int(lib().fls_mlp_workspace_bytes(batch))
        ws = torch.empty(ws_bytes, dtype=torch.uint8, device=self.device)
        grads = torch.empty(MLP_N_PARAMS, dtype=torch.float32, device=self.device)
        m = torch.zeros_like(grads)
        v = torch.zeros_like(grads)
        loss = torch.empty(1, dtype=torch.float32, device=self.device)
        gen = torch.Generator(device=self.device)
        gen.manual_seed(seed)
        losses, t = [], 0
        for ep in range(epochs):
            perm = torch.randperm(n, device=self.device, generator=gen)
            ep_loss = torch.zeros(1, dtype=torch.float32, device=self.device)
            steps = 0
            for s in range(0, n - batch + 1, batch):
                idx = perm[s:s + batch]
                xb = feats.index_select(0, idx).contiguous()
                yb = labels.index_select(0, idx).contiguous()
                check(lib().fls_mlp_gradients(self.params.data_ptr(), xb.data_ptr(), yb.data_ptr(), batch,
                                              ws.data_ptr(), ws_bytes, grads.data_ptr(), loss.data_ptr(), _stream()),
                      "fls_mlp_gradients")
                t += 1
                lr_t = lr * (0.5 * (1 + np.cos(np.pi * ep / max(1, epochs))))
                check(lib().fls_mlp_adam_step(self.params.data_ptr(), grads.data_ptr(), m.data_ptr(), v.data_ptr(),
                                              ctypes.c_float(lr_t), ctypes.c_float(0.9), ctypes.c_float(0.999),
                                              ctypes.c_float(1e-8), t, _stream()), "fls_mlp_adam_step")
                ep_loss += loss
                steps += 1
            losses.append(float(ep_loss.item()) / max(1, steps))
        return losses

    # ------------------------------------------------------------ inference
    def predict(self, feats):
        """(best scheme uint8, confidence float32) per row, on the device."""
        import torch
        n = feats.shape[0]
        best = torch.empty(n, dtype=torch.uint8, device=self.device)
        conf = torch.empty(n, dtype=torch.float32, device=self.device)
        check(lib().fls_mlp_infer(self.params.data_ptr(), feats.data_ptr(), n, 0, best.data_ptr(), conf.data_ptr(),
                                  _stream()), "fls_mlp_infer")
        return best, conf

    def select(self, values: np.ndarray, threshold: float = 0.9, values_dev=None, values_pinned=None):
        """Scheme per vector of a host column: the MLP's pick, or the exhaustive
        choice where the MLP's confidence is below `threshold`.  The column is
        uploaded from `values_pinned` (a pinned host tensor holding `values`)
        when given.  Returns (schemes, info) with the timing of each part."""
        import torch
        t0 = time.perf_counter()
        if values_dev is None:
            src = values_pinned if values_pinned is not None else torch.from_numpy(
                np.ascontiguousarray(values, dtype=np.int32))
            values_dev = src.to(self.device, non_blocking=values_pinned is not None)
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        feats = gpu_features(values_dev)
        best, conf = self.predict(feats)
        best_h, conf_h = best.cpu().numpy(), conf.cpu().numpy()
        t2 = time.perf_counter()
        low = np.nonzero(conf_h < threshold)[0]
        schemes = best_h.copy()
        if low.size:
            sub = np.concatenate([_vector(values, int(v)) for v in low])
            _, sub_best = encode_exhaustive(sub)
            schemes[low] = sub_best
        t3 = time.perf_counter()
        return schemes, {"upload_s": t1 - t0, "gpu_select_s": t2 - t1, "fallback_s": t3 - t2,
                         "fallback_vectors": int(low.size), "vectors": int(schemes.size)}

    def select_device(self, values_dev, values_host: np.ndarray, threshold: float = 0.9, kappa: float = 0.0):
        """Scheme per vector of a device column without leaving the device:
        the MLP's picks (device uint8), replaced by the exhaustive encoder's
        choice (computed on `values_host`, the same values, with the label rule
        of decode_aware_labels(kappa)) where the confidence is below
        `threshold`.  Returns (schemes_dev, info)."""
        import torch
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        best, conf = self.predict(gpu_features(values_dev))
        low = torch.nonzero(conf < threshold).flatten().cpu().numpy()
        t1 = time.perf_counter()
        if low.size:
            sub = np.concatenate([_vector(values_host, int(v)) for v in low])
            sub_sizes, _ = encode_exhaustive(sub)
            sub_best = decode_aware_labels(sub_sizes, kappa)
            best[torch.from_numpy(low).to(best.device)] = torch.from_numpy(sub_best).to(best.device)
        torch.cuda.synchronize()
        t2 = time.perf_counter()
        return best, {"gpu_select_s": t1 - t0, "fallback_s": t2 - t1, "fallback_vectors": int(low.size),
                      "vectors": int(best.numel())}

    def state(self) -> np.ndarray:
        return self.params.cpu().numpy()

    def load(self, params: np.ndarray) -> None:
        import torch
        assert params.size == MLP_N_PARAMS
        self.params.copy_(torch.from_numpy(np.ascontiguousarray(params, dtype=np.float32)))


def _vector(values: np.ndarray, v: int) -> np.ndarray:
    x = values[v * 1024:(v + 1) * 1024]
    if x.size < 1024:
        x = np.concatenate([x, np.full(1024 - x.size, x[-1], x.dtype)])
    return x


def chosen_sizes(sizes: np.ndarray, choice: np.ndarray) -> np.ndarray:
    """Encoded bytes of each vector under `choice` (a CONST pick on a
    non-constant vector is encoded as FOR, as the encoder does)."""
    got = sizes[np.arange(sizes.shape[0]), choice].astype(np.int64)
    bad = got == 0xFFFFFFFF
    got[bad] = sizes[np.nonzero(bad)[0], 0]
    return got


def regret(sizes: np.ndarray, choice: np.ndarray) -> float:
    """Encoded size of the choice over the exhaustive minimum, minus 1."""
    best = sizes.min(axis=1).astype(np.float64).sum()
    return float(chosen_sizes(sizes, choice).sum()) / best - 1.0
