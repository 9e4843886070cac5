"""Batched persistent execution: many filter-aggregate queries over many
columns of uneven length and bit width in one launch (fls_batch_* in
include/fls_gpu.h), replayable as a CUDA graph."""
from __future__ import annotations

import ctypes

from ._lib import BatchQuery, check, lib
from .column import columns_array


def _stream():
    import torch
    return torch.cuda.current_stream().cuda_stream


class Batch:
    """A planned batch: the column descriptors, the queries and the work items
    live in a device workspace owned by this object."""

    def __init__(self, cols, queries, chunk_vectors: int = 64):
        import torch
        self.cols = cols  # keep the device columns alive
        self._arr = columns_array(cols)
        q = (BatchQuery * len(queries))()
        for i, (c, lo, hi, a) in enumerate(queries):
            q[i].col, q[i].lo, q[i].hi, q[i].agg_col = c, lo, hi, a
        self.n_queries = len(queries)
        h = ctypes.c_void_p()
        check(lib().fls_batch_create(self._arr, len(cols), q, len(queries), chunk_vectors, ctypes.byref(h)),
              "fls_batch_create")
        self._h = h
        nbytes = int(lib().fls_batch_workspace_bytes(h))
        self.workspace = torch.empty(nbytes, dtype=torch.uint8, device=cols[0].data.device)
        check(lib().fls_batch_upload(h, self.workspace.data_ptr(), nbytes, _stream()), "fls_batch_upload")
        self.results = torch.zeros(2 * len(queries), dtype=torch.int64, device=cols[0].data.device)

    @property
    def n_items(self) -> int:
        return int(lib().fls_batch_items(self._h))

    def run(self):
        """Enqueue the whole batch; returns the device int64[n_queries, 2]
        {sum, count} tensor (overwritten by every run)."""
        check(lib().fls_batch_run(self._h, self.results.data_ptr(), _stream()), "fls_batch_run")
        return self.results.view(self.n_queries, 2)

    def close(self) -> None:
        if getattr(self, "_h", None):
            lib().fls_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def graph_of(fn):
    """Capture `fn` (which only enqueues device work) into a CUDA graph;
    returns the graph, replayed with .replay()."""
    import torch
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        fn()  # warm-up outside the capture (lazy attribute setup)
    torch.cuda.current_stream().wait_stream(s)
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        fn()
    return g
