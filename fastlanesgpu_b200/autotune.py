"""Autotuner of the staged kernels' launch shape and of the join kernels'
variants.

Sweeps warps per CTA, pipeline stages, tile bytes (vectors per staged tile)
and the dense/row-at-a-time threshold for a workload (DEFAULT_SPACE), or the
join kernels' choices that depend on the query's selectivity -- measure
columns staged or read late, group sums per CTA or per row, how much shared
memory the hash tables take from the staged vectors (JOIN_SPACE) --,
times each candidate with CUDA events after warm-up, keeps the fastest and
caches it in a JSON file keyed by the workload's signature (default
~/.cache/fastlanesgpu_b200/autotune.json, or $FLS_AUTOTUNE_CACHE).  Results
never depend on the choice."""
from __future__ import annotations

import itertools
import json
import os

from . import ops

DEFAULT_SPACE = {
    "warps": [8, 16],
    "stages": [2, 3],
    "tile_bytes": [2048, 6144, 16384],
    "sparse_rows": [2, 4, 8],
}

# The join + group-by kernels' variants whose best choice depends on how many
# rows pass the probes, which the library cannot see before a query runs.
JOIN_SPACE = {
    "late_measure": [0, 1],
    "group_smem": [1, 0],
    "table_kb": [72, 144],
}

_TUNING = {"sparse_rows": 0, "group_smem": 2, "late_measure": 3, "table_kb": 4, "half_vectors": 5}


def cache_path() -> str:
    return os.environ.get("FLS_AUTOTUNE_CACHE",
                          os.path.join(os.path.expanduser("~"), ".cache", "fastlanesgpu_b200", "autotune.json"))


def _load(path):
    try:
        with open(path) as f:
            return json.load(f)
    except Exception:
        return {}


def apply(cfg: dict) -> None:
    """Applies the settings `cfg` names (launch shape and tuning parameters);
    the others keep their current values."""
    if any(k in cfg for k in ("warps", "stages", "tile_bytes")):
        ops.set_launch_config(cfg.get("warps", 0), cfg.get("stages", 0), 0, cfg.get("tile_bytes", 0))
    for k, param in _TUNING.items():
        if k in cfg:
            ops.set_tuning(param, cfg[k])


def time_ms(fn, warmup: int = 3, iters: int = 10) -> float:
    import torch
    for _ in range(warmup):
        fn()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    for _ in range(iters):
        fn()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / iters


def tune(signature: str, fn, space: dict | None = None, iters: int = 10, use_cache: bool = True,
         path: str | None = None, prefer: dict | None = None, margin: float = 0.0, retime: int = 0) -> dict:
    """Best launch configuration for `fn` (a callable enqueueing the workload);
    applies it and returns {config, ms, candidates}.  retime > 0: the
    `retime` fastest candidates (and `prefer`) are timed again, interleaved,
    and ranked by the sum of both timings.  prefer: a configuration (usually
    the library default) kept unless another is faster by more than
    `margin` (a fraction), so timing noise does not move a workload off it."""
    path = path or cache_path()
    cache = _load(path) if use_cache else {}
    if use_cache and signature in cache:
        apply(cache[signature]["config"])
        return cache[signature]
    space = space or DEFAULT_SPACE
    keys = list(space)
    results = []
    for combo in itertools.product(*[space[k] for k in keys]):
        cfg = dict(zip(keys, combo))
        apply(cfg)
        results.append([time_ms(fn, iters=iters), cfg])
    results.sort(key=lambda x: x[0])
    if retime > 0:
        again = results[:retime] + [r for r in results[retime:] if prefer is not None and r[1] == prefer]
        for r in again:
            apply(r[1])
            r[0] += time_ms(fn, iters=iters)
        for r in results:
            if r not in again:
                r[0] *= 2.0
        results.sort(key=lambda x: x[0])
        for r in results:
            r[0] /= 2.0
    chosen = results[0]
    if prefer is not None:
        pref = next((r for r in results if r[1] == prefer), None)
        if pref is not None and chosen[0] > pref[0] * (1.0 - margin):
            chosen = pref
    best = {"config": chosen[1], "ms": chosen[0],
            "candidates": [{"ms": m, **c} for m, c in results]}
    apply(best["config"])
    if use_cache:
        cache[signature] = best
        os.makedirs(os.path.dirname(path), exist_ok=True)
        with open(path, "w") as f:
            json.dump(cache, f, indent=1)
    return best


# The library's defaults for the JOIN_SPACE variants.
JOIN_DEFAULT = {"late_measure": 1, "group_smem": 1, "table_kb": 72}


def reset() -> None:
    """Library defaults for everything the tuner sets."""
    ops.set_launch_config(0, 0, 0, 0)
    ops.set_tuning(0, 0)
    ops.set_tuning(2, 1)
    ops.set_tuning(3, 1)
    ops.set_tuning(4, 0)
    ops.set_tuning(5, 0)
