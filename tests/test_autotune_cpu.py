"""The autotuner's choice logic with a fake timer (no GPU): the fastest
candidate wins; re-timing ranks the leaders by both timings; a preferred
configuration is kept unless another beats it by more than the margin."""
import pytest

from fastlanesgpu_b200 import autotune

SPACE = {"late_measure": [0, 1], "group_smem": [1, 0]}


@pytest.fixture
def fake(monkeypatch):
    state = {"cfg": None, "calls": [], "times": {}}

    def apply(cfg):
        state["cfg"] = dict(cfg)

    def time_ms(fn, warmup=3, iters=10):
        key = (state["cfg"]["late_measure"], state["cfg"]["group_smem"])
        seq = state["times"][key]
        state["calls"].append(key)
        return seq.pop(0) if len(seq) > 1 else seq[0]

    monkeypatch.setattr(autotune, "apply", apply)
    monkeypatch.setattr(autotune, "time_ms", time_ms)
    return state


def test_fastest_wins(fake):
    fake["times"] = {(0, 1): [1.0], (0, 0): [0.8], (1, 1): [0.9], (1, 0): [1.2]}
    best = autotune.tune("t", lambda: None, space=SPACE, use_cache=False)
    assert best["config"] == {"late_measure": 0, "group_smem": 0} and best["ms"] == 0.8
    assert fake["cfg"] == best["config"] and len(best["candidates"]) == 4


def test_retime_ranks_by_both_timings(fake):
    # (0, 0) looks fastest once, but is slow when timed again
    fake["times"] = {(0, 1): [1.0, 1.0], (0, 0): [0.8, 1.4], (1, 1): [0.9, 0.9], (1, 0): [1.2]}
    best = autotune.tune("t", lambda: None, space=SPACE, use_cache=False, retime=2)
    assert best["config"] == {"late_measure": 1, "group_smem": 1}
    assert best["ms"] == pytest.approx(0.9)
    # only the two leaders were timed twice
    assert fake["calls"].count((0, 0)) == 2 and fake["calls"].count((1, 1)) == 2
    assert fake["calls"].count((0, 1)) == 1 and fake["calls"].count((1, 0)) == 1


def test_prefer_kept_within_margin(fake):
    prefer = {"late_measure": 0, "group_smem": 1}
    fake["times"] = {(0, 1): [1.0], (0, 0): [0.99], (1, 1): [1.1], (1, 0): [1.2]}
    best = autotune.tune("t", lambda: None, space=SPACE, use_cache=False, prefer=prefer, margin=0.02)
    assert best["config"] == prefer and fake["cfg"] == prefer
    fake["times"] = {(0, 1): [1.0], (0, 0): [0.9], (1, 1): [1.1], (1, 0): [1.2]}
    best = autotune.tune("t", lambda: None, space=SPACE, use_cache=False, prefer=prefer, margin=0.02)
    assert best["config"] == {"late_measure": 0, "group_smem": 0}


def test_prefer_retimed_with_leaders(fake):
    prefer = {"late_measure": 1, "group_smem": 0}
    fake["times"] = {(0, 1): [1.0, 1.0], (0, 0): [0.8, 0.8], (1, 1): [0.9, 0.9], (1, 0): [1.2, 0.7]}
    best = autotune.tune("t", lambda: None, space=SPACE, use_cache=False, prefer=prefer, margin=0.2, retime=1)
    assert fake["calls"].count((1, 0)) == 2 and fake["calls"].count((0, 0)) == 2
    # (0, 0): 0.8 + 0.8; prefer: 1.2 + 0.7 = 1.9 / 2 = 0.95; 0.8 > 0.95 * 0.8, so prefer is kept
    assert best["config"] == prefer


def test_reset_restores_every_default():
    """reset() puts back the library defaults of everything apply() can set:
    launch shape, sparse-row threshold, group sums per CTA, late measures,
    table budget, half-vector stages (host-side settings, no GPU needed)."""
    from fastlanesgpu_b200 import ops
    before = (ops.get_launch_config(), [ops.get_tuning(p) for p in (0, 2, 3, 4, 5)])
    try:
        autotune.apply({"warps": 8, "stages": 3, "tile_bytes": 2048, "sparse_rows": 12, "group_smem": 0,
                        "late_measure": 0, "table_kb": 144, "half_vectors": 1})
        assert ops.get_launch_config()[0] == 8 and ops.get_launch_config()[1] == 3
        assert [ops.get_tuning(p) for p in (0, 2, 3, 4, 5)] == [12, 0, 0, 144, 1]
        autotune.apply({"table_kb": 100})  # a partial configuration leaves the rest
        assert [ops.get_tuning(p) for p in (0, 2, 3, 4, 5)] == [12, 0, 0, 100, 1]
        autotune.reset()
        assert [ops.get_tuning(p) for p in (0, 2, 3, 4, 5)] == [4, 1, 1, 72, 0]
        assert (ops.get_launch_config(), [ops.get_tuning(p) for p in (0, 2, 3, 4, 5)]) == before
    finally:
        autotune.reset()
