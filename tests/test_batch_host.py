"""Host logic of the batch autotuner's choice (doki_b200/batch.py), on CPU."""
from __future__ import annotations

from doki_b200.batch import pick_trial


def trial(fold, tb, ctas, plan_s, seconds):
    return {"fold": fold, "tile_bits": tb, "ctas_per_sm": ctas, "plan_s": plan_s,
            "seconds": seconds}


def test_planning_noise_does_not_pick_a_slower_kernel():
    # the same fold planned twice (one build per tile width): the 11-bit
    # build happened to plan faster, but its kernel is slower
    trials = [trial(-1, 11, 2, 0.180, 0.0795), trial(-1, 12, 2, 0.195, 0.0669),
              trial(0, 12, 2, 0.354, 0.0655)]
    best, plan = pick_trial(trials)
    assert (best["fold"], best["tile_bits"]) == (-1, 12)
    assert plan == 0.180
    assert all(t["objective_s"] == {-1: 0.180, 0: 0.354}[t["fold"]] + t["seconds"]
               for t in trials)


def test_cheaper_planning_can_outweigh_a_faster_kernel():
    # folding saves device time but costs more planning than it saves
    trials = [trial(-1, 12, 1, 0.28, 0.0669), trial(0, 12, 1, 0.54, 0.0655)]
    best, _ = pick_trial(trials)
    assert best["fold"] == -1
    # and when planning is cheap enough, the faster kernel wins
    trials = [trial(-1, 12, 1, 0.28, 0.0669), trial(0, 12, 1, 0.2805, 0.0655)]
    best, _ = pick_trial(trials)
    assert best["fold"] == 0
