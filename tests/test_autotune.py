"""Autotuner logic on the CPU (the timed trials run on the GPU in test_gpu_autotune)."""
import json

import pytest

from strut_b200 import autotune as T
from strut_b200 import model as M
from strut_b200 import workloads as W


def test_coordinate_search_picks_the_fastest_and_checks_results():
    cost = {"fan_out": {1: 0.0, 0: 5.0}, "element_threads": {640: 3.0, 320: 0.0},
            "commit_team": {0: 1.0, 64: 0.0, 128: 2.0}, "factor_ctas": {0: 0.0}}
    calls = []

    def trial(t):
        calls.append(t)
        return 10.0 + sum(cost[k][t[k]] for k in T.KNOBS), "same"

    cands = {"fan_out": [1, 0], "element_threads": [640, 320], "commit_team": [0, 64, 128], "factor_ctas": [0]}
    best, times = T.coordinate_search(trial, cands)
    assert best == {"fan_out": 1, "element_threads": 320, "commit_team": 64, "factor_ctas": 0}
    assert len(calls) == len(times)  # no tuning timed twice

    def bad(t):
        return 1.0, "a" if t["element_threads"] == 640 else "b"

    with pytest.raises(RuntimeError):
        T.coordinate_search(bad, cands)


def test_workload_class_and_table_round_trip(tmp_path):
    models = [M.Model(c) for c in W.batched_frames(3, steps=5)]
    key = T.workload_class(models, False)
    assert key == "ndf3-fib256-inst4-smem"
    cands = T.candidates(models, False, 5)
    assert cands["fan_out"] == [1, 0] and cands["factor_ctas"] == [0]
    table = tmp_path / "t.json"
    table.write_text(json.dumps({key: {"tuning": {"fan_out": 0, "element_threads": 320, "commit_team": 64,
                                                  "factor_ctas": 0}, "steps": 5, "ms": {}}}))
    assert T.lookup(models, False, table)["element_threads"] == 320
    assert T.lookup(models, True, table) is None
