"""The schedule autotuner's search and its on-disk cache (no GPU: the
measurement is a synthetic cost function)."""
import json

from sumpy_b200 import autotune


def test_coordinate_descent_finds_separable_minimum():
    space = {"a": (1, 2, 4, 8), "b": (2, 4, 8), "c": (False, True)}
    cost = {"a": {1: 3.0, 2: 1.0, 4: 2.0, 8: 5.0}, "b": {2: 2.0, 4: 3.0, 8: 0.5},
            "c": {False: 1.0, True: 0.0}}
    calls = []

    def measure(cfg):
        calls.append(cfg)
        return sum(cost[k][v] for k, v in cfg.items())

    best, t, tried = autotune.coordinate_descent({"a": 8, "b": 4, "c": False}, space, measure)
    assert best == {"a": 2, "b": 8, "c": True}
    assert t == 1.5
    # every configuration is measured once
    assert len(calls) == len(tried) == len({repr(sorted(c.items())) for c in calls})


def test_coordinate_descent_keeps_start_when_nothing_is_better():
    space = {"a": (1, 2), "b": (1, 2)}
    best, t, tried = autotune.coordinate_descent({"a": 1, "b": 1}, space,
                                                 lambda cfg: cfg["a"] + cfg["b"])
    assert best == {"a": 1, "b": 1} and t == 2.0
    assert len(tried) == 3


def test_cache_store_and_load(tmp_path):
    p = tmp_path / "cache.json"
    autotune._store(p, {"k": {"best": {"a": 1}, "ms": 2.0}})
    assert autotune._load(p)["k"]["best"] == {"a": 1}
    p.write_text("not json")
    assert autotune._load(p) == {}
    assert json.loads(json.dumps(autotune.SCHEDULE_SPACE, default=list))
