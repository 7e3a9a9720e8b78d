"""Autotuner: the coordinate descent and the shape cache on the CPU (with a
cost model in place of GPU timing), and one real tuning run on the GPU."""
import json

import pytest

from pic_b200 import autotune


def test_coordinate_descent_finds_the_separable_minimum():
    # cost is separable with its minimum at tile 32, K 40, coarsest 5, omega 1.3, cluster solves
    want = {"tile": 32, "sort_interval": 40, "coarsest_max": 5, "omega": 1.3, "mg_launch": "cluster"}
    calls = []

    def cost(cfg):
        calls.append(cfg)
        return sum(abs(autotune.SPACE[k].index(cfg[k]) - autotune.SPACE[k].index(want[k])) for k in want) + 1.0

    best, c, seen = autotune.coordinate_descent(cost)
    assert best == want and c == 1.0
    # each distinct configuration is measured once
    assert len(calls) == len({tuple(sorted(x.items())) for x in calls}) == len(seen)
    assert len(calls) <= 1 + sum(len(v) for v in autotune.SPACE.values())


def test_ties_keep_the_default():
    best, c, _ = autotune.coordinate_descent(lambda cfg: 5.0)
    assert best == autotune.DEFAULT and c == 5.0


def test_shape_keys_round_particle_counts():
    assert autotune.shape_key(257, 1_000_000) == "257:1048576"
    assert autotune.shape_key(257, 1_100_000) == autotune.shape_key(257, 950_000)
    assert autotune.shape_key(129, 1 << 20) != autotune.shape_key(257, 1 << 20)


def test_cache_round_trip(tmp_path):
    path = str(tmp_path / "tune.json")
    t = autotune.Autotuner(cache_path=path)
    measured = []

    def make(cfg):
        raise AssertionError("a cached shape must not be measured")

    t.cache["129:262144"] = autotune.Choice(8, 40, 9, 1.5)
    t.save()
    t2 = autotune.Autotuner(cache_path=path)
    assert t2.tune("129:262144", make) == autotune.Choice(8, 40, 9, 1.5)
    assert json.load(open(path))["129:262144"]["sort_interval"] == 40
    assert not measured


@pytest.mark.gpu
def test_tuning_a_small_member_on_the_gpu():
    from pic_b200 import workloads

    w = workloads.Workload("tune", 129, 40_000, 40_000, seed=3)
    space = {"tile": (8, 16), "sort_interval": (10, 40), "coarsest_max": (9,), "omega": (1.15,), "mg_launch": ("graph",)}
    t = autotune.Autotuner(space=space, steps=20, warmup=2)
    ch = t.tune_workload(w)
    assert ch.tile in space["tile"] and ch.sort_interval in space["sort_interval"] and ch.coarsest_max == 9
    assert 0.0 < ch.ns_per_particle_step < 1e3
    n = t.measurements
    assert 3 <= n <= 5
    assert t.tune_workload(w) == ch and t.measurements == n  # cached
