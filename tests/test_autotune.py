"""Autotuner logic (no device): the choice per sweep and the JSON cache."""

import json

from symcode import autotune as A


def test_choose_takes_the_fastest_variant_per_sweep():
    counts = [4, 4, 3, 4, 1]
    timings = {
        0: {"z_inverse": 1.0, "y_inverse": 1.6, "x_sweep": 5.6, "y_forward": 3.2},
        1: {"z_inverse": 0.9, "y_inverse": 1.7, "x_sweep": 3.1, "y_forward": 3.3},
        2: {"z_inverse": 1.2, "y_inverse": 1.5, "x_sweep": 6.0, "y_forward": 3.0},
        3: {"z_inverse": 1.1, "y_inverse": 1.9, "y_forward": 3.0},
    }
    best = A.choose(timings, counts)
    assert best == {"z_inverse": 1, "y_inverse": 2, "x_sweep": 1, "y_forward": 2}
    # a tie keeps the lower variant; a sweep without a choice is left out
    assert "z_forward" not in best


def test_choose_ignores_variants_beyond_a_sweeps_count():
    timings = {0: {"x_sweep": 2.0}, 1: {"x_sweep": 1.0}, 2: {"x_sweep": 0.5}}
    assert A.choose(timings, [1, 1, 2, 1, 1]) == {"x_sweep": 1}


def test_cache_round_trip_is_atomic_and_merges(tmp_path):
    path = str(tmp_path / "tune.json")
    k1 = A.cache_key("NVIDIA B200", 3, 810, "float32")
    k2 = A.cache_key("NVIDIA B200", 3, 128, "float32")
    A.save_cache(path, k1, {"variants": {"x_sweep": 0}, "ms": {}})
    A.save_cache(path, k2, {"variants": {"z_inverse": 1}, "ms": {}})
    data = json.load(open(path))
    assert data[k1]["variants"] == {"x_sweep": 0} and data[k2]["variants"] == {"z_inverse": 1}
    assert [p.name for p in tmp_path.iterdir()] == ["tune.json"]  # no temporary file left
    assert A.load_cache(str(tmp_path / "missing.json")) == {}
