"""Autotuner logic on the host (no GPU): coordinate descent finds the minimum of a separable cost,
ignores noise-level gains, and the cache round-trips."""
import json

import pytest

from sirius_b200 import autotune as A


def test_coordinate_descent_finds_separable_minimum():
    space = {"a": [1, 2, 3, 4], "b": ["x", "y", "z"]}
    cost = {"a": {1: 5.0, 2: 3.0, 3: 1.0, 4: 2.0}, "b": {"x": 4.0, "y": 0.5, "z": 2.0}}
    calls = []

    def measure(cfg):
        calls.append(dict(cfg))
        return cost["a"][cfg["a"]] + cost["b"][cfg["b"]]
    best = A.coordinate_descent(space, {"a": 1, "b": "x"}, measure, rounds=3)
    assert best["a"] == 3 and best["b"] == "y"
    assert best["_ms"] == pytest.approx(1.5)
    assert len(calls) < 4 * 3 * 3  # far fewer than the full grid times rounds


def test_noise_level_gain_is_ignored():
    best = A.coordinate_descent({"k": [0, 1]}, {"k": 0}, lambda c: 1.0 - 0.001 * c["k"], rounds=2)
    assert best["k"] == 0


def test_cache_round_trip(tmp_path, monkeypatch):
    monkeypatch.setenv("SJ_AUTOTUNE_CACHE", str(tmp_path / "c.json"))
    A._store_cache({"k": {"block_size": 128}})
    assert A._load_cache() == {"k": {"block_size": 128}}
    assert json.loads((tmp_path / "c.json").read_text())["k"]["block_size"] == 128


def test_size_class():
    assert A.size_class(1) == 0 and A.size_class(1 << 20) == 20 and A.size_class((1 << 20) + 5) == 20
