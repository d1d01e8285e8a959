"""The batched refinement's autotuner on the host: its coordinate descent
over the scheduling knobs and its JSON cache, driven by a stand-in timer
(the GPU test times real launches)."""

import json

import pytest


class _Tunee:
    """What BatchRefiner.autotune uses: a cache key, a timer and a config."""

    def __init__(self, batch, cost, key="B200|sm148|R10|paths8|n4|px1048576"):
        self.config = batch.default_config()
        self._cost, self._k, self.timed = cost, key, []

    def _key(self):
        return self._k

    def time_config(self, cfg, reps=3):
        d = cfg.as_dict()
        self.timed.append(d)
        return self._cost(d)


def _cost(d):
    # separable, one optimum inside the space: 2048 px, 128 threads, 8 CTAs, fetch 64
    return (abs(d["px_per_block"] - 2048) / 512.0 + abs(d["sgm_threads"] - 128) / 64.0
            + abs(d["sgm_ctas_per_sm"] - 8) / 4.0 + (0.0 if d["sgm_fetch"] == 64 else 0.5)
            + 10.0)


@pytest.fixture
def batch(svb, tmp_path, monkeypatch):
    monkeypatch.setenv("SV_B200_CACHE", str(tmp_path))
    from importlib import import_module
    return import_module(svb.__name__ + ".batch")


def test_descent_finds_the_optimum_and_caches_it(batch, tmp_path):
    t = _Tunee(batch, _cost)
    res = batch.BatchRefiner.autotune(t, reps=1)
    want = {"px_per_block": 2048, "sgm_threads": 128, "sgm_ctas_per_sm": 8, "sgm_fetch": 64}
    assert res["config"] == want and not res["cached"]
    assert t.config.as_dict() == want
    assert res["ms"] == pytest.approx(10.0) and res["default_ms"] >= res["ms"]
    # every candidate timed once
    assert len({json.dumps(d, sort_keys=True) for d in t.timed}) == len(t.timed)
    assert res["candidates"] == len(t.timed)
    cache = json.load(open(tmp_path / "batch_tune.json"))
    assert cache[t._key()]["config"] == want

    # a second tunee with the same key takes the cached choice without timing
    u = _Tunee(batch, _cost)
    again = batch.BatchRefiner.autotune(u, reps=1)
    assert again["cached"] and again["config"] == want and u.timed == []
    assert u.config.as_dict() == want


def test_corrupt_cache_is_ignored_and_rewritten(batch, tmp_path):
    (tmp_path / "batch_tune.json").write_text("{not json")
    t = _Tunee(batch, _cost)
    res = batch.BatchRefiner.autotune(t, reps=1)
    assert not res["cached"]
    assert t._key() in json.load(open(tmp_path / "batch_tune.json"))


def test_no_cache_mode_neither_reads_nor_writes(batch, tmp_path):
    t = _Tunee(batch, _cost)
    batch.BatchRefiner.autotune(t, reps=1, use_cache=True)
    u = _Tunee(batch, lambda d: 5.0)            # every config ties: the default stays
    res = batch.BatchRefiner.autotune(u, reps=1, use_cache=False)
    assert not res["cached"] and u.timed
    assert res["config"] == batch.default_config().as_dict()
    cache = json.load(open(tmp_path / "batch_tune.json"))
    assert cache[t._key()]["ms"] == pytest.approx(10.0)     # untouched
