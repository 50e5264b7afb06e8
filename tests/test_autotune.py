"""Autotuner: the coordinate-descent search on a fake measurement (CPU), and one small tuning run
on the GPU whose chosen setting still gives the replay's results."""
import numpy as np
import pytest

from hivehashtable_b200 import autotune


def _fake(costs, bad=()):
    calls = []

    def measure(setting):
        calls.append(dict(setting))
        ms = 10.0 - sum(costs.get((k, v), 0.0) for k, v in setting.items())
        key = tuple(sorted(setting.items()))
        return {"ms": ms, "failed": 5 if key in bad else 0, "correct": True}

    return measure, calls


def test_search_takes_the_fastest_valid_setting():
    measure, calls = _fake({("tags", 2): 1.0, ("second_pass_blocks", 4): 0.5, ("max_evictions", 4): -0.5})
    r = autotune.search(measure)
    assert r["best"] == dict(autotune.DEFAULTS, tags=2, second_pass_blocks=4)
    assert r["best_ms"] == pytest.approx(8.5) and r["default_ms"] == pytest.approx(10.0)
    # each setting measured once
    keys = [tuple(sorted(c.items())) for c in calls]
    assert len(keys) == len(set(keys))


def test_search_rejects_settings_that_lose_inserts_or_answers():
    faster = dict(autotune.DEFAULTS, region_insert=2)
    measure, _ = _fake({("region_insert", 2): 3.0}, bad={tuple(sorted(faster.items()))})
    assert autotune.search(measure)["best"]["region_insert"] == 0

    def wrong(setting):
        return {"ms": 1.0 if setting["tags"] == 0 else 5.0, "failed": 0, "correct": setting["tags"] != 0}

    assert autotune.search(wrong)["best"]["tags"] != 0


def test_cache_lookup_takes_the_nearest_capacity(tmp_path):
    import json

    cache = tmp_path / "tune.json"
    entries = {}
    for cap, spb in ((1 << 20, 2), (1 << 24, 8)):
        best = dict(autotune.DEFAULTS, second_pass_blocks=spb)
        entries[autotune.cache_key("GPU-X", cap, 0.9, 0.5, "Default2Hash")] = {
            "best": best, "gpu": "GPU-X", "capacity_slots": cap, "policy": "Default2Hash"}
    cache.write_text(json.dumps(entries))
    assert autotune.lookup_cached(cache, "GPU-X", 1 << 21, "Default2Hash")["second_pass_blocks"] == 2
    assert autotune.lookup_cached(cache, "GPU-X", 1 << 26, "Default2Hash")["second_pass_blocks"] == 8
    assert autotune.lookup_cached(cache, "GPU-Y", 1 << 21, "Default2Hash") is None
    assert autotune.lookup_cached(cache, "GPU-X", 1 << 21, "MurmurCityHash") is None
    assert autotune.lookup_cached(tmp_path / "none.json", "GPU-X", 1 << 21, "Default2Hash") is None


@pytest.mark.gpu
def test_tuned_setting_keeps_results(cuda, tmp_path, monkeypatch):
    """Tune on the GPU into a cache file; a table created with that cache in HIVE_TUNE_CACHE takes
    the tuned knobs (and eviction bound) and still gives the replay's results."""
    import oracle
    from hivehashtable_b200 import HiveHashTable, u32

    cache = tmp_path / "tune.json"
    r = autotune.autotune(1 << 18, 0.9, reps=1, warmup=1, cache=cache)
    best = r["best"]
    assert set(best) == set(autotune.DEFAULTS) and r["best_ms"] <= r["default_ms"] + 1e-9
    keys, absent, st = oracle.gen_keys(3, int(0.9 * (1 << 18)), 1 << 14)
    vals = oracle.values_for(keys)
    m = oracle.ReplayMap()
    monkeypatch.setenv("HIVE_TUNE_CACHE", str(cache))
    with HiveHashTable(1 << 18) as t:
        assert t.tuned == best
        knobs = t.tuning()
        assert all(knobs[k] == v for k, v in best.items() if k != "max_evictions")
        assert t.info()["max_evictions"] == best["max_evictions"]
        s = t.insert(keys, vals).cpu().numpy()
        assert (s != 0).all()
        m.insert(keys, vals)
        look, _ = oracle.lookup_set(keys, absent, 1 << 14, 1 << 14, st)
        v, f = t.find(look)
        ev, ef = m.find(look)
        np.testing.assert_array_equal(f.cpu().numpy(), ef)
        np.testing.assert_array_equal(u32(v), ev)
        gk, gv = t.dump()
        ok, ov = m.dump()
        np.testing.assert_array_equal(gk, ok)
        np.testing.assert_array_equal(gv, ov)
