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
    measure, calls = _fake({("tags", 2): 1.0, ("second_pass_blocks", 8): 0.5, ("max_evictions", 4): -0.5})
    r = autotune.search(measure)
    assert r["best"] == dict(autotune.DEFAULTS, tags=2, second_pass_blocks=8)
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


@pytest.mark.gpu
def test_tuned_setting_keeps_results(cuda):
    import oracle
    from hivehashtable_b200 import HiveHashTable, u32

    r = autotune.autotune(1 << 18, 0.9, reps=1, warmup=1)
    best = r["best"]
    assert set(best) == set(autotune.DEFAULTS) and r["best_ms"] <= r["default_ms"] + 1e-9
    keys, absent, st = oracle.gen_keys(3, int(0.9 * (1 << 18)), 1 << 14)
    vals = oracle.values_for(keys)
    m = oracle.ReplayMap()
    with HiveHashTable(1 << 18, max_evictions=best["max_evictions"]) as t:
        autotune.apply(t, best)
        s = t.insert(keys, vals).cpu().numpy()
        assert (s != 0).all()
        m.insert(keys, vals)
        look, _ = oracle.lookup_set(keys, absent, 1 << 14, 1 << 14, st)
        v, f = t.find(look)
        ev, ef = m.find(look)
        np.testing.assert_array_equal(f.cpu().numpy(), ef)
        np.testing.assert_array_equal(u32(v), ev)
