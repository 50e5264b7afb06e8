"""Served loop: every result equals the one-at-a-time replay in arrival order (std::unordered_map),
and equals the result of the same request run alone (batches of one); growth under load."""
import numpy as np
import pytest

import oracle
from hivehashtable_b200 import HiveHashTable
from hivehashtable_b200.serving import ServedWorkload, poisson_arrivals, serve

pytestmark = pytest.mark.gpu


def _expected(w, types, keys, vals):
    m = oracle.ReplayMap()
    m.insert(w.preload_keys, w.preload_vals)
    st, ov = m.apply(types, keys, vals)
    # lookups: found + value; upserts: placed (1)
    exp_s = np.where(types == 1, st, 1).astype(np.uint8)
    exp_v = np.where(types == 1, ov, 0).astype(np.uint32)
    return exp_s, exp_v, m


@pytest.mark.parametrize("mix", ["A", "B", "C", "D"])
@pytest.mark.parametrize("depth,rate", [(1, 0.0), (4, 0.0), (4, 2e6)])
def test_served_results_equal_arrival_order_replay(cuda, mix, depth, rate):
    w = ServedWorkload(17, 1 << 15, 1 << 15, mix)
    with HiveHashTable(1 << 16) as t:
        st = t.insert(w.preload_keys, w.preload_vals)
        assert bool((st != 0).all())
        arr = poisson_arrivals(w.keys.size, rate, seed=3)
        r = serve(t, w.types, w.keys, w.vals, arr, depth=depth, max_batch=2048, max_load=0.9)
        exp_s, exp_v, m = _expected(w, w.types, w.keys, w.vals)
        np.testing.assert_array_equal(r.out_status, exp_s)
        np.testing.assert_array_equal(r.out_vals, exp_v)
        assert (r.done >= r.arrival).all()
        gk, gv = t.dump()
        ok, ov = m.dump()
        np.testing.assert_array_equal(gk, ok)
        np.testing.assert_array_equal(gv, ov)
        v = t.verify()
        assert v["tag_mismatch"] == v["misplaced"] == v["duplicate"] == 0, v
        t.check()


def test_each_result_same_alone_and_in_the_mix(cuda):
    w = ServedWorkload(19, 1 << 13, 1 << 13, "A")
    outs = []
    for depth, batch in ((1, 1), (8, 1024)):
        with HiveHashTable(1 << 15) as t:
            t.insert(w.preload_keys, w.preload_vals)
            r = serve(t, w.types, w.keys, w.vals, np.zeros(w.keys.size), depth=depth, max_batch=batch)
            outs.append((r.out_status.copy(), r.out_vals.copy(), t.dump()))
    (s1, v1, d1), (s2, v2, d2) = outs
    np.testing.assert_array_equal(s1, s2)
    np.testing.assert_array_equal(v1, v2)
    np.testing.assert_array_equal(d1[0], d2[0])
    np.testing.assert_array_equal(d1[1], d2[1])


def test_growth_under_inserts(cuda):
    # mix D adds new records; a small table must grow while serving
    w = ServedWorkload(23, 1 << 12, 1 << 16, "D")
    with HiveHashTable(1 << 13) as t:
        t.insert(w.preload_keys, w.preload_vals)
        r = serve(t, w.types, w.keys, w.vals, np.zeros(w.keys.size), depth=4, max_batch=1024, max_load=0.8)
        exp_s, exp_v, m = _expected(w, w.types, w.keys, w.vals)
        np.testing.assert_array_equal(r.out_status, exp_s)
        np.testing.assert_array_equal(r.out_vals, exp_v)
        assert r.stats["resizes"] >= 1 and t.info()["capacity_slots"] > (1 << 13)
        assert t.size() == len(m)


@pytest.mark.parametrize("grow_start", [0.0, 0.6])
def test_incremental_growth_matches_replay(cuda, grow_start):
    """Growth in bounded split steps between batches (no drain) and growth at once after a drain
    both keep every result equal to the arrival-order replay; the incremental run finishes its
    doublings before the load reaches max_load, so it never drains."""
    w = ServedWorkload(37, 1 << 14, 1 << 18, "D")
    with HiveHashTable(1 << 15, max_capacity=1 << 18) as t:
        t.insert(w.preload_keys, w.preload_vals)
        r = serve(t, w.types, w.keys, w.vals, np.zeros(w.keys.size), depth=4, max_batch=512, max_load=0.85,
                  grow_start=grow_start)
        exp_s, exp_v, m = _expected(w, w.types, w.keys, w.vals)
        np.testing.assert_array_equal(r.out_status, exp_s)
        np.testing.assert_array_equal(r.out_vals, exp_v)
        gk, gv = t.dump()
        ok, ov = m.dump()
        np.testing.assert_array_equal(gk, ok)
        np.testing.assert_array_equal(gv, ov)
        assert r.stats["resizes"] >= 1 and t.info()["capacity_slots"] > (1 << 15)
        if grow_start:
            assert r.stats["grow_steps"] > r.stats["resizes"] and r.stats["drains"] == 0, r.stats
        else:
            assert r.stats["grow_steps"] == 0 and r.stats["drains"] == r.stats["resizes"], r.stats
        v = t.verify()
        assert v["tag_mismatch"] == v["misplaced"] == v["duplicate"] == 0, v
        t.check()


def test_grow_start_bounds(cuda):
    from hivehashtable_b200 import HiveError
    w = ServedWorkload(41, 1 << 10, 1 << 10, "A")
    with HiveHashTable(1 << 12) as t:
        t.insert(w.preload_keys, w.preload_vals)
        for gs, ml in ((0.9, 0.9), (-0.1, 0.9), (0.5, 0.0)):
            with pytest.raises(HiveError) as e:
                serve(t, w.types, w.keys, w.vals, np.zeros(w.keys.size), max_load=ml, grow_start=gs)
            assert e.value.code == 1


@pytest.mark.parametrize("mix", ["A", "D"])
def test_large_batches_match_replay(cuda, mix):
    """Batches of up to 2^16 requests (closed loop, then Poisson arrivals at 20 M/s), with growth:
    every result equals the arrival-order replay."""
    w = ServedWorkload(29, 1 << 16, 1 << 19, mix)
    with HiveHashTable(1 << 17, max_capacity=1 << 20) as t:
        for rate in (0.0, 20e6):
            t.clear()
            t.insert(w.preload_keys, w.preload_vals)
            arr = poisson_arrivals(w.keys.size, rate, seed=5)
            r = serve(t, w.types, w.keys, w.vals, arr, depth=4, max_batch=1 << 16, max_load=0.85)
            exp_s, exp_v, m = _expected(w, w.types, w.keys, w.vals)
            np.testing.assert_array_equal(r.out_status, exp_s)
            np.testing.assert_array_equal(r.out_vals, exp_v)
            gk, gv = t.dump()
            ok, ov = m.dump()
            np.testing.assert_array_equal(gk, ok)
            np.testing.assert_array_equal(gv, ov)
            assert r.stats["form_s"] > 0 and r.stats["answer_s"] > 0
        t.check()
