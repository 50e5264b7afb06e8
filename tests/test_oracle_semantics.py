"""Semantics of the unordered_map replay (reference S1-S6) and the CPU bucketed cuckoo table
checked against it (single- and multi-threaded, forced collisions, stash overflow)."""
import numpy as np
import pytest

import oracle


def test_replay_insert_find_erase_semantics():
    m = oracle.ReplayMap()
    st = m.insert([5, 0, 7, 5], [50, 1, 70, 55])
    assert st.tolist() == [1, 0, 1, 2]  # key 0 rejected (S1), second insert of 5 is an update (S2)
    v, f = m.find([5, 7, 0, 9])
    assert f.tolist() == [1, 1, 0, 0] and v.tolist() == [55, 70, 0, 0]
    assert m.erase([7, 7, 0]).tolist() == [1, 0, 0]
    st, ov = m.apply([0, 1, 3, 3, 2, 1, 4], [9, 9, 9, 11, 9, 9, 5], [90, 0, 0, 0, 0, 0, 0])
    assert st.tolist() == [1, 1, 1, 0, 1, 0, 0]
    assert ov.tolist() == [0, 90, 91, 0, 0, 0, 0]
    k, v = m.dump()
    assert k.tolist() == [5] and v.tolist() == [55]


def test_replay_skips_masked_inserts():
    m = oracle.ReplayMap()
    m.insert([1, 2, 3], [1, 2, 3], apply_mask=np.array([1, 0, 1], np.uint8))
    assert m.dump()[0].tolist() == [1, 3]


def _check_cpu_table(policy, cap, n, threads, max_evictions=8, seed=7):
    keys, absent, st = oracle.gen_keys(seed, n, n)
    vals = oracle.values_for(keys)
    t = oracle.CpuTable(policy, cap, max_evictions)
    status, _ = t.insert(keys, vals, threads)
    assert set(np.unique(status).tolist()) <= {0, 1, 3}
    m = oracle.ReplayMap()
    m.insert(keys, vals, apply_mask=(status != 0).astype(np.uint8))
    look, _ = oracle.lookup_set(keys, absent, n // 2, n // 2, st)
    v, f, _ = t.find(look, threads)
    ev, ef = m.find(look)
    np.testing.assert_array_equal(f, ef)
    np.testing.assert_array_equal(v, ev)
    return int((status == 0).sum()), int((status == 3).sum())


@pytest.mark.parametrize("policy", [0, 1])
@pytest.mark.parametrize("lf", [0.65, 0.9, 0.95])
def test_cpu_table_matches_replay(policy, lf):
    cap = 1 << 16
    failed, _ = _check_cpu_table(policy, cap, int(lf * cap), threads=4)
    assert failed == 0


def test_cpu_table_overflow_is_reported_and_consistent():
    # More keys than slots: stash fills and inserts fail; the successful set must still be exact.
    failed, stashed = _check_cpu_table(0, 1024, 1400, threads=1)
    assert failed > 0 and stashed > 0


def test_cpu_table_no_eviction_uses_stash():
    _, stashed = _check_cpu_table(1, 4096, 3900, threads=2, max_evictions=0)
    assert stashed > 0
