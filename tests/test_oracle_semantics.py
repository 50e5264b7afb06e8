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


def _serial(m, ops, fin):
    """ops: (type, key, val, launch, status, out); fin: {key: value} after the run."""
    t, k, v, b, st, ov = (np.array(c) for c in zip(*ops))
    fk = np.array(sorted(fin), dtype=np.uint32)
    fv = np.array([fin[x] for x in sorted(fin)], dtype=np.uint32)
    return m.check_serial(t, k, v, b, st, ov, fk, fv)


def test_serial_check_accepts_any_order_inside_a_launch():
    m = oracle.ReplayMap()
    m.insert([7], [70])
    # one launch: insert 5 twice, look up 5, delete 7, look up 7, increment 7
    ops = [(0, 5, 50, 0, 1, 0), (0, 5, 51, 0, 2, 0), (1, 5, 0, 0, 1, 51), (2, 7, 0, 0, 1, 0),
           (1, 7, 0, 0, 1, 70), (3, 7, 0, 0, 0, 0)]
    assert _serial(m, ops, {5: 51}) == (0, -1)
    assert m.dump()[0].tolist() == [5] and m.dump()[1].tolist() == [51]
    # two launches: the second sees the state the first one left
    m2 = oracle.ReplayMap()
    m2.insert([5], [51])
    ops2 = [(1, 5, 0, 0, 1, 51), (0, 7, 9, 0, 1, 0), (3, 7, 0, 0, 1, 10), (1, 7, 0, 1, 1, 10)]
    assert _serial(m2, ops2, {5: 51, 7: 10}) == (0, -1)


def test_serial_check_rejects_inconsistent_outcomes():
    # both inserts of 5 report a new key with no delete between them
    bad, first = _serial(oracle.ReplayMap(), [(0, 5, 50, 0, 1, 0), (0, 5, 51, 0, 1, 0)], {5: 51})
    assert (bad, first) == (1, 0)
    # "inserted 50, updated 51" cannot end at 50
    assert _serial(oracle.ReplayMap(), [(0, 5, 50, 0, 1, 0), (0, 5, 51, 0, 2, 0)], {5: 50})[0] == 1
    # a key deleted in launch 0 cannot be found in launch 1 without an insert
    m = oracle.ReplayMap()
    m.insert([3], [30])
    assert _serial(m, [(2, 3, 0, 0, 1, 0), (1, 3, 0, 1, 1, 30)], {}) == (1, 0)
    assert m.dump()[0].tolist() == [3]  # a failed check leaves the map as it was
    # launch order is kept: a lookup in launch 0 cannot see launch 1's insert
    assert _serial(oracle.ReplayMap(), [(1, 4, 0, 0, 1, 40), (0, 4, 40, 1, 1, 0)], {4: 40})[0] == 1
    # key 0 is never stored
    assert _serial(oracle.ReplayMap(), [(0, 0, 1, 0, 1, 0)], {})[0] == 1
    # an unplaced insert is possible only while the key is absent
    assert _serial(oracle.ReplayMap(), [(0, 6, 1, 0, 0, 0), (0, 6, 2, 0, 1, 0), (1, 6, 0, 0, 1, 2)], {6: 2})[0] == 0
    m = oracle.ReplayMap()
    m.insert([6], [1])
    assert _serial(m, [(0, 6, 2, 0, 0, 0)], {6: 1})[0] == 1


def test_serial_check_matches_replay_on_single_ops():
    keys, absent, _ = oracle.gen_keys(21, 5000, 5000)
    ref, m = oracle.ReplayMap(), oracle.ReplayMap()
    for r in (ref, m):
        r.insert(keys[:2500], oracle.values_for(keys[:2500]))
    rs = np.random.RandomState(3)
    k = rs.permutation(np.concatenate([keys, absent[:2000]]))[:6000].astype(np.uint32)  # one op per key
    t = rs.randint(0, 4, size=k.size).astype(np.uint8)
    v = rs.randint(1, 2**31, size=k.size).astype(np.uint32)
    est, eov = ref.apply(t, k, v)
    fk, fv = ref.dump()
    launch = np.zeros(k.size, np.uint32)
    assert m.check_serial(t, k, v, launch, est, eov, fk, fv) == (0, -1)
    gk, gv = m.dump()
    assert np.array_equal(gk, fk) and np.array_equal(gv, fv)
    eov2 = eov.copy()
    j = int(np.flatnonzero(t == 1)[0])
    eov2[j] ^= 1  # one wrong out value is found
    m3 = oracle.ReplayMap()
    m3.insert(keys[:2500], oracle.values_for(keys[:2500]))
    assert m3.check_serial(t, k, v, launch, est, eov2, fk, fv) == (1, j)


def test_serial_closed_form_agrees_with_search():
    # random one-launch groups of inserts / lookups / deletes: the counting decision used for
    # large groups equals the exhaustive search over orders
    assert oracle.serial_selftest(1, 200_000, 7) == 0


def test_serial_check_large_groups():
    # one key, 40 ops in one launch: 1 new insert, 20 updates, 19 lookups seeing various values
    vals = list(range(100, 121))
    ops = [(0, 9, vals[0], 0, 1, 0)] + [(0, 9, v, 0, 2, 0) for v in vals[1:]]
    ops += [(1, 9, 0, 0, 1, vals[(3 * i) % 21]) for i in range(19)]
    assert _serial(oracle.ReplayMap(), ops, {9: vals[7]}) == (0, -1)
    assert _serial(oracle.ReplayMap(), ops, {9: 999})[0] == 1  # the final value is no write's
    ops2 = ops[:-1] + [(1, 9, 0, 0, 1, 555)]  # a lookup sees a value nobody wrote
    assert _serial(oracle.ReplayMap(), ops2, {9: vals[7]})[0] == 1
