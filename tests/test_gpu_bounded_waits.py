"""Bounded waits, tested without a fault: an insert that needs a bucket lock held elsewhere gives
up after its bounded spin with HIVE_ST_ERROR and the sticky lock-timeout error, and the table is
usable again once the lock is released and the table cleared."""
import numpy as np
import pytest

import oracle
from hivehashtable_b200 import ST_ERROR, HiveError, HiveHashTable, u32

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("policy,pid", [("Default2Hash", 0), ("MurmurCityHash", 1)])
def test_lock_wait_expires_with_an_error_status(cuda, policy, pid):
    cap = 1 << 12
    nb = cap // 8
    cand, _, _ = oracle.gen_keys(77, 200_000, 0)
    b0, b1 = oracle.buckets(pid, cand, nb)
    i = int(np.flatnonzero(b0 != b1)[0])
    k, kb0, kb1 = cand[i], int(b0[i]), int(b1[i])
    # fill both of k's buckets with keys whose canonical bucket they are
    fill0 = cand[(b0 == kb0) & (cand != k)][:8]
    fill1 = cand[(b0 == kb1) & (cand != k)][:8]
    assert fill0.size == 8 and fill1.size == 8
    fill = np.concatenate([fill0, fill1])
    with HiveHashTable(cap, policy) as t:
        assert bool((t.insert(fill, oracle.values_for(fill)) == 1).all())
        t.debug_hold_lock(kb0)  # as if an evictor held k's canonical bucket
        st = t.insert(np.array([k], dtype=np.uint32), np.array([123], dtype=np.uint32))
        assert int(st.cpu()[0]) == ST_ERROR
        with pytest.raises(HiveError) as e:
            t.check()
        assert e.value.code == 4  # HIVE_ERR_LOCK_TIMEOUT
        c = t.counters()
        assert c["lock_timeout"] >= 1 and c["lock_waits"] >= 1 << 16
        # the failed op changed nothing; the table works again after release + clear
        v, f = t.find(fill)
        assert bool((f == 1).all())
        np.testing.assert_array_equal(u32(v), oracle.values_for(fill))
        t.debug_hold_lock(kb0, held=False)
        t.clear()
        t.check()
        keys = np.concatenate([fill, [k]]).astype(np.uint32)
        assert bool((t.insert(keys, oracle.values_for(keys)) != 0).all())
        v, f = t.find(keys)
        assert bool((f == 1).all())
        np.testing.assert_array_equal(u32(v), oracle.values_for(keys))
        t.check()


def test_hold_lock_rejects_bad_arguments(cuda):
    with HiveHashTable(1 << 10) as t:
        with pytest.raises(HiveError):
            t.debug_hold_lock(1 << 10)  # one past the last bucket
        assert t._lib.hive_debug_hold_lock(t._h, 0, 2, None) == 1  # held must be 0 or 1
