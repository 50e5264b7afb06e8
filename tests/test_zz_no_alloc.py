"""hive_insert_noalloc: the insert entry point for callers that cannot allocate device memory.

hive_insert may grow its second-pass queue with cudaMalloc; callers that own all device memory
through their own pool, or must not let an allocation stall the device in a latency-bound loop,
use hive_insert_noalloc, whose queue is a fixed array compiled into the library (at most
HIVE_NOALLOC_MAX_OPS ops per call).  These tests call both entry points through the C ABI, two
calls in a row, and require the same outcome: the same per-op result class (new key / updated
key / not placed), the same lookups and the same key->value set, each also equal to the
std::unordered_map replay.  One case fills the table to load factor 0.95, so that many ops take
the second pass through the static queue (checked through the slow-path counter); one runs on a
table that has had deletes, where every new key goes through the queue.

The file is named to be collected last; it must pass alone in a fresh process as well.
"""
import numpy as np
import pytest
import torch

import oracle
from hivehashtable_b200 import HiveHashTable, as_device_u32, library, u32

pytestmark = pytest.mark.gpu

HIVE_NOALLOC_MAX_OPS = 1 << 20
HIVE_ERR_TOO_LARGE = 8


def _classes(st: np.ndarray) -> np.ndarray:
    # 1 inserted / 3 stashed are both "new key placed"; 2 updated; 0 not placed
    return np.where(st == 3, 1, st)


def _call(fn, table, keys, vals):
    dev = table.device
    k, v = as_device_u32(keys, dev), as_device_u32(vals, dev)
    st = torch.full((k.numel(),), 0xEE, dtype=torch.uint8, device=dev)
    rc = fn(table.handle, k.data_ptr(), v.data_ptr(), k.numel(), st.data_ptr(),
            torch.cuda.current_stream(dev).cuda_stream)
    assert rc == 0, rc
    st = st.cpu().numpy()
    assert not (st == 0xEE).any() and not (st == 255).any()
    return st


def _same_as_replay(table, m, keys, vals, st):
    """Per-op classes equal the replay's (ops not placed are left out of the replay)."""
    exp = m.insert(keys, vals, apply_mask=(st != 0).astype(np.uint8))
    ok = st != 0
    np.testing.assert_array_equal(_classes(st)[ok], exp[ok])
    gk, gv = table.dump()
    ok_k, ok_v = m.dump()
    np.testing.assert_array_equal(gk, ok_k)
    np.testing.assert_array_equal(gv, ok_v)
    v = table.verify()
    assert v["tag_mismatch"] == v["misplaced"] == v["duplicate"] == 0, v


def _same_lookups(ta, tb, keys):
    va, fa = ta.find(keys)
    vb, fb = tb.find(keys)
    np.testing.assert_array_equal(fb.cpu().numpy(), fa.cpu().numpy())
    np.testing.assert_array_equal(u32(vb), u32(va))


@pytest.mark.parametrize("policy", ["Default2Hash", "MurmurCityHash"])
def test_noalloc_insert_matches_insert(cuda, policy):
    lib = library()
    cap = 1 << 21
    n1 = int(0.3 * cap)
    keys, fresh, _ = oracle.gen_keys(29, n1, HIVE_NOALLOC_MAX_OPS)
    vals = oracle.values_for(keys)
    # second call: a full-size batch (the maximum) of new keys mixed with updates of first-call
    # keys; the table ends near load factor 0.65, where every insert is placed
    upd = keys[: n1 // 2]
    keys2 = np.concatenate([fresh[: HIVE_NOALLOC_MAX_OPS - upd.size], upd])
    vals2 = oracle.values_for(keys2) ^ np.uint32(0xA5A5A5A5)
    assert keys2.size == HIVE_NOALLOC_MAX_OPS
    ma, mb = oracle.ReplayMap(), oracle.ReplayMap()
    with HiveHashTable(cap, policy) as ta, HiveHashTable(cap, policy) as tb:
        for kk, vv in ((keys, vals), (keys2, vals2)):
            sa = _call(lib.hive_insert, ta, kk, vv)
            sb = _call(lib.hive_insert_noalloc, tb, kk, vv)
            np.testing.assert_array_equal(_classes(sb), _classes(sa))
            _same_lookups(ta, tb, kk)
            _same_as_replay(ta, ma, kk, vv, sa)
            _same_as_replay(tb, mb, kk, vv, sb)
        tb.check()


@pytest.mark.parametrize("policy", ["Default2Hash", "MurmurCityHash"])
def test_noalloc_second_pass_at_high_load(cuda, policy):
    """Two calls that fill the table to load factor 0.95: ops whose two buckets are full go
    through the static queue to the locked path (eviction, stash)."""
    lib = library()
    cap = 1 << 21
    n_total = int(0.95 * cap)
    n2 = HIVE_NOALLOC_MAX_OPS
    keys, _, _ = oracle.gen_keys(31, n_total, 0)
    vals = oracle.values_for(keys)
    calls = [(keys[:n2], vals[:n2]), (keys[n2:], vals[n2:])]  # to load factor 0.5, then 0.95
    assert n_total - n2 <= HIVE_NOALLOC_MAX_OPS
    ma, mb = oracle.ReplayMap(), oracle.ReplayMap()
    with HiveHashTable(cap, policy) as ta, HiveHashTable(cap, policy) as tb:
        for kk, vv in calls:
            sa = _call(lib.hive_insert, ta, kk, vv)
            sb = _call(lib.hive_insert_noalloc, tb, kk, vv)
            np.testing.assert_array_equal(_classes(sb), _classes(sa))
            _same_lookups(ta, tb, kk)
            _same_as_replay(ta, ma, kk, vv, sa)
            _same_as_replay(tb, mb, kk, vv, sb)
        assert (sb != 0).all()
        c = tb.counters()
        assert c["slow_path"] > 1000 and c["evictions"] > 0, "the second call used the no-alloc queue"
        tb.check()


def test_noalloc_after_deletes(cuda):
    """On a table that has had deletes, every new key is claimed under its canonical bucket's lock
    on the second pass, so each call sends all its new keys through the static queue.  Two calls
    of re-inserts, updates, new keys and repeated keys; the repeated keys are checked with the
    per-key serialisation check."""
    lib = library()
    cap = 1 << 20
    keys, fresh, _ = oracle.gen_keys(37, int(0.6 * cap), 400_000)
    vals = oracle.values_for(keys)
    gone = keys[::3]
    rs = np.random.RandomState(7)
    ma, mb = oracle.ReplayMap(), oracle.ReplayMap()
    with HiveHashTable(cap) as ta, HiveHashTable(cap) as tb:
        for t, m in ((ta, ma), (tb, mb)):
            _call(lib.hive_insert, t, keys, vals)
            m.insert(keys, vals)
            assert (t.erase(gone).cpu().numpy() == 1).all()
            m.erase(gone)
        for c in range(2):
            part = slice(c * 150_000, (c + 1) * 150_000)
            base = np.concatenate([gone[part.start // 3: part.stop // 3], keys[1::3][part], fresh[part]])
            kk = np.repeat(base, rs.randint(1, 3, size=base.size)).astype(np.uint32)
            kk = kk[rs.permutation(kk.size)]
            vv = rs.randint(1, 2**32 - 1, size=kk.size).astype(np.uint32)
            n_new = np.unique(kk[~np.isin(kk, mb.dump()[0])]).size
            before = tb.counters()["slow_path"]
            sa = _call(lib.hive_insert, ta, kk, vv)
            sb = _call(lib.hive_insert_noalloc, tb, kk, vv)
            assert tb.counters()["slow_path"] - before >= n_new
            zeros = np.zeros(kk.size, np.uint32)
            for t, m, st in ((ta, ma, sa), (tb, mb, sb)):
                assert (st != 0).all()
                gk, gv = t.dump()
                assert np.unique(gk).size == gk.size
                bad, first = m.check_serial(np.zeros(kk.size, np.uint8), kk, vv, zeros, st, zeros, gk, gv)
                assert bad == 0, (c, bad, first)
                v = t.verify()
                assert v["tag_mismatch"] == v["misplaced"] == v["duplicate"] == 0, v
            # a key inserted twice in one call may keep either value (both orders are valid), so
            # the two tables' values are compared on the keys inserted once
            uk, cnt = np.unique(kk, return_counts=True)
            _same_lookups(ta, tb, uk[cnt == 1])
            np.testing.assert_array_equal(ta.dump()[0], tb.dump()[0])
        tb.check()


def test_noalloc_rejects_oversized_batch(cuda):
    lib = library()
    with HiveHashTable(1 << 12) as t:
        k = torch.zeros(4, dtype=torch.int32, device=t.device)
        st = torch.zeros(4, dtype=torch.uint8, device=t.device)
        rc = lib.hive_insert_noalloc(t.handle, k.data_ptr(), k.data_ptr(), HIVE_NOALLOC_MAX_OPS + 1, st.data_ptr(),
                                     torch.cuda.current_stream(t.device).cuda_stream)
        assert rc == HIVE_ERR_TOO_LARGE
        assert lib.hive_strerror(rc) == b"batch larger than HIVE_NOALLOC_MAX_OPS"
        assert t.size() == 0
