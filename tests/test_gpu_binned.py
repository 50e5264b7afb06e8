"""The binned bulk insert (HIVE_TUNE_BINNED) against the std::unordered_map replay, bit-exact.

The binned path partitions a batch by the 1024-bucket bin of each key's canonical bucket, runs the
canonical-bucket stage of every op in shared memory, then the second-bucket stage and the locked
passes.  Every case compares each op's status and the full key->value set with the replay, and
with the unbinned insert (binned=0) on the same keys; `hive_verify` must be clean.
"""
import numpy as np
import pytest
import torch

import oracle
from hivehashtable_b200 import ST_ERROR, ST_FAIL, ST_INSERTED, ST_STASHED, ST_UPDATED, HiveHashTable, u32

pytestmark = pytest.mark.gpu
POLICIES = ["Default2Hash", "MurmurCityHash"]
POLID = {"Default2Hash": 0, "MurmurCityHash": 1}
CLEAN = {"tag_mismatch": 0, "misplaced": 0, "duplicate": 0, "stale_tag": 0}


def _np(t):
    return t.cpu().numpy()


def _insert_and_check(t, m, keys, vals):
    st = _np(t.insert(keys, vals))
    assert not (st == ST_ERROR).any()
    exp = m.insert(keys, vals, apply_mask=(st != ST_FAIL).astype(np.uint8))
    ok = st != ST_FAIL
    np.testing.assert_array_equal(np.where(st[ok] == ST_UPDATED, 2, 1), exp[ok])
    return st


def _same_set(t, m):
    gk, gv = t.dump()
    rk, rv = m.dump()
    np.testing.assert_array_equal(gk, rk)
    np.testing.assert_array_equal(gv, rv)
    assert t.size() == len(m)
    assert t.verify() == CLEAN


def _lookups_match(t, m, keys, absent):
    look = np.concatenate([keys, absent])
    v, f = t.find(look)
    ev, ef = m.find(look)
    np.testing.assert_array_equal(_np(f), ef)
    np.testing.assert_array_equal(u32(v), ev)


@pytest.mark.parametrize("policy", POLICIES)
@pytest.mark.parametrize("cap_log", [14, 20, 22])
@pytest.mark.parametrize("lf", [0.5, 0.9, 0.95, 1.0])
def test_binned_one_batch(cuda, policy, cap_log, lf):
    cap = 1 << cap_log
    n = int(lf * cap)
    keys, absent, _ = oracle.gen_keys(7, n, n // 4)
    vals = oracle.values_for(keys)
    m = oracle.ReplayMap()
    with HiveHashTable(cap, policy) as t:
        t.set_tuning(binned=2)
        st = _insert_and_check(t, m, keys, vals)
        if lf <= 0.95:
            assert (st != ST_FAIL).all()
        c = t.counters()
        assert c["failed"] == int((st == ST_FAIL).sum()) and c["error_bits"] == 0
        assert c["stash_push"] == int((st == ST_STASHED).sum())
        _lookups_match(t, m, keys, absent)
        _same_set(t, m)
        t.check()


@pytest.mark.parametrize("policy", POLICIES)
def test_binned_into_a_filled_table(cuda, policy):
    """A second and third batch into a table the first filled to 60 %: half the keys exist (updates
    with new values, from H0, H1 or the stash), half are new; the load reaches 0.95."""
    cap = 1 << 18
    keys, absent, _ = oracle.gen_keys(21, int(0.95 * cap), 1 << 14)
    vals = oracle.values_for(keys)
    n1 = int(0.6 * cap)
    m = oracle.ReplayMap()
    rs = np.random.RandomState(5)
    with HiveHashTable(cap, policy) as t:
        t.set_tuning(binned=2)
        _insert_and_check(t, m, keys[:n1], vals[:n1])
        for lo, hi in ((n1, n1 + (keys.size - n1) // 2), (n1 + (keys.size - n1) // 2, keys.size)):
            old = keys[rs.choice(hi if lo > n1 else n1, size=hi - lo, replace=False)]
            old = old[~np.isin(old, keys[lo:hi])]
            b = np.concatenate([keys[lo:hi], old])
            b = b[rs.permutation(b.size)]
            bv = oracle.values_for(b) ^ np.uint32(0x2545F491)
            st = _insert_and_check(t, m, b, bv)
            assert (st != ST_FAIL).all()
            assert (st[np.isin(b, old)] == ST_UPDATED).all()
        _lookups_match(t, m, keys, absent)
        _same_set(t, m)


def test_binned_duplicates_and_key_zero(cuda):
    """Each key three times in one batch, plus key 0: one insert and two updates per key, the value
    one of its ops' values, key 0 refused."""
    base = np.arange(1, 40001, dtype=np.uint32) * np.uint32(2654435761)
    keys = np.concatenate([np.repeat(base, 3), np.zeros(5, np.uint32)])
    vals = np.arange(keys.size, dtype=np.uint32)
    perm = np.random.RandomState(2).permutation(keys.size)
    keys, vals = keys[perm], vals[perm]
    with HiveHashTable(1 << 17) as t:
        t.set_tuning(binned=2)
        st = _np(t.insert(keys, vals))
        assert (st[keys == 0] == ST_FAIL).all()
        live = keys != 0
        assert (st[live] != ST_FAIL).all()
        order = np.argsort(keys[live], kind="stable")
        s3 = st[live][order].reshape(-1, 3)
        assert (((s3 == ST_INSERTED) | (s3 == ST_STASHED)).sum(1) == 1).all()
        assert ((s3 == ST_UPDATED).sum(1) == 2).all()
        gk, gv = t.dump()
        np.testing.assert_array_equal(gk, np.sort(base))
        kv = dict(zip(keys.tolist(), [set() for _ in keys]))
        for k, v in zip(keys.tolist(), vals.tolist()):
            kv[k].add(v)
        assert all(v in kv[k] for k, v in zip(gk.tolist(), gv.tolist()))
        assert t.verify() == CLEAN


@pytest.mark.parametrize("policy", POLICIES)
def test_binned_ragged_last_bin_and_crowded_bins(cuda, policy):
    """3000 buckets (the last bin holds 952) and a batch with 1200 keys whose two buckets both lie
    in the first 64 (512 slots and 512 stash slots): their canonical buckets overflow, the
    second-bucket stage, the locked path and the stash take the rest and some inserts fail, beside
    6000 keys in the last bin; every result matches the replay."""
    cap = 3000 * 8
    pool, absent, _ = oracle.gen_keys(33, 4_000_000, 4096)
    b0, b1 = oracle.buckets(POLID[policy], pool, 3000)
    crowd = pool[(b0 < 64) & (b1 < 64)][:1200]
    assert crowd.size == 1200
    tail = pool[b0 >= 2048][:6000]
    keys = np.concatenate([crowd, tail])
    keys = keys[np.random.RandomState(3).permutation(keys.size)]
    vals = oracle.values_for(keys)
    m = oracle.ReplayMap()
    with HiveHashTable(cap, policy) as t:
        t.set_tuning(binned=2)
        st = _insert_and_check(t, m, keys, vals)
        assert (st == ST_STASHED).any() and (st == ST_FAIL).any()
        _lookups_match(t, m, keys, absent)
        _same_set(t, m)


@pytest.mark.parametrize("policy", POLICIES)
def test_binned_and_unbinned_agree(cuda, policy):
    """The binned insert (forced) and the unbinned insert at 2^22 slots, LF 0.9: both place every
    key, same key->value set, both clean."""
    cap = 1 << 22
    keys, _, _ = oracle.gen_keys(9, int(0.9 * cap), 0)
    vals = oracle.values_for(keys)
    out = []
    for binned in (2, 0):
        with HiveHashTable(cap, policy) as t:
            t.set_tuning(binned=binned)
            st = _np(t.insert(keys, vals))
            assert (st == ST_INSERTED).sum() + (st == ST_STASHED).sum() == keys.size
            gk, gv = t.dump()
            assert t.verify() == CLEAN
            out.append((gk, gv))
    np.testing.assert_array_equal(out[0][0], out[1][0])
    np.testing.assert_array_equal(out[0][1], out[1][1])
    np.testing.assert_array_equal(out[0][0], np.sort(keys))


def test_binned_host_and_stream_calls(cuda):
    """The binned insert on a side stream with torch tensors, and after a clear."""
    cap = 1 << 20
    keys, _, _ = oracle.gen_keys(12, int(0.9 * cap), 0)
    vals = oracle.values_for(keys)
    kd = torch.from_numpy(keys.view(np.int32)).to(cuda)
    vd = torch.from_numpy(vals.view(np.int32)).to(cuda)
    s = torch.cuda.Stream(cuda)
    with HiveHashTable(cap) as t:
        for _ in range(2):
            t.clear()
            with torch.cuda.stream(s):
                st = t.insert(kd, vd)
            s.synchronize()
            assert bool((st == ST_INSERTED).logical_or(st == ST_STASHED).all())
            v, f = t.find(kd)
            assert bool(f.all()) and torch.equal(v, vd)
            assert t.verify() == CLEAN


@pytest.mark.parametrize("policy", POLICIES)
@pytest.mark.parametrize("lf", [0.9, 1.0])
def test_binned_2p24(cuda, policy, lf):
    """The binned insert (forced) at 2^24 slots, LF 0.9 and 1.0: every status and the full
    key->value set equal the replay's; none unplaced at 0.9."""
    cap = 1 << 24
    keys, absent, _ = oracle.gen_keys(17, int(lf * cap), 1 << 16)
    vals = oracle.values_for(keys)
    m = oracle.ReplayMap()
    with HiveHashTable(cap, policy) as t:
        t.set_tuning(binned=2)
        st = _insert_and_check(t, m, keys, vals)
        if lf <= 0.9:
            assert (st != ST_FAIL).all()
        _lookups_match(t, m, keys, absent)
        _same_set(t, m)
