"""CUDA path vs the oracle, bit-exact, through the C ABI (libhive_b200.so).

Small and medium cases are compared op by op with the std::unordered_map replay and by the full
key->value set (hive_dump); the full-size case is checked through size-independent properties.
"""
from pathlib import Path

import numpy as np
import pytest
import torch

import oracle
from hivehashtable_b200 import (HINT_UNIQUE_KEYS, OP_DELETE, OP_INCREMENT, OP_INSERT, OP_LOOKUP, OP_NONE, ST_ERROR,
                                ST_FAIL, HiveError, ST_INSERTED, ST_STASHED, ST_UPDATED, HiveHashTable, u32)
from hivehashtable_b200 import workload

pytestmark = pytest.mark.gpu
GOLD = Path(__file__).resolve().parent / "golden"
POLICIES = ["Default2Hash", "MurmurCityHash"]


def _np(t):
    return t.cpu().numpy()


def _assert_same_set(table: HiveHashTable, m: oracle.ReplayMap):
    gk, gv = table.dump()
    ok, ov = m.dump()
    assert gk.size == ok.size, (gk.size, ok.size)
    np.testing.assert_array_equal(gk, ok)
    np.testing.assert_array_equal(gv, ov)
    assert table.size() == len(m)
    # fingerprints, placement, no duplicates (and no stale fingerprints without holes)
    assert table.verify() == {"tag_mismatch": 0, "misplaced": 0, "duplicate": 0, "stale_tag": 0}


def _insert_and_check(table, m, keys, vals):
    st = _np(table.insert(keys, vals))
    assert not (st == ST_ERROR).any()
    exp = m.insert(keys, vals, apply_mask=(st != ST_FAIL).astype(np.uint8))
    ok = st != ST_FAIL
    # inserted/stashed <-> new key, updated <-> existing key
    np.testing.assert_array_equal(np.where(st[ok] == ST_UPDATED, 2, 1), exp[ok])
    return st


def _find_and_check(table, m, keys):
    v, f = table.find(keys)
    ev, ef = m.find(keys)
    np.testing.assert_array_equal(_np(f), ef)
    np.testing.assert_array_equal(u32(v), ev)
    return _np(f)


@pytest.mark.parametrize("policy", POLICIES)
def test_golden_bulk_small(cuda, policy):
    g = np.load(GOLD / "bulk_small.npz")
    with HiveHashTable(int(g["capacity"]), policy) as t:
        st = _np(t.insert(g["keys"], g["values"]))
        np.testing.assert_array_equal(st != ST_FAIL, g["insert_status"] == 1)
        assert set(np.unique(st).tolist()) <= {ST_INSERTED, ST_STASHED}
        v, f = t.find(g["lookup_keys"])
        np.testing.assert_array_equal(_np(f), g["found"])
        np.testing.assert_array_equal(u32(v), g["found_values"])
        k, vals = t.dump()
        order = np.argsort(g["keys"])
        np.testing.assert_array_equal(k, g["keys"][order])
        np.testing.assert_array_equal(vals, g["values"][order])
        t.check()


def test_plain_bulk_small_config(cuda):
    """2^20 unique keys (seed 42) into a table sized for LF 0.8, Default2Hash; 2^20 lookups with
    half present, shuffled; every result bit-exact against the replay."""
    n = 1 << 20
    cap = -(-n * 10 // 8)
    keys, absent, st = oracle.gen_keys(42, n, n // 2)
    vals = oracle.values_for(keys)
    look, _ = oracle.lookup_set(keys, absent, n // 2, n // 2, st)
    m = oracle.ReplayMap()
    with HiveHashTable(cap, "Default2Hash") as t:
        ins = _insert_and_check(t, m, keys, vals)
        assert (ins != ST_FAIL).all()
        f = _find_and_check(t, m, look)
        assert f.sum() == n // 2
        _assert_same_set(t, m)
        t.check()


@pytest.mark.parametrize("policy", POLICIES)
@pytest.mark.parametrize("cap_log", [16, 20, 22, 24])
@pytest.mark.parametrize("lf", [0.65, 0.80, 0.90, 0.95, 1.0])
def test_bulk_sweep(cuda, policy, cap_log, lf):
    """The bulk sweep (seed 7): capacity x load factor x both policies, every insert's status and
    then n lookups at each present fraction compared op by op with the replay, and the full
    key->value set.  2^22 and 2^24 slots are the sweep's own capacities; 2^26 is covered by
    test_full_size_properties."""
    cap = 1 << cap_log
    n = int(lf * cap)
    keys, absent, st = oracle.gen_keys(7, n, n)
    vals = oracle.values_for(keys)
    m = oracle.ReplayMap()
    with HiveHashTable(cap, policy) as t:
        ins = _insert_and_check(t, m, keys, vals)
        failed = int((ins == ST_FAIL).sum())
        if lf <= 0.95:
            assert failed == 0, failed
        c = t.counters()
        assert c["failed"] == failed and c["error_bits"] == 0
        placed = keys[ins != ST_FAIL]
        for p in (0.0, 0.25, 0.5, 0.75, 1.0):
            npres = int(round(p * n))
            look, st = oracle.lookup_set(placed, absent, min(npres, placed.size), n - npres, st)
            _find_and_check(t, m, look)
        _assert_same_set(t, m)


@pytest.mark.parametrize("policy", POLICIES)
@pytest.mark.parametrize("mode,subbatches", [(1, 0), (1, 1), (1, 3), (1, 8), (2, 0)])
def test_region_ordered_batches(cuda, policy, mode, subbatches):
    """Region-ordered insert and find (counting sort by bucket region, statuses permuted back):
    same per-op results and the same final key set as the replay, at 2^18 buckets (the smallest
    table that takes the region path) and LF 0.95.  Mode 1: sub-batches with an H0-only first
    pass; mode 2: one pass claiming H0 then H1, evicting from H1 before the stash."""
    cap = 1 << 21
    n = int(0.95 * cap)
    keys, absent, st = oracle.gen_keys(11, n, 1 << 16)
    vals = oracle.values_for(keys)
    m = oracle.ReplayMap()
    with HiveHashTable(cap, policy) as t:
        t.set_tuning(region_insert=mode, region_find=1, subbatches=subbatches)
        assert t.tuning()["subbatches"] == subbatches
        ins = _insert_and_check(t, m, keys, vals)
        failed = int((ins == ST_FAIL).sum())
        assert t.counters()["failed"] == failed
        if subbatches in (0, 8):  # the automatic choice (mode 1) at this load is 8 sub-batches
            assert failed == 0, failed
        # re-insert a slice with new values: updates in region order
        upd = keys[: n // 2][::-1].copy()
        _insert_and_check(t, m, upd, oracle.values_for(upd) ^ np.uint32(0x5A5A5A5A))
        look, _ = oracle.lookup_set(keys, absent, n // 2, 1 << 16, st)  # >= num_buckets lookups
        _find_and_check(t, m, look)
        _assert_same_set(t, m)
        assert t.counters()["error_bits"] == 0


@pytest.mark.parametrize("pinned", [True, False])
def test_host_buffer_calls(cuda, pinned):
    """hive_insert_host / hive_find_host: chunked uploads overlapped with the work.  Per-op results
    equal the replay's and the key->value set equals the one hive_insert builds from the same
    batch -- 2^23 slots at LF 0.9, two chunks."""
    cap = 1 << 23
    n = int(0.9 * cap)
    keys, absent, st = oracle.gen_keys(5, n, 1 << 20)
    vals = oracle.values_for(keys)
    look, _ = oracle.lookup_set(keys, absent, 1 << 20, 1 << 20, st)
    host = lambda a: torch.from_numpy(a.view(np.int32)).pin_memory() if pinned else a
    m = oracle.ReplayMap()
    with HiveHashTable(cap) as t, HiveHashTable(cap) as ref:
        status = torch.empty(n, dtype=torch.uint8).pin_memory() if pinned else None
        s = t.insert_host(host(keys), host(vals), status, sync=not pinned)
        if pinned:
            torch.cuda.current_stream().synchronize()
        s = s.numpy()
        exp = m.insert(keys, vals, apply_mask=(s != ST_FAIL).astype(np.uint8))
        assert (s != ST_FAIL).all() and (exp == 1).all()
        v, f = t.find_host(host(look))
        ev, ef = m.find(look)
        np.testing.assert_array_equal(f.numpy(), ef)
        np.testing.assert_array_equal(v.numpy().view(np.uint32), ev)
        _assert_same_set(t, m)
        # the same batch through the device-buffer call: the same key->value set
        ref.insert(keys, vals)
        gk, gv = t.dump()
        rk, rv = ref.dump()
        np.testing.assert_array_equal(gk, rk)
        np.testing.assert_array_equal(gv, rv)
        # updates and an empty call through the host path
        upd = np.ascontiguousarray(keys[::3])
        s2 = t.insert_host(upd, upd).numpy()
        np.testing.assert_array_equal(s2, np.full(upd.size, ST_UPDATED, np.uint8))
        assert t.insert_host(np.empty(0, np.uint32), np.empty(0, np.uint32)).numel() == 0
        v2, f2 = t.find_host(upd)
        assert f2.numpy().all()
        np.testing.assert_array_equal(v2.numpy().view(np.uint32), upd)
        t.check()


@pytest.mark.parametrize("policy", POLICIES)
@pytest.mark.parametrize("retag", [0, 2])
def test_tag_upkeep_modes(cuda, policy, retag):
    """Per-slot fingerprints kept per op (0) or rebuilt after each bulk insert (2): the same
    results as the replay through bulk insert, updates, erases and re-inserts, and the
    fingerprint invariant holds after every step."""
    cap = 1 << 20
    n = int(0.92 * cap)
    keys, absent, st = oracle.gen_keys(23, n, 1 << 15)
    vals = oracle.values_for(keys)
    m = oracle.ReplayMap()
    with HiveHashTable(cap, policy) as t:
        t.set_tuning(bulk_retag=retag)
        ins = _insert_and_check(t, m, keys, vals)
        assert (ins != ST_FAIL).all()
        _assert_same_set(t, m)
        upd = keys[::5].copy()
        _insert_and_check(t, m, upd, oracle.values_for(upd) + np.uint32(9))
        gone = keys[1::3].copy()
        st_e = _np(t.erase(gone))
        np.testing.assert_array_equal(st_e, m.erase(gone))
        _assert_same_set(t, m)
        _insert_and_check(t, m, gone[::2].copy(), oracle.values_for(gone[::2]))
        look, _ = oracle.lookup_set(keys, absent, 1 << 15, 1 << 15, st)
        _find_and_check(t, m, look)
        _assert_same_set(t, m)
        t.check()


@pytest.mark.parametrize("policy", POLICIES)
def test_tags_switched_off_and_on(cuda, policy):
    """Fingerprints off (HIVE_TUNE_TAGS 0, as for tables too large for their tag words to stay in
    L2), then on again: lookups read whole buckets while off, the stale tag words are rebuilt on
    the first launch after they are switched on, and results equal the replay throughout."""
    cap = 1 << 18
    keys, absent, st = oracle.gen_keys(31, int(0.9 * cap), 1 << 14)
    vals = oracle.values_for(keys)
    m = oracle.ReplayMap()
    third = keys.size // 3
    with HiveHashTable(cap, policy) as t:
        t.set_tuning(tags=0)
        _insert_and_check(t, m, keys[:third], vals[:third])
        look, st = oracle.lookup_set(keys[:third], absent, 1 << 13, 1 << 13, st)
        _find_and_check(t, m, look)
        gone = keys[: third // 4].copy()
        np.testing.assert_array_equal(_np(t.erase(gone)), m.erase(gone))
        _assert_same_set(t, m)
        t.set_tuning(tags=2)
        small = keys[third: third + 2000].copy()  # a small batch: per-op fingerprint upkeep
        _insert_and_check(t, m, small, oracle.values_for(small))
        _find_and_check(t, m, np.concatenate([look, small]))
        _assert_same_set(t, m)
        t.set_tuning(tags=0)
        _insert_and_check(t, m, keys[third + 2000:], vals[third + 2000:])
        t.set_tuning(tags=2)
        look, st = oracle.lookup_set(keys, absent, 1 << 14, 1 << 14, st)
        _find_and_check(t, m, look)
        types = np.where(np.arange(look.size) % 3 == 0, OP_INSERT, OP_LOOKUP).astype(np.uint8)
        uk, ui = np.unique(look, return_index=True)
        st_a, ov_a = t.apply(types[ui], uk, oracle.values_for(uk) ^ np.uint32(7), hints=HINT_UNIQUE_KEYS)
        est, eov = m.apply(types[ui], uk, oracle.values_for(uk) ^ np.uint32(7))
        np.testing.assert_array_equal(np.where(_np(st_a) == ST_STASHED, 1, _np(st_a)), est)
        np.testing.assert_array_equal(u32(ov_a), eov)
        _assert_same_set(t, m)
        t.check()


def test_tuning_bounds(cuda):
    with HiveHashTable(1 << 12) as t:
        assert t.tuning() == {"region_insert": 0, "region_find": 0, "subbatches": 0, "second_pass_blocks": 8,
                              "bulk_retag": 1, "tags": 1, "l2_window": 0, "stash_depth": 8, "binned": 1}
        for bad in ({"region_insert": 3}, {"subbatches": 9}, {"second_pass_blocks": 0}, {"bulk_retag": 3},
                    {"tags": 3}, {"l2_window": 3}, {"stash_depth": 0}, {"stash_depth": 9}, {"binned": 3}):
            with pytest.raises(HiveError):
                t.set_tuning(**bad)
        t.set_tuning(second_pass_blocks=2)
        keys, _, _ = oracle.gen_keys(3, 3000, 0)
        m = oracle.ReplayMap()
        _insert_and_check(t, m, keys, oracle.values_for(keys))
        _assert_same_set(t, m)


@pytest.mark.parametrize("policy", POLICIES)
def test_read_only_lookup_paths(cuda, policy):
    """The read-only lookup path answers as the replay through hive_find, the host-buffer path and
    lookup-only reference records."""
    n = 300_000
    keys, absent, st = oracle.gen_keys(43, n, n)
    vals = oracle.values_for(keys)
    m = oracle.ReplayMap()
    with HiveHashTable(int(n / 0.9), policy) as t:
        _insert_and_check(t, m, keys, vals)
        look, _ = oracle.lookup_set(keys, absent, n // 2, n // 2, st)
        _find_and_check(t, m, look)
        hv, hf = t.find_host(look)
        ev, ef = m.find(look)
        np.testing.assert_array_equal(np.asarray(hf).astype(np.uint8), ef)
        np.testing.assert_array_equal(np.asarray(hv).view(np.uint32), ev)
        ops = torch.from_numpy(np.stack([np.full(look.size, OP_LOOKUP, np.int64), look.astype(np.int64)], 1))
        res = _np(t.apply_reference_ops(ops, hints=2))
        np.testing.assert_array_equal(res, ef.astype(np.int64))


def test_reference_record_path(cuda):
    """16-byte Operation records, value = key + 1, uint64 0/1 results (the reference's kernel
    contract, include/hive_kernels.cuh:119-266)."""
    n = 50_000
    keys, absent, _ = oracle.gen_keys(11, n, n // 4)
    ops = np.zeros((n, 2), dtype=np.int64)
    ops[:, 0] = 0
    ops[:, 1] = keys.astype(np.int64)
    with HiveHashTable(1 << 17) as t:
        r = _np(t.apply_reference_ops(torch.from_numpy(ops), hints=1))
        assert (r == 1).all()
        look = np.concatenate([keys[: n // 2], absent])
        lops = np.stack([np.full(look.size, 1, np.int64), look.astype(np.int64)], axis=1)
        r = _np(t.apply_reference_ops(torch.from_numpy(lops)))
        np.testing.assert_array_equal(r, np.r_[np.ones(n // 2), np.zeros(absent.size)].astype(np.int64))
        v, f = t.find(keys[:100])
        np.testing.assert_array_equal(u32(v), keys[:100] + np.uint32(1))
        # delete / ATOMIC_INC (3) / NONE (4) records
        dops = np.stack([np.array([2, 2, 3, 3, 4], np.int64),
                         np.array([keys[0], absent[0], keys[1], absent[1], keys[2]], np.int64)], axis=1)
        r = _np(t.apply_reference_ops(torch.from_numpy(dops)))
        assert r.tolist() == [1, 0, 1, 0, 0]
        v, f = t.find(keys[:3])
        assert _np(f).tolist() == [0, 1, 1] and u32(v)[1] == keys[1] + 2


@pytest.mark.parametrize("policy", POLICIES)
def test_erase_then_reinsert(cuda, policy):
    n = 200_000
    cap = int(n / 0.9)
    keys, absent, st = oracle.gen_keys(13, n, n // 2)
    vals = oracle.values_for(keys)
    m = oracle.ReplayMap()
    with HiveHashTable(cap, policy) as t:
        _insert_and_check(t, m, keys, vals)
        gone = keys[::2]
        est = _np(t.erase(np.concatenate([gone, absent[:1000], [0]])))
        exp = m.erase(np.concatenate([gone, absent[:1000], [0]]))
        np.testing.assert_array_equal(est, exp)
        _assert_same_set(t, m)
        # holes mode: upserts of survivors, re-inserts of erased keys, new keys
        mix = np.concatenate([keys[1:20000:2], gone[:20000], absent[:20000]])
        _insert_and_check(t, m, mix, oracle.values_for(mix) ^ np.uint32(0x5A5A5A5A))
        look, _ = oracle.lookup_set(keys, absent, 50_000, 50_000, st)
        _find_and_check(t, m, look)
        _assert_same_set(t, m)
        assert t.info()["flags"] & 1


@pytest.mark.parametrize("policy", POLICIES)
@pytest.mark.parametrize("hints", [0, HINT_UNIQUE_KEYS])
def test_mixed_batches(cuda, policy, hints):
    """Batches of 50 % insert (new keys), 10 % upsert of live keys, 30 % lookup (80 % present),
    10 % delete (live keys); at most one op per key per batch, so every op's result is fixed and
    the unique-keys hint holds."""
    rng_state = 11
    pre, pool, rng_state = oracle.gen_keys(rng_state, 60_000, 400_000)
    m = oracle.ReplayMap()
    live = list(pre)
    with HiveHashTable(1 << 17, policy) as t:
        _insert_and_check(t, m, pre, oracle.values_for(pre))
        pool_i = 0
        rs = np.random.RandomState(5)
        for b in range(12):
            size = int(2 ** rs.uniform(10, 15))
            ni, nu, nl = size // 2, size // 10, size * 3 // 10
            nd = size - ni - nu - nl
            new = pool[pool_i: pool_i + ni]
            pool_i += ni
            livea = np.array(live, dtype=np.uint32)
            sel = rs.choice(livea.size, size=nu + nl + nd, replace=False)
            upd = livea[sel[:nu]]
            lk_present = livea[sel[nu: nu + int(nl * 0.8)]]
            lk_absent = pool[pool_i: pool_i + (nl - lk_present.size)]
            pool_i += lk_absent.size
            dels = livea[sel[nu + nl: nu + nl + nd]]
            keys = np.concatenate([new, upd, lk_present, lk_absent, dels]).astype(np.uint32)
            types = np.concatenate([np.full(ni + nu, OP_INSERT), np.full(nl, OP_LOOKUP),
                                    np.full(nd, OP_DELETE)]).astype(np.uint8)
            vals = oracle.values_for(keys) ^ np.uint32(b)
            perm = rs.permutation(keys.size)
            keys, types, vals = keys[perm], types[perm], vals[perm]
            st, ov = t.apply(types, keys, vals, hints=hints)
            st, ov = _np(st), u32(ov)
            assert not (st == ST_ERROR).any()
            ok_ins = (types != OP_INSERT) | (st != ST_FAIL)
            est, eov = m.apply(types, keys, vals, apply_mask=ok_ins.astype(np.uint8))
            gst = np.where((types == OP_INSERT) & (st == ST_STASHED), 1, st)
            np.testing.assert_array_equal(gst, est)
            np.testing.assert_array_equal(ov, eov)
            live = sorted((set(live) | set(new.tolist())) - set(dels.tolist()))
        _assert_same_set(t, m)
        t.check()


def test_duplicate_keys_in_one_batch(cuda):
    keys = np.repeat(np.arange(1, 5001, dtype=np.uint32) * np.uint32(2654435761), 3)
    vals = np.arange(keys.size, dtype=np.uint32)
    perm = np.random.RandomState(1).permutation(keys.size)
    keys, vals = keys[perm], vals[perm]
    with HiveHashTable(1 << 14) as t:
        st = _np(t.insert(keys, vals))
        assert (st != ST_FAIL).all()
        for k in np.unique(keys)[:200]:
            s = st[keys == k]
            assert ((s == ST_INSERTED) | (s == ST_STASHED)).sum() == 1 and (s == ST_UPDATED).sum() == 2
        gk, gv = t.dump()
        assert gk.size == np.unique(keys).size and np.unique(gk).size == gk.size
        for k, v in zip(gk[:500], gv[:500]):
            assert v in vals[keys == k]


def test_key_zero_and_empty_inputs(cuda):
    with HiveHashTable(1024) as t:
        e = np.zeros(0, np.uint32)
        assert t.insert(e, e).numel() == 0
        assert t.find(e)[0].numel() == 0
        assert _np(t.insert([0, 5], [9, 9])).tolist() == [ST_FAIL, ST_INSERTED]
        v, f = t.find([0, 5])
        assert _np(f).tolist() == [0, 1] and u32(v).tolist() == [0, 9]
        assert _np(t.erase([0])).tolist() == [0]
        st, ov = t.apply([OP_NONE, OP_LOOKUP, OP_INCREMENT, OP_INCREMENT], [5, 0, 5, 6], [0, 0, 0, 0])
        assert _np(st).tolist() == [0, 0, 1, 0] and u32(ov).tolist() == [0, 0, 10, 0]
        assert t.size() == 1
        t.clear()
        assert t.size() == 0 and _np(t.find([5])[1]).tolist() == [0]


@pytest.mark.parametrize("max_ev", [0, 8])
def test_forced_collisions_stash_and_overflow(cuda, max_ev):
    """64 slots (8 buckets) and 300 keys: the stash fills and inserts fail; the successful set and
    every lookup still match the replay exactly."""
    keys, absent, _ = oracle.gen_keys(3, 300, 100)
    vals = oracle.values_for(keys)
    m = oracle.ReplayMap()
    with HiveHashTable(64, max_evictions=max_ev) as t:
        st = _insert_and_check(t, m, keys, vals)
        assert (st == ST_FAIL).sum() > 0 and (st == ST_STASHED).sum() > 0
        c = t.counters()
        assert c["stash_push"] == (st == ST_STASHED).sum() and c["failed"] == (st == ST_FAIL).sum()
        _find_and_check(t, m, np.concatenate([keys, absent]))
        _assert_same_set(t, m)
        # erase stashed keys and re-insert: stash slots are reused
        _np(t.erase(keys[:150]))
        m.erase(keys[:150])
        _assert_same_set(t, m)
        st2 = _insert_and_check(t, m, keys[:150], vals[:150] + np.uint32(1))
        assert (st2 != ST_FAIL).sum() > 0
        _find_and_check(t, m, np.concatenate([keys, absent]))
        _assert_same_set(t, m)


@pytest.mark.parametrize("depth", [1, 2, 4])
def test_stash_depth_limits_the_stash(cuda, depth):
    """HIVE_TUNE_STASH_DEPTH: forced collisions place at most `depth` keys in each canonical stash;
    the placed set and every lookup still match the replay."""
    keys, absent, _ = oracle.gen_keys(3, 300, 100)
    vals = oracle.values_for(keys)
    m = oracle.ReplayMap()
    with HiveHashTable(64) as t:
        t.set_tuning(stash_depth=depth)
        st = _insert_and_check(t, m, keys, vals)
        assert 0 < (st == ST_STASHED).sum() <= depth * 8  # 8 buckets, `depth` stash slots each
        _find_and_check(t, m, np.concatenate([keys, absent]))
        _assert_same_set(t, m)
        t.set_tuning(stash_depth=8)  # deeper stashes take the keys that found no room
        more = keys[st == ST_FAIL]
        st2 = _insert_and_check(t, m, more, oracle.values_for(more))
        assert (st2 == ST_STASHED).sum() > 0
        _assert_same_set(t, m)


@pytest.mark.parametrize("policy", POLICIES)
def test_resize_grow_and_shrink(cuda, policy):
    keys, absent, st = oracle.gen_keys(13, 120_000, 20_000)
    vals = oracle.values_for(keys)
    m = oracle.ReplayMap()
    with HiveHashTable(1 << 14, policy) as t:
        done = 0
        for chunk in range(12):
            part = keys[done: done + 10_000]
            done += part.size
            info = t.info()
            if (len(m) + part.size) / info["capacity_slots"] > 0.85:
                t.resize(info["capacity_slots"] * 2)
                _assert_same_set(t, m)
            _insert_and_check(t, m, part, vals[done - part.size: done])
            _assert_same_set(t, m)
        inf = t.info()
        assert inf["capacity_slots"] > (1 << 14) and inf["num_buckets"] == inf["capacity_slots"] // 8
        # odd intermediate size (split pointer mid-level), then shrink
        t.resize(inf["capacity_slots"] + 8 * 1000)
        _assert_same_set(t, m)
        look, _ = oracle.lookup_set(keys, absent, 20_000, 20_000, st)
        _find_and_check(t, m, look)
        gone = keys[: 100_000]
        np.testing.assert_array_equal(_np(t.erase(gone)), m.erase(gone))
        t.resize(1 << 15)
        assert t.info()["capacity_slots"] == 1 << 15
        _assert_same_set(t, m)
        _find_and_check(t, m, look)
        # 20,000 live keys do not fit 2^14 slots at LF <= 0.9: refused, table unchanged
        with pytest.raises(HiveError) as e:
            t.resize(1 << 10)
        assert e.value.code == 6 and t.info()["capacity_slots"] == 1 << 15
        # 24,000 slots would hold them at LF 0.83, but mid-level its 2^14 unsplit slots would take
        # them at 1.22: refused as well
        with pytest.raises(HiveError) as e:
            t.resize(24_000)
        assert e.value.code == 6 and t.info()["capacity_slots"] == 1 << 15
        _assert_same_set(t, m)
        more = keys[100_000: 110_000]
        np.testing.assert_array_equal(_np(t.erase(more)), m.erase(more))
        t.resize(1 << 10)  # clamped to the creation size
        assert t.info()["capacity_slots"] == 1 << 14
        _assert_same_set(t, m)
        _find_and_check(t, m, look)
        t.check()


@pytest.mark.parametrize("policy", POLICIES)
def test_dump_load_and_checkpoint(cuda, policy, tmp_path):
    """dump -> load into a smaller table (which grows) and save -> restore give the replay's
    key->value set; a restored table keeps the saved geometry, split pointer included."""
    keys, absent, st = oracle.gen_keys(29, 150_000, 20_000)
    vals = oracle.values_for(keys)
    m = oracle.ReplayMap()
    with HiveHashTable(1 << 15, policy, max_capacity=1 << 19) as a:
        a.resize(1 << 18)
        _insert_and_check(a, m, keys, vals)
        gone = keys[::3]
        np.testing.assert_array_equal(_np(a.erase(gone)), m.erase(gone))
        a.resize((1 << 18) + 8 * 777)  # split pointer mid-level
        _assert_same_set(a, m)
        kv = a.dump_packed()
        assert kv.numel() == len(m)
        look, _ = oracle.lookup_set(keys, absent, 30_000, 30_000, st)
        with HiveHashTable(1 << 14, policy) as b:
            b.insert(absent[:5000], absent[:5000])  # replaced by the load
            b.load(kv)
            assert b.info()["capacity_slots"] >= len(m) / 0.9
            _assert_same_set(b, m)
            _find_and_check(b, m, look)
            # the unpacked form, into the table's existing size
            k, v = a.dump()
            b.load(k, v)
            _assert_same_set(b, m)
            b.check()
        path = tmp_path / "table.npz"
        a.save(path)
        with HiveHashTable.restore(path) as c:
            ia, ic = a.info(), c.info()
            for f in ("num_buckets", "base_buckets", "level", "split", "max_buckets", "max_evictions", "policy"):
                assert ia[f] == ic[f], f
            _assert_same_set(c, m)
            _find_and_check(c, m, look)
            # the restored table takes further batches like the original
            more = absent[:10_000]
            _insert_and_check(c, m, more, oracle.values_for(more))
            _assert_same_set(c, m)
            c.check()


def test_load_edge_cases(cuda):
    """Empty input, key 0 (reported as unplaced), and a load across two internal chunks."""
    with HiveHashTable(1 << 16) as t:
        t.insert(np.arange(1, 1001, dtype=np.uint32), np.arange(1, 1001, dtype=np.uint32))
        t.load(torch.empty(0, dtype=torch.int64, device="cuda"))
        assert t.size() == 0 and t.info()["capacity_slots"] == 1 << 16
        # key 0 is not storable: reported, the rest placed
        k = np.array([0, 5, 6, 7], dtype=np.uint32)
        with pytest.raises(HiveError) as e:
            t.load(k, k + np.uint32(1))
        assert e.value.code == 6 and "1 of 4" in str(e.value)
        gk, gv = t.dump()
        np.testing.assert_array_equal(gk, [5, 6, 7])
        np.testing.assert_array_equal(gv, [6, 7, 8])
    # 2^22 + 4321 entries: two chunks of the load's staging, and growth from 2^16 slots
    n = (1 << 22) + 4321
    keys, _, _ = oracle.gen_keys(31, n, 0)
    vals = oracle.values_for(keys)
    with HiveHashTable(1 << 16, max_capacity=1 << 24) as t:
        t.load(keys, vals)
        assert t.size() == n and t.info()["capacity_slots"] >= n / 0.9
        gk, gv = t.dump()
        order = np.argsort(keys)
        np.testing.assert_array_equal(gk, keys[order])
        np.testing.assert_array_equal(gv, vals[order])
        assert t.verify() == {"tag_mismatch": 0, "misplaced": 0, "duplicate": 0, "stale_tag": 0}


def test_bucket_choice_matches_oracle(cuda):
    keys = np.random.RandomState(0).randint(0, 2**32, size=100_000, dtype=np.uint64).astype(np.uint32)
    for policy, pid in (("Default2Hash", 0), ("MurmurCityHash", 1)):
        for cap in (8, 1_310_720, 1 << 26):
            with HiveHashTable(cap, policy) as t:
                b0, b1 = t.bucket_of(keys)
                e0, e1 = oracle.buckets(pid, keys, t.info()["num_buckets"])
                np.testing.assert_array_equal(u32(b0), e0)
                np.testing.assert_array_equal(u32(b1), e1)


@pytest.mark.parametrize("policy", POLICIES)
def test_full_size_properties(cuda, policy):
    """Headline size: 2^26 slots at LF 0.9 (60,397,977 keys, seed 7), both policies.
    Size-independent checks: every insert succeeds, size equals n, every inserted key is found
    with its own value, absent keys are missed, and the dump's key and value checksums equal the
    inputs'."""
    cap = 1 << 26
    n = int(0.9 * cap)
    keys, absent, _ = workload.gen_keys(7, n, 1 << 20)
    vals = workload.values_for(keys)
    with HiveHashTable(cap, policy) as t:
        st = _np(t.insert(keys, vals))
        assert (st != ST_FAIL).all() and not (st == ST_UPDATED).any()
        assert t.size() == n
        v, f = t.find(keys)
        assert bool((f == 1).all())
        np.testing.assert_array_equal(u32(v), vals)
        _, fa = t.find(absent)
        assert int(fa.sum()) == 0
        gk, gv = t.dump()
        assert gk.size == n and np.unique(gk).size == n
        assert int(gk.astype(np.uint64).sum()) == int(keys.astype(np.uint64).sum())
        assert int(gv.astype(np.uint64).sum()) == int(vals.astype(np.uint64).sum())
        assert t.verify() == {"tag_mismatch": 0, "misplaced": 0, "duplicate": 0, "stale_tag": 0}
        t.check()
