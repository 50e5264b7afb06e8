"""Same-key concurrency: batches whose keys carry several ops each, checked against a
serialisation that keeps each key's op order.

The ops of one launch are unordered (as in the reference's mixed kernel,
include/hive_kernels.cuh:119-192), so for every key some order of its ops inside a launch -- and
launch order across launches -- must reproduce every status, every returned value and the key's
state in the table afterwards (oracle.ReplayMap.check_serial).  Ops on the same key are placed
both side by side (same warp) and far apart.  Every batch ends with the structural check, which
counts a key with more than one copy anywhere (H0, H1, canonical stash).
"""
import numpy as np
import pytest
import torch

import oracle
from hivehashtable_b200 import (HINT_NO_DELETES, OP_DELETE, OP_INCREMENT, OP_INSERT, OP_LOOKUP, ST_ERROR,
                                HiveHashTable, as_device_u32, u32)
from hivehashtable_b200.table import as_device_u8

pytestmark = pytest.mark.gpu
POLICIES = ["Default2Hash", "MurmurCityHash"]
SOUND = {"tag_mismatch": 0, "misplaced": 0, "duplicate": 0}


def _sound(t):
    v = t.verify()
    assert {k: v[k] for k in SOUND} == SOUND, v


def _dump_unique(t):
    gk, gv = t.dump()
    assert np.unique(gk).size == gk.size, "a key has two copies"
    return gk, gv


def same_key_batch(rs, live, pool, n_hot, n_single, types_allowed, max_ops=6):
    """A batch where n_hot keys (half live, half fresh from `pool`) carry 2..max_ops ops each and
    n_single other keys one op; half of the hot keys have their ops side by side."""
    live = np.asarray(live, dtype=np.uint32)
    n_live = min(n_hot // 2, live.size)
    hot = np.concatenate([rs.choice(live, n_live, replace=False), pool[: n_hot - n_live]])
    pool = pool[n_hot - n_live:]
    ta = np.asarray(types_allowed, dtype=np.uint8)
    chunks = []
    for k in hot:
        ops = [(int(rs.choice(ta)), int(k), int(rs.randint(1, 2**32 - 1))) for _ in range(rs.randint(2, max_ops + 1))]
        if rs.rand() < 0.5:
            chunks.append(ops)
        else:
            chunks.extend([o] for o in ops)
    n_old = min(n_single // 2, live.size)
    others = np.concatenate([rs.choice(live, n_old, replace=False), pool[: n_single - n_old]])
    pool = pool[n_single - n_old:]
    for k in others[~np.isin(others, hot)]:
        chunks.append([(int(rs.choice(ta)), int(k), int(rs.randint(1, 2**32 - 1)))])
    flat = [op for i in rs.permutation(len(chunks)) for op in chunks[i]]
    t = np.array([o[0] for o in flat], dtype=np.uint8)
    k = np.array([o[1] for o in flat], dtype=np.uint32)
    v = np.array([o[2] for o in flat], dtype=np.uint32)
    return t, k, v, pool


def _apply_and_check(t, m, ty, k, v, hints, what):
    st, ov = t.apply(ty, k, v, hints=hints)
    st, ov = st.cpu().numpy(), u32(ov)
    assert not (st == ST_ERROR).any()
    gk, gv = _dump_unique(t)
    bad, first = m.check_serial(ty, k, v, np.zeros(k.size, np.uint32), st, ov, gk, gv)
    assert bad == 0, f"{what}: {bad} keys with no valid order (first op {first}: key {k[first]})"
    ok, ovv = m.dump()
    np.testing.assert_array_equal(gk, ok)
    np.testing.assert_array_equal(gv, ovv)
    _sound(t)


def _run_batches(t, m, rs, pool, n_batches, types_allowed, hints, n_hot=3000, n_single=6000, max_ops=6):
    for b in range(n_batches):
        live, _ = m.dump()
        ty, k, v, pool = same_key_batch(rs, live, pool, n_hot, n_single, types_allowed, max_ops)
        _apply_and_check(t, m, ty, k, v, hints, f"batch {b}")
    return pool


def _prefilled(policy, cap, seed, n_pre, n_pool):
    pre, pool, _ = oracle.gen_keys(seed, n_pre, n_pool)
    m = oracle.ReplayMap()
    t = HiveHashTable(cap, policy)
    t.insert(pre, oracle.values_for(pre))
    m.insert(pre, oracle.values_for(pre))
    return t, m, pre, pool


@pytest.mark.parametrize("policy", POLICIES)
def test_same_key_ops_with_deletes(cuda, policy):
    """Insert / insert / delete / lookup / increment on the same keys in one launch (a table with
    holes: new keys are claimed under the canonical bucket's lock)."""
    rs = np.random.RandomState(101)
    t, m, _, pool = _prefilled(policy, 1 << 16, 71, 24_000, 200_000)
    with t:
        _run_batches(t, m, rs, pool, 8, [OP_INSERT, OP_INSERT, OP_DELETE, OP_LOOKUP, OP_INCREMENT], hints=0)
        assert t.info()["flags"] & 1
        t.check()


@pytest.mark.parametrize("policy", POLICIES)
def test_same_key_ops_without_deletes(cuda, policy):
    """Inserts, lookups and increments on the same keys with the no-deletes hint (a table without
    holes: claims are lock-free and two inserts of a key race for the same slot)."""
    rs = np.random.RandomState(102)
    t, m, _, pool = _prefilled(policy, 1 << 16, 72, 20_000, 200_000)
    with t:
        _run_batches(t, m, rs, pool, 6, [OP_INSERT, OP_INSERT, OP_LOOKUP, OP_INCREMENT], hints=HINT_NO_DELETES)
        assert not (t.info()["flags"] & 1)
        t.check()


def test_hot_keys_in_one_warp(cuda):
    """64 keys with up to 24 ops each, mostly inserts of different values, many in one warp."""
    rs = np.random.RandomState(103)
    t, m, _, pool = _prefilled("Default2Hash", 1 << 13, 73, 4000, 10_000)
    with t:
        _run_batches(t, m, rs, pool, 4, [OP_INSERT, OP_INSERT, OP_INSERT, OP_DELETE, OP_LOOKUP], hints=0,
                     n_hot=64, n_single=200, max_ops=24)


@pytest.mark.parametrize("holes", [False, True])
def test_bulk_insert_with_repeated_keys(cuda, holes):
    """Bulk inserts (hive_insert: first pass, deferred passes) whose keys repeat up to four times
    with different values, into a table filled to load factor ~0.85 (so repeats also meet on the
    locked path); with holes after deletes."""
    rs = np.random.RandomState(104)
    cap = 1 << 17
    t, m, pre, pool = _prefilled("Default2Hash", cap, 74, int(0.5 * cap), cap)
    with t:
        if holes:
            gone = pre[::3]
            assert (t.erase(gone).cpu().numpy() == 1).all()
            m.erase(gone)
        for b in range(3):
            fresh, pool = pool[:12_000], pool[12_000:]
            live, _ = m.dump()
            base = np.concatenate([fresh, rs.choice(live, 4000, replace=False)])
            k = np.repeat(base, rs.randint(1, 5, size=base.size))
            k = k[rs.permutation(k.size)].astype(np.uint32)
            v = rs.randint(1, 2**32 - 1, size=k.size).astype(np.uint32)
            st = t.insert(k, v).cpu().numpy()
            assert not (st == ST_ERROR).any()
            gk, gv = _dump_unique(t)
            zeros = np.zeros(k.size, np.uint32)
            bad, first = m.check_serial(np.zeros(k.size, np.uint8), k, v, zeros, st, zeros, gk, gv)
            assert bad == 0, (b, bad, first)
            _sound(t)


def test_persistent_batches_keep_launch_order(cuda):
    """Several batches in one persistent launch (grid barriers between them): a key's ops in
    batch b come after all its ops in earlier batches."""
    rs = np.random.RandomState(105)
    t, m, pre, pool = _prefilled("Default2Hash", 1 << 16, 75, 16_000, 200_000)
    dev = cuda
    with t:
        live = pre.copy()
        tys, ks, vs, launch = [], [], [], []
        for b in range(6):
            ty, k, v, pool = same_key_batch(rs, live, pool, 1500, 3000,
                                            [OP_INSERT, OP_INSERT, OP_DELETE, OP_LOOKUP, OP_INCREMENT])
            live = np.unique(np.concatenate([live, k[ty == OP_INSERT]]))
            tys.append(ty)
            ks.append(k)
            vs.append(v)
            launch.append(np.full(k.size, b, np.uint32))
        offs = np.cumsum([0] + [a.size for a in ks]).astype(np.int64)
        ty, k, v, launch = (np.concatenate(a) for a in (tys, ks, vs, launch))
        st = torch.zeros(k.size, dtype=torch.uint8, device=dev)
        ov = torch.zeros(k.size, dtype=torch.int32, device=dev)
        t.apply_batches(as_device_u8(ty, dev), as_device_u32(k, dev), as_device_u32(v, dev),
                        torch.from_numpy(offs).to(dev), int(np.diff(offs).max()), st, ov, blocks_per_sm=1)
        st, ovh = st.cpu().numpy(), u32(ov)
        assert not (st == ST_ERROR).any()
        gk, gv = _dump_unique(t)
        bad, first = m.check_serial(ty, k, v, launch, st, ovh, gk, gv)
        assert bad == 0, (bad, first)
        _sound(t)
