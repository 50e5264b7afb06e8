"""Resize while ops run (hive_apply_ops_split): each call splits the next window of buckets of
the current level in the same launch as a batch of mixed ops, most of them on keys whose buckets
are in that window -- lookups that must find keys mid-move, and upserts, new inserts, deletes and
increments that must land in the right home.  Every op's result equals the std::unordered_map
replay (keys are unique within a batch, so each result is fixed), and after every call the full
key->value set equals the replay's and the table is structurally sound, through a whole doubling
and into the next level."""
import numpy as np
import pytest

import oracle
from hivehashtable_b200 import OP_DELETE, OP_INCREMENT, OP_INSERT, OP_LOOKUP, ST_ERROR, HiveHashTable, u32

pytestmark = pytest.mark.gpu
POLID = {"Default2Hash": 0, "MurmurCityHash": 1}


def _in_window(policy, keys, n_lo, lo, hi):
    b0, b1 = oracle.buckets(POLID[policy], keys, n_lo)
    return ((b0 >= lo) & (b0 < hi)) | ((b1 >= lo) & (b1 < hi))


def _batch(rs, policy, live, pool, n_lo, lo, hi, size):
    """Unique keys: ~3/4 with a candidate bucket in the window [lo, hi) of the level's n_lo
    buckets, the rest anywhere; types mixed."""
    live = np.asarray(live, dtype=np.uint32)
    win_live = live[_in_window(policy, live, n_lo, lo, hi)]
    win_new = pool[_in_window(policy, pool, n_lo, lo, hi)]
    a = rs.choice(win_live, min(win_live.size, size // 2), replace=False)
    b = win_new[: min(win_new.size, size // 4)]
    c = rs.choice(live, size // 8, replace=False)
    d = pool[~np.isin(pool, b)][: size // 8]
    keys = np.unique(np.concatenate([a, b, c, d]).astype(np.uint32))
    keys = keys[rs.permutation(keys.size)]
    is_live = np.isin(keys, live)
    types = np.where(is_live, rs.choice([OP_INSERT, OP_LOOKUP, OP_LOOKUP, OP_DELETE, OP_INCREMENT], size=keys.size),
                     rs.choice([OP_INSERT, OP_INSERT, OP_LOOKUP], size=keys.size)).astype(np.uint8)
    vals = rs.randint(1, 2**32 - 1, size=keys.size).astype(np.uint32)
    used = np.isin(pool, keys)
    return types, keys, vals, pool[~used]


@pytest.mark.parametrize("policy", ["Default2Hash", "MurmurCityHash"])
@pytest.mark.parametrize("hints", [0, 4])
def test_split_while_ops_run(cuda, policy, hints):
    rs = np.random.RandomState(61)
    cap = 1 << 15
    pre, pool, _ = oracle.gen_keys(61, int(0.7 * cap), 200_000)
    m = oracle.ReplayMap()
    with HiveHashTable(cap, policy, max_capacity=cap * 4) as t:
        t.insert(pre, oracle.values_for(pre))
        m.insert(pre, oracle.values_for(pre))
        window = 512
        calls = 0
        while t.info()["level"] < 2:
            inf = t.info()
            n_lo = inf["base_buckets"] << inf["level"]
            lo = inf["split"]
            hi = min(lo + window, n_lo)
            live, _ = m.dump()
            types, keys, vals, pool = _batch(rs, policy, live, pool, n_lo, lo, hi, 4000)
            st, ov = t.apply_split(types, keys, vals, split_buckets=window, hints=hints)
            st, ov = st.cpu().numpy(), u32(ov)
            assert not (st == ST_ERROR).any()
            est, eov = m.apply(types, keys, vals, apply_mask=((types != OP_INSERT) | (st != 0)).astype(np.uint8))
            assert (st[types == OP_INSERT] != 0).all()
            np.testing.assert_array_equal(np.where((types == OP_INSERT) & (st == 3), 1, st), est,
                                          err_msg=f"call {calls}: window [{lo}, {hi}) of {n_lo}")
            np.testing.assert_array_equal(ov, eov, err_msg=f"call {calls}")
            after = t.info()
            assert (after["split"], after["level"]) == ((hi, inf["level"]) if hi < n_lo else (0, inf["level"] + 1))
            gk, gv = t.dump()
            rk, rv = m.dump()
            np.testing.assert_array_equal(gk, rk)
            np.testing.assert_array_equal(gv, rv)
            v = t.verify()
            assert v["tag_mismatch"] == v["misplaced"] == v["duplicate"] == 0, v
            calls += 1
        assert calls >= 2 * (cap // 8) // window
        t.check()


def test_split_without_ops_and_lookups_after(cuda):
    """A split with an empty batch, then read-only lookups in the new geometry."""
    cap = 1 << 14
    keys, absent, _ = oracle.gen_keys(63, int(0.8 * cap), 5000)
    vals = oracle.values_for(keys)
    with HiveHashTable(cap, max_capacity=cap * 2) as t:
        t.insert(keys, vals)
        nb = t.info()["num_buckets"]
        e = np.zeros(0, np.uint32)
        t.apply_split(e.astype(np.uint8), e, e, split_buckets=nb // 2)
        assert t.info()["split"] == nb // 2
        t.apply_split(e.astype(np.uint8), e, e, split_buckets=nb)
        inf = t.info()
        assert inf["level"] == 1 and inf["split"] == 0 and inf["num_buckets"] == 2 * nb
        v, f = t.find(np.concatenate([keys, absent]))
        f = f.cpu().numpy()
        assert f[: keys.size].all() and not f[keys.size:].any()
        np.testing.assert_array_equal(u32(v)[: keys.size], vals)
        assert t.size() == keys.size
