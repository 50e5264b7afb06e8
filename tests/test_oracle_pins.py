"""The oracle pinned against the reference's own code and the committed golden fixtures.

hash_kats_*.npz hold outputs of the reference's hash functions compiled from its tree
(include/hash.hpp, UniformHashFunction/src/hash_function.cu); see tests/golden/make_golden.py.
"""
from pathlib import Path

import numpy as np
import pytest

import oracle

GOLD = Path(__file__).resolve().parent / "golden"


def _raw(policy, idx, keys):
    return np.array([oracle.raw_hash(policy, idx, int(k)) for k in keys], dtype=np.uint64)


def test_hash1_murmur_city_match_reference_hash_hpp():
    g = np.load(GOLD / "hash_kats_inc.npz")
    keys = g["keys"]
    assert keys.size >= 1024 and 0 in keys and 0xFFFFFFFF in keys
    np.testing.assert_array_equal(_raw(0, 0, keys).astype(np.uint32), g["hash1"])
    mur, cty = _raw(1, 0, keys), _raw(1, 1, keys)
    for j, m in enumerate(g["mods"].astype(np.uint64)):
        np.testing.assert_array_equal((mur % m).astype(np.uint32), g["murmur"][:, j], err_msg=f"murmur % {m}")
        np.testing.assert_array_equal((cty % m).astype(np.uint32), g["city"][:, j], err_msg=f"city % {m}")


def test_hash2_matches_reference_plain_c_form():
    g = np.load(GOLD / "hash_kats_uhf.npz")
    keys, p = g["keys"], np.uint64(g["prime"])
    np.testing.assert_array_equal((_raw(0, 0, keys) % p).astype(np.uint32), g["hash1"])
    np.testing.assert_array_equal((_raw(0, 1, keys) % p).astype(np.uint32), g["hash2"])


def test_bucket_policy_is_hash_mod_num_buckets():
    keys = np.arange(1, 5000, dtype=np.uint32) * np.uint32(2654435761)
    for policy in (0, 1):
        for nb in (1, 3, 163840, 1 << 23):
            b0, b1 = oracle.buckets(policy, keys, nb)
            np.testing.assert_array_equal(b0, (_raw(policy, 0, keys) % nb).astype(np.uint32))
            np.testing.assert_array_equal(b1, (_raw(policy, 1, keys) % nb).astype(np.uint32))


@pytest.mark.parametrize("seed", [42, 7, 11, 13, 17])
def test_generators_match_golden(seed):
    g = np.load(GOLD / "generators.npz")
    present, absent, st = oracle.gen_keys(seed, 64, 16)
    np.testing.assert_array_equal(present, g[f"present_{seed}"])
    np.testing.assert_array_equal(absent, g[f"absent_{seed}"])
    np.testing.assert_array_equal(oracle.values_for(present), g[f"values_{seed}"])
    assert present.min() >= 1 and present.max() <= 0xFFFFFFFD
    assert len(set(present.tolist()) | set(absent.tolist())) == 80
    sh = np.arange(64, dtype=np.uint32)
    st2 = oracle.shuffle(sh, st)
    np.testing.assert_array_equal(sh, g[f"shuffle_{seed}"])
    look, st3 = oracle.lookup_set(present, absent, 24, 8, st2)
    np.testing.assert_array_equal(look, g[f"lookup_{seed}"])
    np.testing.assert_array_equal(np.array([st, st2, st3], dtype=np.uint64), g[f"states_{seed}"])


def test_bulk_small_replay_matches_golden():
    g = np.load(GOLD / "bulk_small.npz")
    m = oracle.ReplayMap()
    np.testing.assert_array_equal(m.insert(g["keys"], g["values"]), g["insert_status"])
    v, f = m.find(g["lookup_keys"])
    np.testing.assert_array_equal(f, g["found"])
    np.testing.assert_array_equal(v, g["found_values"])
    assert f.sum() == g["keys"].size // 2
