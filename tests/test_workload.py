"""The product's workload generator equals the oracle's restatement bit-for-bit."""
import numpy as np
import pytest

import oracle
from hivehashtable_b200 import workload


@pytest.mark.parametrize("seed,n,na", [(42, 1 << 12, 1 << 11), (7, 100_000, 5_000), (11, 0, 10), (13, 3, 0)])
def test_keys_values_shuffle_lookup_match_oracle(seed, n, na):
    p1, a1, s1 = workload.gen_keys(seed, n, na)
    p2, a2, s2 = oracle.gen_keys(seed, n, na)
    np.testing.assert_array_equal(p1, p2)
    np.testing.assert_array_equal(a1, a2)
    assert s1 == s2
    np.testing.assert_array_equal(workload.values_for(p1), oracle.values_for(p2))
    x1 = np.arange(n, dtype=np.uint32)
    x2 = x1.copy()
    assert workload.shuffle(x1, s1) == oracle.shuffle(x2, s2)
    np.testing.assert_array_equal(x1, x2)
    npres = n // 2
    l1, t1 = workload.lookup_set(p1, a1, npres, na, s1)
    l2, t2 = oracle.lookup_set(p2, a2, npres, na, s2)
    np.testing.assert_array_equal(l1, l2)
    assert t1 == t2


def test_bitmap_path_matches_oracle():
    # > 2^21 keys switches the product generator to its 512 MiB bitmap membership test.
    p1, a1, s1 = workload.gen_keys(7, 2_200_000, 1000)
    p2, a2, s2 = oracle.gen_keys(7, 2_200_000, 1000)
    assert s1 == s2
    np.testing.assert_array_equal(p1, p2)
    np.testing.assert_array_equal(a1, a2)
    assert np.unique(p1).size == p1.size


def test_bulk_workload_shapes():
    keys, vals, look = workload.bulk_workload(42, 1000, 0.5)
    assert keys.size == 1000 and vals.size == 1000 and look.size == 1000
    assert np.isin(look, keys).sum() == 500
