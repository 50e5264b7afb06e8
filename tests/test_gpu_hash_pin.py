"""Device hashing pinned against the reference's own device code: oracle/_ref/libhive_ref_hashdev.so
is the reference's include/HashPolicies.cuh + include/hash.hpp (hash2 with its inline-PTX steps)
compiled for sm_100a by oracle/build.py.  The oracle, the reference and the product's kernels
must choose the same two buckets for every key."""
import ctypes

import numpy as np
import pytest

import oracle
from hivehashtable_b200 import HiveHashTable, u32

pytestmark = pytest.mark.gpu
REF = oracle.REF_DIR / "libhive_ref_hashdev.so"


@pytest.fixture(scope="module")
def ref():
    if not REF.exists():
        pytest.skip("reference device pin not built (needs the reference tree at build time)")
    L = ctypes.CDLL(str(REF))
    L.ref_dev_buckets.restype = ctypes.c_int
    L.ref_dev_buckets.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_uint32,
                                  ctypes.c_void_p, ctypes.c_void_p]
    return L


@pytest.mark.parametrize("pid,policy", [(0, "Default2Hash"), (1, "MurmurCityHash")])
def test_reference_device_buckets(cuda, ref, pid, policy):
    rs = np.random.RandomState(pid)
    keys = np.concatenate([np.array([0, 1, 2, 0x7FFFFFFF, 0x80000000, 0xFFFFFFFE, 0xFFFFFFFF], np.uint32),
                           rs.randint(0, 2**32, size=200_000, dtype=np.uint64).astype(np.uint32)])
    for cap in (8, 1_310_720, 1 << 22, 1 << 26, 7 * 8):
        nb = cap // 8
        r0 = np.empty_like(keys)
        r1 = np.empty_like(keys)
        assert ref.ref_dev_buckets(pid, keys.ctypes.data, keys.size, nb, r0.ctypes.data, r1.ctypes.data) == 0
        o0, o1 = oracle.buckets(pid, keys, nb)
        np.testing.assert_array_equal(o0, r0)
        np.testing.assert_array_equal(o1, r1)
        with HiveHashTable(cap, policy) as t:
            b0, b1 = t.bucket_of(keys)
            np.testing.assert_array_equal(u32(b0), r0)
            np.testing.assert_array_equal(u32(b1), r1)
    # full-range raw hashes: modulus 2^32 - 1 leaves every value but one intact
    r0 = np.empty_like(keys)
    r1 = np.empty_like(keys)
    assert ref.ref_dev_buckets(pid, keys.ctypes.data, keys.size, 0xFFFFFFFF, r0.ctypes.data, r1.ctypes.data) == 0
    o0, o1 = oracle.buckets(pid, keys, 0xFFFFFFFF)
    np.testing.assert_array_equal(o0, r0)
    np.testing.assert_array_equal(o1, r1)
