"""hive_insert_noalloc: the insert entry point for callers that cannot allocate device memory.

hive_insert may grow its second-pass queue with cudaMalloc; callers that own all device memory
through their own pool, or must not let an allocation stall the device in a latency-bound loop,
use hive_insert_noalloc, whose queue is a fixed array compiled into the library (at most
HIVE_NOALLOC_MAX_OPS ops per call).  This test calls both entry points through the C ABI on
two tables, two calls in a row, and requires the same outcome: the same per-op result class
(new key / updated key / not placed), the same lookups and the same key->value set.

The file is named to be collected last; it must pass alone in a fresh process as well.
"""
import ctypes

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
    return st.cpu().numpy()


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
    with HiveHashTable(cap, policy) as ta, HiveHashTable(cap, policy) as tb:
        for kk, vv in ((keys, vals), (keys2, vals2)):
            sa = _call(lib.hive_insert, ta, kk, vv)
            sb = _call(lib.hive_insert_noalloc, tb, kk, vv)
            assert not (sb == 0xEE).any() and not (sb == 255).any()
            np.testing.assert_array_equal(_classes(sb), _classes(sa))
            va, fa = ta.find(kk)
            vb, fb = tb.find(kk)
            np.testing.assert_array_equal(fb.cpu().numpy(), fa.cpu().numpy())
            np.testing.assert_array_equal(u32(vb), u32(va))
            ka, xa = ta.dump()
            kb, xb = tb.dump()
            np.testing.assert_array_equal(kb, ka)
            np.testing.assert_array_equal(xb, xa)
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
