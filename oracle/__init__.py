"""TEST INFRASTRUCTURE: the oracle (CPU restatement of the Hive table's semantics and algorithm).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg (`cpu_baseline`,
`--impl reference`) may import this package, and only as the checker or the CPU baseline; the
product (hivehashtable_b200) never calls it.  Sources: oracle/hive_oracle.cpp (each function cites
the reference file:line it restates); build: oracle/build.py.
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path
from typing import Optional, Tuple

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "lib" / "libhive_oracle.so"
REF_DIR = HERE / "_ref"

_lib = None
_P, _U64, _U32, _I32, _D = ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint32, ctypes.c_int, ctypes.c_double


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            from . import build
            build.build_oracle()
        L = ctypes.CDLL(str(LIB_PATH))
        sig = {
            "hive_oracle_raw_hash": (_U32, [_I32, _I32, _U32]),
            "hive_oracle_buckets": (None, [_I32, _P, _U64, _U32, _P, _P]),
            "hive_oracle_sm64": (_U64, [ctypes.POINTER(_U64)]),
            "hive_oracle_gen_keys": (_U64, [_U64, _U64, _U64, _P, _P]),
            "hive_oracle_values": (None, [_P, _U64, _P]),
            "hive_oracle_shuffle_u32": (None, [_P, _U64, ctypes.POINTER(_U64)]),
            "hive_oracle_lookup_set": (None, [_P, _U64, _P, _U64, _U64, ctypes.POINTER(_U64), _P]),
            "hive_oracle_map_new": (_P, []),
            "hive_oracle_map_free": (None, [_P]),
            "hive_oracle_map_clear": (None, [_P]),
            "hive_oracle_map_size": (_U64, [_P]),
            "hive_oracle_map_insert": (None, [_P, _P, _P, _U64, _P, _P]),
            "hive_oracle_map_find": (None, [_P, _P, _U64, _P, _P]),
            "hive_oracle_map_erase": (None, [_P, _P, _U64, _P]),
            "hive_oracle_map_apply": (None, [_P, _P, _P, _P, _U64, _P, _P, _P]),
            "hive_oracle_map_dump": (_U64, [_P, _P, _P, _U64]),
            "hive_oracle_serial_selftest": (_U64, [_U64, _U64, _I32]),
            "hive_oracle_map_check_serial": (_U64, [_P, _P, _P, _P, _P, _U64, _P, _P, _P, _P, _U64,
                                                    ctypes.POINTER(_U64)]),
            "hive_oracle_cpu_new": (_P, [_I32, _U64, _I32]),
            "hive_oracle_cpu_free": (None, [_P]),
            "hive_oracle_cpu_failed": (_U64, [_P]),
            "hive_oracle_cpu_insert": (_D, [_P, _P, _P, _U64, _P, _I32]),
            "hive_oracle_cpu_find": (_D, [_P, _P, _U64, _P, _P, _I32]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _p(a: Optional[np.ndarray]):
    return None if a is None else a.ctypes.data


def _u32(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.uint32))


# ---- hashes ------------------------------------------------------------------------------------
def raw_hash(policy: int, idx: int, key: int) -> int:
    return lib().hive_oracle_raw_hash(policy, idx, key)


def buckets(policy: int, keys, num_buckets: int) -> Tuple[np.ndarray, np.ndarray]:
    k = _u32(keys)
    b0 = np.empty_like(k)
    b1 = np.empty_like(k)
    lib().hive_oracle_buckets(policy, _p(k), k.size, num_buckets, _p(b0), _p(b1))
    return b0, b1


# ---- generators ----------------------------------------------------------------------------------
def gen_keys(seed: int, n_present: int, n_absent: int = 0):
    present = np.empty(n_present, dtype=np.uint32)
    absent = np.empty(n_absent, dtype=np.uint32)
    st = lib().hive_oracle_gen_keys(seed, n_present, n_absent, _p(present), _p(absent))
    return present, absent, int(st)


def values_for(keys) -> np.ndarray:
    k = _u32(keys)
    v = np.empty_like(k)
    lib().hive_oracle_values(_p(k), k.size, _p(v))
    return v


def shuffle(a: np.ndarray, state: int) -> int:
    st = ctypes.c_uint64(state)
    lib().hive_oracle_shuffle_u32(_p(a), a.size, ctypes.byref(st))
    return int(st.value)


def lookup_set(inserted, absent, n_present: int, n_absent: int, state: int):
    ins, ab = _u32(inserted), _u32(absent)
    out = np.empty(n_present + n_absent, dtype=np.uint32)
    st = ctypes.c_uint64(state)
    lib().hive_oracle_lookup_set(_p(ins), ins.size, _p(ab), n_present, n_absent, ctypes.byref(st), _p(out))
    return out, int(st.value)


# ---- std::unordered_map replay -----------------------------------------------------------------
class ReplayMap:
    """The semantic oracle: a std::unordered_map<uint32_t, uint32_t> replay of every op."""

    def __init__(self):
        self._h = lib().hive_oracle_map_new()

    def __del__(self):
        if getattr(self, "_h", None):
            lib().hive_oracle_map_free(self._h)
            self._h = None

    def __len__(self):
        return int(lib().hive_oracle_map_size(self._h))

    def clear(self):
        lib().hive_oracle_map_clear(self._h)

    def insert(self, keys, vals, apply_mask=None) -> np.ndarray:
        k, v = _u32(keys), _u32(vals)
        m = None if apply_mask is None else np.ascontiguousarray(apply_mask, dtype=np.uint8)
        st = np.empty(k.size, dtype=np.uint8)
        lib().hive_oracle_map_insert(self._h, _p(k), _p(v), k.size, _p(m), _p(st))
        return st

    def find(self, keys):
        k = _u32(keys)
        v = np.empty_like(k)
        f = np.empty(k.size, dtype=np.uint8)
        lib().hive_oracle_map_find(self._h, _p(k), k.size, _p(v), _p(f))
        return v, f

    def erase(self, keys) -> np.ndarray:
        k = _u32(keys)
        st = np.empty(k.size, dtype=np.uint8)
        lib().hive_oracle_map_erase(self._h, _p(k), k.size, _p(st))
        return st

    def apply(self, types, keys, vals, apply_mask=None):
        t = np.ascontiguousarray(types, dtype=np.uint8)
        k, v = _u32(keys), _u32(vals)
        m = None if apply_mask is None else np.ascontiguousarray(apply_mask, dtype=np.uint8)
        st = np.empty(k.size, dtype=np.uint8)
        ov = np.empty(k.size, dtype=np.uint32)
        lib().hive_oracle_map_apply(self._h, _p(t), _p(k), _p(v), k.size, _p(m), _p(st), _p(ov))
        return st, ov

    def check_serial(self, types, keys, vals, launch, status, out_vals, fin_keys, fin_vals):
        """Per-key serialisation check of concurrent launches (hive_oracle_map_check_serial): for
        every key, some order of its ops that keeps launch order (any order inside a launch) must
        give each observed status / out value and the key's state in the final contents
        (fin_keys sorted).  Returns (number of keys with no such order, lowest op index of one of
        them or -1); with 0 the map advances to the final state of every key the run touched."""
        t = np.ascontiguousarray(types, dtype=np.uint8)
        k, v = _u32(keys), _u32(vals)
        b = _u32(launch)
        st = np.ascontiguousarray(status, dtype=np.uint8)
        ov = _u32(out_vals)
        fk, fv = _u32(fin_keys), _u32(fin_vals)
        assert t.size == k.size == v.size == b.size == st.size == ov.size and fk.size == fv.size
        first = ctypes.c_uint64()
        bad = lib().hive_oracle_map_check_serial(self._h, _p(t), _p(k), _p(v), _p(b), k.size, _p(st), _p(ov),
                                                 _p(fk), _p(fv), fk.size, ctypes.byref(first))
        return int(bad), (-1 if bad == 0 else int(first.value))

    def dump(self):
        n = len(self)
        k = np.empty(n, dtype=np.uint32)
        v = np.empty(n, dtype=np.uint32)
        lib().hive_oracle_map_dump(self._h, _p(k), _p(v), n)
        return k, v


def serial_selftest(seed: int, trials: int, max_ops: int) -> int:
    """Disagreements between the closed-form and the searched per-key serialisation checks on
    random single-launch groups (0 expected)."""
    return int(lib().hive_oracle_serial_selftest(seed, trials, max_ops))


# ---- multithreaded CPU bucketed cuckoo table ----------------------------------------------------
class CpuTable:
    """The CPU baseline: same policy, 8-slot buckets, CAS claims, depth-1 eviction, stash."""

    def __init__(self, policy: int, capacity_slots: int, max_evictions: int = 8):
        self._h = lib().hive_oracle_cpu_new(policy, capacity_slots, max_evictions)

    def __del__(self):
        if getattr(self, "_h", None):
            lib().hive_oracle_cpu_free(self._h)
            self._h = None

    def insert(self, keys, vals, threads: int = 1):
        k, v = _u32(keys), _u32(vals)
        st = np.empty(k.size, dtype=np.uint8)
        t = lib().hive_oracle_cpu_insert(self._h, _p(k), _p(v), k.size, _p(st), threads)
        return st, t

    def find(self, keys, threads: int = 1):
        k = _u32(keys)
        v = np.empty_like(k)
        f = np.empty(k.size, dtype=np.uint8)
        t = lib().hive_oracle_cpu_find(self._h, _p(k), k.size, _p(v), _p(f), threads)
        return v, f, t

    @property
    def failed(self) -> int:
        return int(lib().hive_oracle_cpu_failed(self._h))


def host_threads() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1
