"""Seeded synthetic workloads (ctypes over lib/libhive_workload.so, csrc/hive_workload.cpp).

The generator definitions (key draws, values, shuffles, lookup sets) are stated in
csrc/hive_workload.cpp; the seeds per workload are the ones below.
"""
from __future__ import annotations

import ctypes
from pathlib import Path
from typing import Tuple

import numpy as np

_LIB = Path(__file__).resolve().parent / "lib" / "libhive_workload.so"
_lib = None

SEED_SMALL = 42       # plain bulk path, 2^20 keys at LF 0.8
SEED_SWEEP = 7        # bulk sweep over capacity x load factor x present fraction
SEED_MIXED = 11       # batched mixed ops
SEED_RESIZE = 13      # dynamic resize
SEED_SERVED = 17      # served skewed workload


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not _LIB.exists():
            raise ImportError(f"{_LIB} is missing: build it with `python -m hivehashtable_b200.build`")
        L = ctypes.CDLL(str(_LIB))
        P, U64 = ctypes.c_void_p, ctypes.c_uint64
        L.hive_wl_sm64.restype = U64
        L.hive_wl_sm64.argtypes = [ctypes.POINTER(U64)]
        L.hive_wl_gen_keys.restype = U64
        L.hive_wl_gen_keys.argtypes = [U64, U64, U64, P, P]
        L.hive_wl_values.restype = None
        L.hive_wl_values.argtypes = [P, U64, P]
        L.hive_wl_shuffle.restype = None
        L.hive_wl_shuffle.argtypes = [P, U64, ctypes.POINTER(U64)]
        L.hive_wl_lookup_set.restype = None
        L.hive_wl_lookup_set.argtypes = [P, U64, P, U64, U64, ctypes.POINTER(U64), P]
        D = ctypes.c_double
        L.hive_wl_mixed_plan.restype = U64
        L.hive_wl_mixed_plan.argtypes = [U64, U64, D, D, P]
        L.hive_wl_mixed_fill.restype = U64
        L.hive_wl_mixed_fill.argtypes = [U64, U64, U64, D, D, P, P, P, P, P]
        _lib = L
    return _lib


def _p(a: np.ndarray) -> int:
    return a.ctypes.data


def gen_keys(seed: int, n_present: int, n_absent: int = 0) -> Tuple[np.ndarray, np.ndarray, int]:
    """n_present unique keys, then n_absent more unique keys not among them; returns the
    stream state after the last draw."""
    present = np.empty(n_present, dtype=np.uint32)
    absent = np.empty(n_absent, dtype=np.uint32)
    state = lib().hive_wl_gen_keys(seed, n_present, n_absent, _p(present), _p(absent))
    return present, absent, int(state)


def values_for(keys: np.ndarray) -> np.ndarray:
    keys = np.ascontiguousarray(keys, dtype=np.uint32)
    out = np.empty_like(keys)
    lib().hive_wl_values(_p(keys), keys.size, _p(out))
    return out


def shuffle(a: np.ndarray, state: int) -> int:
    """In-place Fisher-Yates of a uint32 array; returns the new stream state."""
    assert a.dtype == np.uint32 and a.flags.c_contiguous
    st = ctypes.c_uint64(state)
    lib().hive_wl_shuffle(_p(a), a.size, ctypes.byref(st))
    return int(st.value)


def lookup_set(inserted: np.ndarray, absent: np.ndarray, n_present: int, n_absent: int,
               state: int) -> Tuple[np.ndarray, int]:
    inserted = np.ascontiguousarray(inserted, dtype=np.uint32)
    absent = np.ascontiguousarray(absent, dtype=np.uint32)
    assert n_present <= inserted.size and n_absent <= absent.size
    out = np.empty(n_present + n_absent, dtype=np.uint32)
    st = ctypes.c_uint64(state)
    lib().hive_wl_lookup_set(_p(inserted), inserted.size, _p(absent), n_present, n_absent,
                             ctypes.byref(st), _p(out))
    return out, int(st.value)


def bulk_workload(seed: int, n: int, present_fraction: float, n_lookups: int | None = None):
    """Keys and values for a bulk insert of n unique keys, then a lookup set of n_lookups keys
    (default n) with the given present fraction (absent keys drawn from the same stream).

    Returns (keys, values, lookup_keys)."""
    n_lookups = n if n_lookups is None else n_lookups
    n_present = int(round(n_lookups * present_fraction))
    n_absent = n_lookups - n_present
    keys, absent, state = gen_keys(seed, n, n_absent)
    vals = values_for(keys)
    lk, _ = lookup_set(keys, absent, n_present, n_absent, state)
    return keys, vals, lk


class MixedWorkload:
    """Prefill keys and a sequence of mixed batches (csrc/hive_workload.cpp, hive_wl_mixed_fill):
    each batch is 50 % inserts of new keys, 40 % lookups (80 % of live keys), 10 % deletes of live
    keys, at most one op per key per batch, sizes floor(2^U) with U uniform in [log_lo, log_hi)."""

    def __init__(self, seed: int, prefill: int, n_batches: int, log_lo: float = 10.0, log_hi: float = 20.0):
        L = lib()
        sizes = np.empty(n_batches, dtype=np.uint64)
        total = L.hive_wl_mixed_plan(seed, n_batches, log_lo, log_hi, _p(sizes))
        self.prefill_keys = np.empty(prefill, dtype=np.uint32)
        self.types = np.empty(total, dtype=np.uint8)
        self.keys = np.empty(total, dtype=np.uint32)
        self.vals = np.empty(total, dtype=np.uint32)
        self.offsets = np.empty(n_batches + 1, dtype=np.uint64)
        self.final_live = int(L.hive_wl_mixed_fill(seed, prefill, n_batches, log_lo, log_hi, _p(self.prefill_keys),
                                                   _p(self.types), _p(self.keys), _p(self.vals), _p(self.offsets)))
        self.prefill_vals = values_for(self.prefill_keys)
        self.seed, self.n_batches = seed, n_batches

    @property
    def total_ops(self) -> int:
        return int(self.offsets[-1])

    def batch(self, b: int):
        lo, hi = int(self.offsets[b]), int(self.offsets[b + 1])
        return self.types[lo:hi], self.keys[lo:hi], self.vals[lo:hi]

    def live_after(self) -> np.ndarray:
        """Live-key count after each batch (prefill + inserts - deletes so far)."""
        ins = np.add.reduceat((self.types == 0).astype(np.int64), self.offsets[:-1].astype(np.int64))
        dels = np.add.reduceat((self.types == 2).astype(np.int64), self.offsets[:-1].astype(np.int64))
        return self.prefill_keys.size + np.cumsum(ins - dels)
