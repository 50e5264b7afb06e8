"""Python mirror of the Hive table interface over the C ABI (include/hive_c.h).

The reference's host interface is C++ (include/hive_hash_table.cuh:50-144); its C++ form is
rebuilt in csrc/hive_compat.cpp.  This module gives the same operations to Python callers (the
tests and bench.py) with torch tensors as device memory.  It loads the in-tree
lib/libhive_b200.so and raises if that library is missing: there is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import os
import warnings
from pathlib import Path
from typing import Optional, Tuple

import numpy as np
import torch

_LIB_DIR = Path(__file__).resolve().parent / "lib"
CORE_LIB = _LIB_DIR / "libhive_b200.so"

# Status codes (include/hive_c.h)
HIVE_OK = 0
ERRORS = {
    1: "HIVE_ERR_INVALID_ARG",
    2: "HIVE_ERR_CUDA",
    3: "HIVE_ERR_OOM",
    4: "HIVE_ERR_LOCK_TIMEOUT",
    5: "HIVE_ERR_RETRY_LIMIT",
    6: "HIVE_ERR_CAPACITY",
    7: "HIVE_ERR_NO_DEVICE",
    8: "HIVE_ERR_TOO_LARGE",
}
ST_FAIL, ST_INSERTED, ST_UPDATED, ST_STASHED, ST_ERROR = 0, 1, 2, 3, 255
OP_INSERT, OP_LOOKUP, OP_DELETE, OP_INCREMENT, OP_NONE = 0, 1, 2, 3, 4
HINT_NO_DELETES = 1
HINT_LOOKUPS_ONLY = 2
HINT_UNIQUE_KEYS = 4
NUM_COUNTERS = 16
COUNTER_NAMES = {0: "slow_path", 1: "evictions", 2: "stash_push", 3: "failed", 4: "lock_timeout",
                 5: "retry_out", 6: "dup_fixed", 7: "lock_waits", 15: "error_bits"}
# Launch-tuning knobs (HIVE_TUNE_*): how a batch runs, never what it computes
TUNES = {"region_insert": 0, "region_find": 1, "subbatches": 2, "second_pass_blocks": 3, "bulk_retag": 4,
         "tags": 5, "l2_window": 6, "stash_depth": 7, "binned": 8}

# Policy names accepted by the reference's dispatcher (src/hive_dispatch.cu:829-871).  The
# ones outside the hot path fall back to Default2Hash with a message, as the reference does for
# unknown names.
POLICIES = {"Default2Hash": 0, "MurmurCityHash": 1}


class HiveError(RuntimeError):
    def __init__(self, code: int, what: str):
        self.code = code
        super().__init__(f"{what}: {ERRORS.get(code, code)} ({_strerror(code)})")


class _Config(ctypes.Structure):
    _fields_ = [("capacity_slots", ctypes.c_uint64), ("max_capacity_slots", ctypes.c_uint64),
                ("policy", ctypes.c_int32), ("max_evictions", ctypes.c_int32),
                ("device", ctypes.c_int32), ("reserved", ctypes.c_uint32)]


class Info(ctypes.Structure):
    _fields_ = [("num_buckets", ctypes.c_uint64), ("capacity_slots", ctypes.c_uint64),
                ("max_buckets", ctypes.c_uint64), ("base_buckets", ctypes.c_uint32),
                ("level", ctypes.c_uint32), ("split", ctypes.c_uint32), ("policy", ctypes.c_int32),
                ("max_evictions", ctypes.c_int32), ("flags", ctypes.c_uint32),
                ("device", ctypes.c_int32), ("reserved", ctypes.c_uint32)]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_ if name != "reserved"}


_lib: Optional[ctypes.CDLL] = None

# (name, restype, argtypes) of every entry point declared in include/hive_c.h
_P, _U64, _I32, _U32 = ctypes.c_void_p, ctypes.c_uint64, ctypes.c_int32, ctypes.c_uint32
ABI = [
    ("hive_create", _I32, [ctypes.POINTER(_Config), ctypes.POINTER(_P)]),
    ("hive_destroy", _I32, [_P]),
    ("hive_clear", _I32, [_P, _P]),
    ("hive_insert", _I32, [_P, _P, _P, _U64, _P, _P]),
    ("hive_insert_noalloc", _I32, [_P, _P, _P, _U64, _P, _P]),
    ("hive_find", _I32, [_P, _P, _U64, _P, _P, _P]),
    ("hive_insert_host", _I32, [_P, _P, _P, _U64, _P, _P]),
    ("hive_find_host", _I32, [_P, _P, _U64, _P, _P, _P]),
    ("hive_erase", _I32, [_P, _P, _U64, _P, _P]),
    ("hive_apply_ops", _I32, [_P, _P, _P, _P, _U64, _P, _P, _U32, _P]),
    ("hive_apply_reference_ops", _I32, [_P, _P, _U64, _P, _U32, _P]),
    ("hive_apply_ops_split", _I32, [_P, _P, _P, _P, _U64, _P, _P, _U32, _U64, _P]),
    ("hive_apply_batches", _I32, [_P, _P, _P, _P, _P, _U32, _U64, _P, _P, _U32, _I32, _I32, _P]),
    ("hive_size", _I32, [_P, ctypes.POINTER(_U64), _P]),
    ("hive_dump", _I32, [_P, _P, _U64, ctypes.POINTER(_U64), _P]),
    ("hive_load", _I32, [_P, _P, _U64, ctypes.POINTER(_U64), _P]),
    ("hive_resize", _I32, [_P, _U64, _P]),
    ("hive_bucket_of", _I32, [_P, _P, _U64, _P, _P, _P]),
    ("hive_get_info", _I32, [_P, ctypes.POINTER(Info)]),
    ("hive_counters", _I32, [_P, _P, _P]),
    ("hive_check", _I32, [_P, _P]),
    ("hive_verify", _I32, [_P, _P, _P]),
    ("hive_debug_hold_lock", _I32, [_P, _U64, _I32, _P]),
    ("hive_set_tuning", _I32, [_P, _I32, ctypes.c_int64]),
    ("hive_get_tuning", _I32, [_P, _I32, ctypes.POINTER(ctypes.c_int64)]),
    ("hive_strerror", ctypes.c_char_p, [_I32]),
    ("hive_last_cuda_error", _I32, []),
]


def library(path: Optional[Path] = None) -> ctypes.CDLL:
    """Load libhive_b200.so (once).  Raises if it has not been built."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = Path(path) if path else CORE_LIB
    if not p.exists():
        raise ImportError(f"{p} is missing: build it with `python -m hivehashtable_b200.build` "
                          "(the table has no CPU implementation)")
    lib = ctypes.CDLL(str(p))
    for name, res, args in ABI:
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _lib = lib
    return lib


def _strerror(code: int) -> str:
    try:
        return library().hive_strerror(code).decode()
    except Exception:  # the library itself may be what is missing
        return "?"


def _check(rc: int, what: str) -> None:
    if rc != HIVE_OK:
        raise HiveError(rc, what)


def _ptr(t: Optional[torch.Tensor]) -> Optional[int]:
    return None if t is None else t.data_ptr()


def as_device_u32(x, device: torch.device) -> torch.Tensor:
    """A contiguous 4-byte device tensor holding the uint32 bit patterns of x (int32 storage)."""
    if isinstance(x, torch.Tensor):
        if x.element_size() != 4:
            x = x.to(torch.int64).to(torch.int32)
        t = x.view(torch.int32) if x.dtype != torch.int32 else x
        return t.to(device).contiguous()
    a = np.ascontiguousarray(np.asarray(x, dtype=np.uint32)).view(np.int32)
    return torch.from_numpy(a).to(device)


def as_device_u8(x, device: torch.device) -> torch.Tensor:
    if isinstance(x, torch.Tensor):
        return x.to(torch.uint8).to(device).contiguous()
    return torch.from_numpy(np.ascontiguousarray(np.asarray(x, dtype=np.uint8))).to(device)


def as_host_u32(x) -> torch.Tensor:
    """A contiguous 4-byte CPU tensor holding the uint32 bit patterns of x (no copy when x already
    is one, so a page-locked tensor stays page-locked)."""
    if isinstance(x, torch.Tensor):
        if x.device.type != "cpu":
            raise ValueError("host-buffer calls take CPU tensors or numpy arrays")
        if x.element_size() != 4:
            x = x.to(torch.int64).to(torch.int32)
        return (x.view(torch.int32) if x.dtype != torch.int32 else x).contiguous()
    return torch.from_numpy(np.ascontiguousarray(np.asarray(x, dtype=np.uint32)).view(np.int32))


def u32(t: torch.Tensor) -> np.ndarray:
    """Device int32 tensor -> host numpy uint32 (bit pattern preserved)."""
    return t.cpu().numpy().view(np.uint32)


class HiveHashTable:
    """A Hive hash table resident in one GPU's HBM.

    capacity       slots at creation (buckets = ceil(capacity / 8), as table_size / 8 in
                   src/hive_dispatch.cu:630-631)
    policy         "Default2Hash" or "MurmurCityHash" (include/HashPolicies.cuh); other reference
                   policy names fall back to Default2Hash with a warning
    max_evictions  cuckoo victims tried per insert (include/hive_hash_table.cuh:21, default 8)
    max_capacity   slots reserved for later growth (resize beyond it reallocates)
    """

    def __init__(self, capacity: int, policy: str = "Default2Hash", max_evictions: int = 8,
                 max_capacity: Optional[int] = None, device=None, tuning=None):
        lib = library()
        if not torch.cuda.is_available():
            raise HiveError(7, "HiveHashTable")
        if policy not in POLICIES:
            warnings.warn(f"Unknown Hash Policy: {policy}. Using Default2HashPolicy.")
            policy = "Default2Hash"
        self.policy = policy
        self.device = torch.device("cuda", torch.cuda.current_device() if device is None
                                   else torch.device(device).index or 0)
        # a tuned setting (hivehashtable_b200.autotune): a dict, or "cache" for the entry of this
        # GPU / policy / nearest capacity in the HIVE_TUNE_CACHE file (used by default when set)
        if tuning is None and os.environ.get("HIVE_TUNE_CACHE"):
            tuning = "cache"
        self.tuned = None
        if tuning == "cache":
            from .autotune import lookup_cached

            self.tuned = lookup_cached(Path(os.environ.get("HIVE_TUNE_CACHE", "")), torch.cuda.get_device_name(self.device),
                                       int(capacity), policy)
        elif isinstance(tuning, dict):
            self.tuned = dict(tuning)
        if self.tuned and "max_evictions" in self.tuned:
            max_evictions = int(self.tuned["max_evictions"])
        cfg = _Config(int(capacity), int(max_capacity or 0), POLICIES[policy], int(max_evictions),
                      self.device.index, 0)
        h = ctypes.c_void_p()
        _check(lib.hive_create(ctypes.byref(cfg), ctypes.byref(h)), "hive_create")
        self._h = h
        self._lib = lib
        if self.tuned:
            self.set_tuning(**{k: v for k, v in self.tuned.items() if k != "max_evictions"})

    # -- plumbing ---------------------------------------------------------------------------
    def _stream(self, stream=None) -> int:
        s = stream if stream is not None else torch.cuda.current_stream(self.device)
        return s.cuda_stream

    def _sync(self, stream=None) -> None:
        (stream if stream is not None else torch.cuda.current_stream(self.device)).synchronize()

    @property
    def handle(self) -> int:
        return self._h.value

    def close(self) -> None:
        if getattr(self, "_h", None) and self._h.value:
            _check(self._lib.hive_destroy(self._h), "hive_destroy")
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # -- operations ---------------------------------------------------------------------------
    def insert(self, keys, values, status: Optional[torch.Tensor] = None, stream=None) -> torch.Tensor:
        k = as_device_u32(keys, self.device)
        v = as_device_u32(values, self.device)
        if k.numel() != v.numel():
            raise ValueError("keys and values differ in length")
        if status is None:
            status = torch.empty(k.numel(), dtype=torch.uint8, device=self.device)
        _check(self._lib.hive_insert(self._h, _ptr(k), _ptr(v), k.numel(), _ptr(status),
                                     self._stream(stream)), "hive_insert")
        return status

    def find(self, keys, values: Optional[torch.Tensor] = None, found: Optional[torch.Tensor] = None,
             stream=None) -> Tuple[torch.Tensor, torch.Tensor]:
        k = as_device_u32(keys, self.device)
        if values is None:
            values = torch.empty(k.numel(), dtype=torch.int32, device=self.device)
        if found is None:
            found = torch.empty(k.numel(), dtype=torch.uint8, device=self.device)
        _check(self._lib.hive_find(self._h, _ptr(k), k.numel(), _ptr(values), _ptr(found),
                                   self._stream(stream)), "hive_find")
        return values, found

    def insert_host(self, keys, values, status: Optional[torch.Tensor] = None, stream=None,
                    sync: bool = True) -> torch.Tensor:
        """insert() from host memory with the copies overlapped with the work (hive_insert_host).
        Pass page-locked CPU tensors (and a page-locked `status`) for overlap.  With sync=False
        the call returns once queued: inputs and `status` belong to it until `stream` completes."""
        k, v = as_host_u32(keys), as_host_u32(values)
        if k.numel() != v.numel():
            raise ValueError("keys and values differ in length")
        if status is None:
            status = torch.empty(k.numel(), dtype=torch.uint8)
        s = self._stream(stream)
        _check(self._lib.hive_insert_host(self._h, _ptr(k), _ptr(v), k.numel(), _ptr(status), s),
               "hive_insert_host")
        if sync:
            self._sync(stream)
        return status

    def find_host(self, keys, values: Optional[torch.Tensor] = None, found: Optional[torch.Tensor] = None,
                  stream=None, sync: bool = True) -> Tuple[torch.Tensor, torch.Tensor]:
        """find() from host memory (hive_find_host); same rules as insert_host."""
        k = as_host_u32(keys)
        if values is None:
            values = torch.empty(k.numel(), dtype=torch.int32)
        if found is None:
            found = torch.empty(k.numel(), dtype=torch.uint8)
        s = self._stream(stream)
        _check(self._lib.hive_find_host(self._h, _ptr(k), k.numel(), _ptr(values), _ptr(found), s),
               "hive_find_host")
        if sync:
            self._sync(stream)
        return values, found

    def erase(self, keys, status: Optional[torch.Tensor] = None, stream=None) -> torch.Tensor:
        k = as_device_u32(keys, self.device)
        if status is None:
            status = torch.empty(k.numel(), dtype=torch.uint8, device=self.device)
        _check(self._lib.hive_erase(self._h, _ptr(k), k.numel(), _ptr(status), self._stream(stream)),
               "hive_erase")
        return status

    def apply(self, types, keys, values=None, hints: int = 0, stream=None) -> Tuple[torch.Tensor, torch.Tensor]:
        t = as_device_u8(types, self.device)
        k = as_device_u32(keys, self.device)
        v = None if values is None else as_device_u32(values, self.device)
        n = k.numel()
        status = torch.empty(n, dtype=torch.uint8, device=self.device)
        outv = torch.empty(n, dtype=torch.int32, device=self.device)
        _check(self._lib.hive_apply_ops(self._h, _ptr(t), _ptr(k), _ptr(v), n, _ptr(status), _ptr(outv),
                                        hints, self._stream(stream)), "hive_apply_ops")
        return status, outv

    def apply_split(self, types, keys, values=None, split_buckets: int = 0, hints: int = 0,
                    stream=None) -> Tuple[torch.Tensor, torch.Tensor]:
        """apply() while the same launch splits the next `split_buckets` buckets of the current
        level (hive_apply_ops_split): the table grows while the batch runs."""
        t = as_device_u8(types, self.device)
        k = as_device_u32(keys, self.device)
        v = None if values is None else as_device_u32(values, self.device)
        n = k.numel()
        status = torch.empty(n, dtype=torch.uint8, device=self.device)
        outv = torch.empty(n, dtype=torch.int32, device=self.device)
        _check(self._lib.hive_apply_ops_split(self._h, _ptr(t), _ptr(k), _ptr(v), n, _ptr(status), _ptr(outv), hints,
                                              int(split_buckets), self._stream(stream)), "hive_apply_ops_split")
        return status, outv

    def apply_batches(self, types: torch.Tensor, keys: torch.Tensor, values: Optional[torch.Tensor],
                      offsets: torch.Tensor, max_batch_ops: int, status: torch.Tensor, out_values: torch.Tensor,
                      hints: int = 0, threads_per_block: int = 256, blocks_per_sm: int = 0, stream=None) -> None:
        """Batches [offsets[b], offsets[b+1]) of device op arrays in one persistent launch
        (hive_apply_batches); outputs are written into status / out_values at global positions."""
        nb = offsets.numel() - 1
        _check(self._lib.hive_apply_batches(self._h, _ptr(types), _ptr(keys), _ptr(values), _ptr(offsets), nb,
                                            int(max_batch_ops), _ptr(status), _ptr(out_values), hints,
                                            threads_per_block, blocks_per_sm, self._stream(stream)),
               "hive_apply_batches")

    def apply_reference_ops(self, ops: torch.Tensor, hints: int = 0, stream=None) -> torch.Tensor:
        """ops: int64 tensor of shape (n, 2) holding the reference's 16-byte Operation records
        (row = [type, key]); returns int64 results (1 success, 0 otherwise)."""
        ops = ops.to(self.device).contiguous()
        if ops.dtype != torch.int64 or ops.dim() != 2 or ops.shape[1] != 2:
            raise ValueError("ops must be an int64 tensor of shape (n, 2)")
        res = torch.empty(ops.shape[0], dtype=torch.int64, device=self.device)
        _check(self._lib.hive_apply_reference_ops(self._h, _ptr(ops), ops.shape[0], _ptr(res), hints,
                                                  self._stream(stream)), "hive_apply_reference_ops")
        return res

    def size(self, stream=None) -> int:
        n = ctypes.c_uint64()
        _check(self._lib.hive_size(self._h, ctypes.byref(n), self._stream(stream)), "hive_size")
        return n.value

    def dump(self, stream=None) -> Tuple[np.ndarray, np.ndarray]:
        """All entries as host arrays (keys, values), sorted by key."""
        cap = self.size(stream)
        kv = torch.empty(max(cap, 1), dtype=torch.int64, device=self.device)
        n = ctypes.c_uint64()
        _check(self._lib.hive_dump(self._h, _ptr(kv), cap, ctypes.byref(n), self._stream(stream)),
               "hive_dump")
        if n.value != cap:
            raise HiveError(1, f"hive_dump: table changed size during dump ({n.value} != {cap})")
        a = kv[:cap].cpu().numpy().view(np.uint64)
        keys = (a & 0xFFFFFFFF).astype(np.uint32)
        vals = (a >> 32).astype(np.uint32)
        order = np.argsort(keys, kind="stable")
        return keys[order], vals[order]

    def dump_packed(self, stream=None) -> torch.Tensor:
        """All entries as one device int64 tensor of packed (value << 32) | key words, unordered:
        the format load() takes back."""
        cap = self.size(stream)
        kv = torch.empty(max(cap, 1), dtype=torch.int64, device=self.device)
        n = ctypes.c_uint64()
        _check(self._lib.hive_dump(self._h, _ptr(kv), cap, ctypes.byref(n), self._stream(stream)),
               "hive_dump")
        if n.value != cap:
            raise HiveError(1, f"hive_dump: table changed size during dump ({n.value} != {cap})")
        return kv[:cap]

    def load(self, keys, values=None, stream=None) -> None:
        """Replace the contents with the given entries (unique keys): `keys` alone is a packed
        int64 tensor as dump_packed() returns; with `values`, two uint32 arrays.  Grows the table
        to the next full level when the entries exceed load factor 0.9 of its unsplit level.  Raises HiveError(6) if any entry found no room
        (or has key 0); the table then holds the others."""
        if values is None:
            kv = keys.to(self.device).contiguous() if isinstance(keys, torch.Tensor) else \
                torch.from_numpy(np.ascontiguousarray(np.asarray(keys, dtype=np.uint64)).view(np.int64)).to(self.device)
            if kv.dtype != torch.int64 or kv.dim() != 1:
                raise ValueError("packed entries must be a 1-D int64 tensor")
        else:
            k = as_device_u32(keys, self.device).to(torch.int64) & 0xFFFFFFFF
            v = as_device_u32(values, self.device).to(torch.int64)
            if k.numel() != v.numel():
                raise ValueError("keys and values differ in length")
            kv = (v << 32) | k
        bad = ctypes.c_uint64()
        rc = self._lib.hive_load(self._h, _ptr(kv), kv.numel(), ctypes.byref(bad), self._stream(stream))
        if rc == 6 and bad.value:
            raise HiveError(6, f"hive_load: {bad.value} of {kv.numel()} entries not placed")
        _check(rc, "hive_load")

    def save(self, path, stream=None) -> None:
        """Write a checkpoint file (numpy .npz): the policy, the capacity and every entry."""
        kv = self.dump_packed(stream).cpu().numpy().view(np.uint64)
        inf = self.info()
        with open(path, "wb") as f:
            np.savez(f, kv=kv, policy=np.array(self.policy), base_buckets=np.uint64(inf["base_buckets"]),
                     num_buckets=np.uint64(inf["num_buckets"]), max_buckets=np.uint64(inf["max_buckets"]),
                     max_evictions=np.uint32(inf["max_evictions"]))

    @classmethod
    def restore(cls, path, device=None, stream=None) -> "HiveHashTable":
        """A new table from a checkpoint file written by save(): the saved policy, eviction bound and
        bucket geometry (creation size, then grown to the saved size), holding the saved entries."""
        with np.load(path) as z:
            kv, policy = z["kv"], str(z["policy"])
            base, nb, mx = int(z["base_buckets"]), int(z["num_buckets"]), int(z["max_buckets"])
            ev = int(z["max_evictions"])
        t = cls(base * 8, policy, max_evictions=ev, max_capacity=mx * 8, device=device)
        try:
            if nb > base:
                t.resize(nb * 8, stream)
            t.load(kv, stream=stream)
        except Exception:
            t.close()
            raise
        return t

    def clear(self, stream=None) -> None:
        _check(self._lib.hive_clear(self._h, self._stream(stream)), "hive_clear")

    def resize(self, target_slots: int, stream=None) -> None:
        _check(self._lib.hive_resize(self._h, int(target_slots), self._stream(stream)), "hive_resize")

    def bucket_of(self, keys, stream=None) -> Tuple[torch.Tensor, torch.Tensor]:
        k = as_device_u32(keys, self.device)
        b0 = torch.empty(k.numel(), dtype=torch.int32, device=self.device)
        b1 = torch.empty(k.numel(), dtype=torch.int32, device=self.device)
        _check(self._lib.hive_bucket_of(self._h, _ptr(k), k.numel(), _ptr(b0), _ptr(b1), self._stream(stream)),
               "hive_bucket_of")
        return b0, b1

    def info(self) -> dict:
        inf = Info()
        _check(self._lib.hive_get_info(self._h, ctypes.byref(inf)), "hive_get_info")
        return inf.as_dict()

    def counters(self, stream=None) -> dict:
        buf = (ctypes.c_uint64 * NUM_COUNTERS)()
        _check(self._lib.hive_counters(self._h, ctypes.cast(buf, ctypes.c_void_p), self._stream(stream)),
               "hive_counters")
        return {name: int(buf[i]) for i, name in COUNTER_NAMES.items()}

    def check(self, stream=None) -> None:
        _check(self._lib.hive_check(self._h, self._stream(stream)), "hive_check")

    def verify(self, stream=None) -> dict:
        """Structural check on the device (hive_verify): violation counts, all 0 when sound."""
        buf = (ctypes.c_uint64 * 4)()
        _check(self._lib.hive_verify(self._h, ctypes.cast(buf, ctypes.c_void_p), self._stream(stream)),
               "hive_verify")
        return {name: int(buf[i]) for i, name in enumerate(("tag_mismatch", "misplaced", "duplicate", "stale_tag"))}

    def debug_hold_lock(self, bucket: int, held: bool = True, stream=None) -> None:
        """Test hook: hold (or release) a bucket's eviction lock (hive_debug_hold_lock)."""
        _check(self._lib.hive_debug_hold_lock(self._h, int(bucket), int(bool(held)), self._stream(stream)),
               "hive_debug_hold_lock")

    def set_tuning(self, **knobs) -> None:
        """set_tuning(region_insert=1, subbatches=4, ...): see TUNES."""
        for name, value in knobs.items():
            _check(self._lib.hive_set_tuning(self._h, TUNES[name], int(value)), f"hive_set_tuning({name})")

    def tuning(self) -> dict:
        out = {}
        for name, key in TUNES.items():
            v = ctypes.c_int64()
            _check(self._lib.hive_get_tuning(self._h, key, ctypes.byref(v)), "hive_get_tuning")
            out[name] = v.value
        return out

    def load_factor(self) -> float:
        return self.size() / self.info()["capacity_slots"]
