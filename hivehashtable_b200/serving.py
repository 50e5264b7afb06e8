"""Served request loop (lib/libhive_serve.so, include/hive_serve.h) and its workloads.

The reference's nearest path is its YCSB driver (src/hashTableBenchmark.cc:434-570): one
closed-loop bulk launch.  Here requests arrive open-loop (Poisson) and a native loop batches them
continuously; latency is arrival -> result on the host.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass
from pathlib import Path
from typing import Optional

import numpy as np

from . import workload as wl
from .table import HiveHashTable, HiveError, library

_LIB = Path(__file__).resolve().parent / "lib" / "libhive_serve.so"
_lib = None

MIXES = {"A": 0, "B": 1, "C": 2, "D": 3}  # 50/50 lookup/update, 95/5, 100 % lookup, 95 % lookup / 5 % new


class ServeConfig(ctypes.Structure):
    _fields_ = [("depth", ctypes.c_uint32), ("max_batch", ctypes.c_uint32), ("max_load", ctypes.c_double),
                ("live_keys", ctypes.c_uint64), ("grow_start", ctypes.c_double)]


class ServeStats(ctypes.Structure):
    _fields_ = [("batches", ctypes.c_uint64), ("device_lookups", ctypes.c_uint64),
                ("device_upserts", ctypes.c_uint64), ("resizes", ctypes.c_uint64), ("refused", ctypes.c_uint64),
                ("wall_s", ctypes.c_double), ("grow_steps", ctypes.c_uint64), ("drains", ctypes.c_uint64),
                ("form_s", ctypes.c_double), ("launch_s", ctypes.c_double), ("answer_s", ctypes.c_double),
                ("idle_s", ctypes.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not _LIB.exists():
            raise ImportError(f"{_LIB} is missing: build it with `python -m hivehashtable_b200.build`")
        library()  # the core library first (libhive_serve.so links it)
        L = ctypes.CDLL(str(_LIB))
        P = ctypes.c_void_p
        L.hive_serve_run.restype = ctypes.c_int32
        L.hive_serve_run.argtypes = [P, ctypes.POINTER(ServeConfig), P, P, P, P, ctypes.c_uint64, P, P, P,
                                     ctypes.POINTER(ServeStats)]
        _lib = L
    return _lib


class ServedWorkload:
    """n_records preloaded records and n_requests requests of a mix, keys Zipf(theta) over the
    records (csrc/hive_workload.cpp, hive_wl_served)."""

    def __init__(self, seed: int, n_records: int, n_requests: int, mix: str, theta: float = 0.99):
        L = wl.lib()
        if not hasattr(L, "_served_bound"):
            L.hive_wl_served.restype = None
            L.hive_wl_served.argtypes = [ctypes.c_uint64] * 3 + [ctypes.c_int, ctypes.c_double] + [ctypes.c_void_p] * 4
            L._served_bound = True
        self.preload_keys = np.empty(n_records, dtype=np.uint32)
        self.types = np.empty(n_requests, dtype=np.uint8)
        self.keys = np.empty(n_requests, dtype=np.uint32)
        self.vals = np.empty(n_requests, dtype=np.uint32)
        L.hive_wl_served(seed, n_records, n_requests, MIXES[mix], theta, self.preload_keys.ctypes.data,
                         self.types.ctypes.data, self.keys.ctypes.data, self.vals.ctypes.data)
        self.preload_vals = wl.values_for(self.preload_keys)
        self.mix = mix


def poisson_arrivals(n: int, rate: float, seed: int = 0) -> np.ndarray:
    """Arrival times (s) of a Poisson process of `rate` requests/s; rate <= 0: all at 0."""
    if rate <= 0:
        return np.zeros(n, dtype=np.float64)
    rng = np.random.default_rng(seed)
    return np.cumsum(rng.exponential(1.0 / rate, size=n))


@dataclass
class ServeResult:
    out_vals: np.ndarray
    out_status: np.ndarray
    done: np.ndarray
    arrival: np.ndarray
    stats: dict

    @property
    def latency(self) -> np.ndarray:
        return self.done - self.arrival

    def summary(self) -> dict:
        lat = self.latency * 1e3
        n = self.done.size
        span = float(self.done.max() - self.arrival.min()) if n else 0.0
        return {"requests": n, "mops": n / span / 1e6 if span > 0 else None,
                "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
                "p999_ms": float(np.percentile(lat, 99.9)), "max_ms": float(lat.max()), **self.stats}


def serve(table: HiveHashTable, types, keys, vals, arrival, depth: int = 4, max_batch: int = 1 << 14,
          max_load: float = 0.9, live_keys: Optional[int] = None, grow_start: Optional[float] = None) -> ServeResult:
    """Run the request stream through the native loop.  Growth is incremental from `grow_start`
    (default 0.8 * max_load; 0 = off, grow at once after a drain when max_load would be passed)."""
    types = np.ascontiguousarray(types, dtype=np.uint8)
    keys = np.ascontiguousarray(keys, dtype=np.uint32)
    vals = np.ascontiguousarray(vals, dtype=np.uint32)
    arrival = np.ascontiguousarray(arrival, dtype=np.float64)
    n = keys.size
    # written (not just allocated) before the loop: np.zeros maps zero pages lazily, and the page
    # faults of first writes would land on the answering thread inside the timed loop
    out_v = np.empty(n, dtype=np.uint32)
    out_s = np.empty(n, dtype=np.uint8)
    done = np.empty(n, dtype=np.float64)
    for a in (out_v, out_s, done):
        a.fill(0)
    if grow_start is None:
        grow_start = 0.8 * max_load
    cfg = ServeConfig(depth, max_batch, max_load, table.size() if live_keys is None else live_keys, grow_start)
    st = ServeStats()
    rc = lib().hive_serve_run(table.handle, ctypes.byref(cfg), types.ctypes.data, keys.ctypes.data, vals.ctypes.data,
                              arrival.ctypes.data, n, out_v.ctypes.data, out_s.ctypes.data, done.ctypes.data,
                              ctypes.byref(st))
    if rc:
        raise HiveError(rc, "hive_serve_run")
    return ServeResult(out_v, out_s, done, arrival, st.as_dict())
