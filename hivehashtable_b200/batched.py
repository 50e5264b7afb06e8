"""Batched mixed-op execution (the reference's host loop of one hive_mixed_kernel launch per batch,
src/hive_dispatch.cu:119-226, rebuilt B200-first).

Two ways to run a sequence of uneven mixed batches on one table:

  plain       one hive_apply_ops call (a first pass and a deferred pass) per batch
  persistent  hive_apply_batches: one cooperative launch per segment of batches, a grid barrier
              between batches (include/hive_c.h)

Growth is planned on the host from the workload's known live-key counts: before a segment whose
peak would exceed `max_load` of the capacity, the table is grown (hive_resize doubles it by
linear-hashing splits), so a segment never needs the geometry to change while it runs.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np
import torch

from .table import HINT_UNIQUE_KEYS, HiveHashTable, as_device_u32, as_device_u8, library
from .workload import MixedWorkload


@dataclass
class RunResult:
    mode: str
    ms: float                 # device time of the whole sequence (CUDA events), growth included
    ops: int
    launches: int             # calls into the library that launch kernels
    resizes: int
    segments: List[tuple] = field(default_factory=list)

    @property
    def mops(self) -> float:
        return self.ops / (self.ms * 1e3)


class BatchedRunner:
    """hints: HIVE_HINT_* passed with every batch.  The workload generator puts each key in at
    most one op of a batch, so HINT_UNIQUE_KEYS holds by construction and is the default."""

    def __init__(self, table: HiveHashTable, wl: MixedWorkload, max_load: float = 0.85, hints: int = HINT_UNIQUE_KEYS):
        self.t, self.wl, self.max_load, self.hints = table, wl, max_load, hints
        dev = table.device
        self.types = as_device_u8(wl.types, dev)
        self.keys = as_device_u32(wl.keys, dev)
        self.vals = as_device_u32(wl.vals, dev)
        self.offsets = torch.from_numpy(wl.offsets.astype(np.int64)).to(dev)
        self.status = torch.zeros(wl.total_ops, dtype=torch.uint8, device=dev)
        self.outv = torch.zeros(wl.total_ops, dtype=torch.int32, device=dev)
        sizes = np.diff(wl.offsets.astype(np.int64))
        ins = np.add.reduceat((wl.types == 0).astype(np.int64), wl.offsets[:-1].astype(np.int64))
        ins[sizes == 0] = 0
        live_after = wl.live_after()
        live_before = np.concatenate([[wl.prefill_keys.size], live_after[:-1]])
        self.peak = live_before + ins          # most keys a batch can leave in the table mid-flight
        self.sizes = sizes

    def prefill(self) -> None:
        st = self.t.insert(self.wl.prefill_keys, self.wl.prefill_vals)
        assert bool((st != 0).all()), "prefill did not place every key"

    def _grow_for(self, peak: int) -> bool:
        cap = self.t.info()["capacity_slots"]
        if peak <= self.max_load * cap:
            return False
        while peak > self.max_load * cap:
            cap *= 2
        self.t.resize(cap)
        return True

    def plan(self, max_segment: int = 1 << 30) -> List[tuple]:
        """Segments [b0, b1) whose peak fits max_load of the capacity current at their start,
        with the capacity each needs (doubling)."""
        segs, b0 = [], 0
        cap = self.t.info()["capacity_slots"]
        nb = self.wl.n_batches
        while b0 < nb:
            while self.peak[b0] > self.max_load * cap:
                cap *= 2
            b1 = b0
            while b1 < nb and self.peak[b1] <= self.max_load * cap and b1 - b0 < max_segment:
                b1 += 1
            segs.append((b0, b1, cap))
            b0 = b1
        return segs

    def run_plain(self, stream=None) -> RunResult:
        lib, h = library(), self.t.handle
        s = torch.cuda.current_stream(self.t.device) if stream is None else stream
        tp, kp, vp = self.types.data_ptr(), self.keys.data_ptr(), self.vals.data_ptr()
        sp, op = self.status.data_ptr(), self.outv.data_ptr()
        offs = self.wl.offsets
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        resizes = launches = 0
        a.record(s)
        for bi in range(self.wl.n_batches):
            resizes += self._grow_for(int(self.peak[bi]))
            lo, n = int(offs[bi]), int(offs[bi + 1] - offs[bi])
            if n == 0:
                continue
            rc = lib.hive_apply_ops(h, tp + lo, kp + 4 * lo, vp + 4 * lo, n, sp + lo, op + 4 * lo, self.hints,
                                    s.cuda_stream)
            assert rc == 0, rc
            launches += 1
        b.record(s)
        torch.cuda.synchronize()
        return RunResult("plain", a.elapsed_time(b), self.wl.total_ops, launches, resizes)

    def run_persistent(self, threads_per_block: int = 256, blocks_per_sm: int = 0, max_segment: int = 1 << 30,
                       stream=None) -> RunResult:
        s = torch.cuda.current_stream(self.t.device) if stream is None else stream
        segs = self.plan(max_segment)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        resizes = 0
        a.record(s)
        for b0, b1, cap in segs:
            if self.t.info()["capacity_slots"] < cap:
                self.t.resize(cap)
                resizes += 1
            mx = int(self.sizes[b0:b1].max()) if b1 > b0 else 1
            self.t.apply_batches(self.types, self.keys, self.vals, self.offsets[b0:b1 + 1], max(mx, 1),
                                 self.status, self.outv, self.hints, threads_per_block, blocks_per_sm, stream=s)
        b.record(s)
        torch.cuda.synchronize()
        return RunResult("persistent", a.elapsed_time(b), self.wl.total_ops, len(segs), resizes, segs)
