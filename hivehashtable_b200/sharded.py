"""Hash-partitioned Hive table over several GPUs (one process per GPU, torch.distributed).

Each rank owns the keys whose owner(key) is its rank and keeps them in its own table.  A batch
submitted on any rank goes through one exchange step:

  1. owner of every op: a multiply-shift range reduction of an independent 32-bit mixer (not
     the table's own hash1/hash2, so each shard's bucket choice stays uniform);
  2. ops grouped by owner (a stable sort), per-destination counts exchanged, then the packed
     records -- key u32, value u32, type u8: 9 bytes per op -- exchanged with all_to_all_single
     (NCCL over NVLink/NVSwitch on GPUs, gloo on CPU);
  3. each rank applies what it received to its shard (ops unordered within a batch, as locally);
  4. the results -- status u8, value u32: 5 bytes per op -- travel back with the reverse
     all_to_all_single and are put back in submission order.

All ranks must call apply() together, in the same order (the exchange is a collective).  The
reference is single-GPU; this is the sharding it has no counterpart for.
"""
from __future__ import annotations

import ctypes
from pathlib import Path
from typing import Callable, Optional, Tuple

import numpy as np
import torch
import torch.distributed as dist

_SHARD_LIB = Path(__file__).resolve().parent / "lib" / "libhive_shard.so"
_shard_lib = None


def shard_library() -> ctypes.CDLL:
    """libhive_shard.so: the exchange kernels (include/hive_shard.h).  Raises if not built."""
    global _shard_lib
    if _shard_lib is None:
        if not _SHARD_LIB.exists():
            raise ImportError(f"{_SHARD_LIB} is missing: build it with `python -m hivehashtable_b200.build`")
        lib = ctypes.CDLL(str(_SHARD_LIB))
        P, U64, U32 = ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint32
        lib.hive_shard_blocks.restype = U64
        lib.hive_shard_blocks.argtypes = [U64]
        for name, args in (("hive_shard_count", [P, U64, U32, P, P]),
                           ("hive_shard_scatter", [P, P, P, U64, U32, P, P, P, P, P, P]),
                           ("hive_shard_gather", [P, U64, P, P, P, P, P])):
            fn = getattr(lib, name)
            fn.restype = ctypes.c_int
            fn.argtypes = args
        _shard_lib = lib
    return _shard_lib


def owner_of(keys_i32: torch.Tensor, world: int) -> torch.Tensor:
    """Owner rank of each key: (mix(key) * world) >> 32, mix = the MurmurHash3 32-bit finaliser
    of key ^ 0x9E3779B9 (computed in int64 to stay exact in torch)."""
    k = keys_i32.to(torch.int64) & 0xFFFFFFFF
    h = k ^ 0x9E3779B9
    h = h ^ (h >> 16)
    h = (h * 0x85EBCA6B) & 0xFFFFFFFF
    h = h ^ (h >> 13)
    h = (h * 0xC2B2AE35) & 0xFFFFFFFF
    h = h ^ (h >> 16)
    return ((h * world) >> 32).to(torch.int64)


# A local shard applies (types u8, keys i32, vals i32) -> (status u8, values i32), all on one device.
LocalApply = Callable[[torch.Tensor, torch.Tensor, torch.Tensor], Tuple[torch.Tensor, torch.Tensor]]


class ShardedHiveTable:
    """`local` is this rank's shard: a HiveHashTable (its apply() is used) or any callable with
    the LocalApply signature.  `device` holds the exchange buffers (cuda for NCCL, cpu for gloo)."""

    def __init__(self, local, device: torch.device, group: Optional[dist.ProcessGroup] = None,
                 hints: int = 0):
        self.group = group
        self.world = dist.get_world_size(group)
        self.rank = dist.get_rank(group)
        self.device = device
        self.hints = hints
        self.local = None
        if callable(local) and not hasattr(local, "apply"):
            self._apply = local
        else:
            self.local = local
            self._apply = lambda t, k, v: local.apply(t, k, v, hints=self.hints)

    def _a2a(self, x: torch.Tensor, send_counts, recv_counts) -> torch.Tensor:
        out = torch.empty((int(sum(recv_counts)),) + tuple(x.shape[1:]), dtype=x.dtype, device=x.device)
        dist.all_to_all_single(out, x, list(recv_counts), list(send_counts), group=self.group)
        return out

    @staticmethod
    def _i32(x, dev) -> torch.Tensor:
        """uint32 bit patterns as an int32 tensor on dev."""
        t = torch.as_tensor(x)
        if t.dtype != torch.int32:
            t = t.to(torch.int64).to(torch.int32)
        return t.to(dev)

    @staticmethod
    def _bytes(x: torch.Tensor) -> torch.Tensor:
        """(n,) 4-byte tensor -> (n, 4) uint8 view of its bytes."""
        return x.contiguous().view(torch.uint8).view(-1, 4)

    def apply(self, types, keys, vals, local: Optional[LocalApply] = None) -> Tuple[torch.Tensor, torch.Tensor]:
        """One batch of mixed ops (types as in HiveHashTable.apply) through the exchange; returns
        (status u8, value i32) per op in submission order.  `local` replaces the shard's own
        apply for this batch (insert() and find() pass the shard's bulk calls)."""
        local = local or self._apply
        dev = self.device
        types = torch.as_tensor(types).to(dev).to(torch.uint8).contiguous()
        keys, vals = self._i32(keys, dev).contiguous(), self._i32(vals, dev).contiguous()
        if dev.type == "cuda":
            return self._apply_device(types, keys, vals, local)
        n = keys.numel()
        dest = owner_of(keys, self.world)
        order = torch.argsort(dest, stable=True)
        send = torch.bincount(dest, minlength=self.world).to(torch.int64)
        recv = torch.empty_like(send)
        dist.all_to_all_single(recv, send, group=self.group)
        send_l, recv_l = send.tolist(), recv.tolist()
        # one 9-byte record per op: key, value, type
        rec = torch.cat([self._bytes(keys[order]), self._bytes(vals[order]), types[order].view(-1, 1)], dim=1)
        got = self._a2a(rec.contiguous(), send_l, recv_l)
        gk = got[:, 0:4].contiguous().view(torch.int32).view(-1)
        gv = got[:, 4:8].contiguous().view(torch.int32).view(-1)
        gt = got[:, 8].contiguous()
        if got.shape[0]:
            st, ov = local(gt, gk, gv)
            st = st.to(dev).to(torch.uint8)
            ov = ov.to(dev).to(torch.int32)
        else:
            st = torch.empty(0, dtype=torch.uint8, device=dev)
            ov = torch.empty(0, dtype=torch.int32, device=dev)
        # one 5-byte result per op: status, value
        res = torch.cat([st.view(-1, 1), self._bytes(ov)], dim=1).contiguous()
        back = self._a2a(res, recv_l, send_l)
        status = torch.empty(n, dtype=torch.uint8, device=dev)
        outv = torch.empty(n, dtype=torch.int32, device=dev)
        status[order] = back[:, 0]
        outv[order] = back[:, 1:5].contiguous().view(torch.int32).view(-1)
        return status, outv

    def _apply_device(self, types, keys, vals, local) -> Tuple[torch.Tensor, torch.Tensor]:
        """apply() with the batch on the GPU: the owner split by the native count/scatter kernels
        (keys, values, types kept as separate arrays, so the exchange moves 9 bytes per op and the
        shard reads them without unpacking), the results put back by the native gather."""
        lib = shard_library()
        dev = self.device
        s = torch.cuda.current_stream(dev).cuda_stream
        n, w = keys.numel(), self.world
        nb = int(lib.hive_shard_blocks(n))
        counts = torch.zeros(w * max(nb, 1), dtype=torch.int32, device=dev)
        if n and lib.hive_shard_count(keys.data_ptr(), n, w, counts.data_ptr(), s):
            raise RuntimeError("hive_shard_count failed")
        c64 = counts.to(torch.int64)
        starts = torch.cumsum(c64, 0) - c64
        send = c64.view(w, -1).sum(1)
        recv = torch.empty_like(send)
        dist.all_to_all_single(recv, send, group=self.group)
        out_k = torch.empty(n, dtype=torch.int32, device=dev)
        out_v = torch.empty(n, dtype=torch.int32, device=dev)
        out_t = torch.empty(n, dtype=torch.uint8, device=dev)
        pos = torch.empty(n, dtype=torch.int64, device=dev)
        if n and lib.hive_shard_scatter(keys.data_ptr(), vals.data_ptr(), types.data_ptr(), n, w, starts.data_ptr(),
                                        out_k.data_ptr(), out_v.data_ptr(), out_t.data_ptr(), pos.data_ptr(), s):
            raise RuntimeError("hive_shard_scatter failed")
        send_l, recv_l = send.tolist(), recv.tolist()
        gk, gv, gt = self._a2a(out_k, send_l, recv_l), self._a2a(out_v, send_l, recv_l), self._a2a(out_t, send_l, recv_l)
        if gk.numel():
            st, ov = local(gt, gk, gv)
            st = st.to(dev).to(torch.uint8).contiguous()
            ov = ov.to(dev).to(torch.int32).contiguous()
        else:
            st = torch.empty(0, dtype=torch.uint8, device=dev)
            ov = torch.empty(0, dtype=torch.int32, device=dev)
        back_st, back_v = self._a2a(st, recv_l, send_l), self._a2a(ov, recv_l, send_l)
        status = torch.empty(n, dtype=torch.uint8, device=dev)
        outv = torch.empty(n, dtype=torch.int32, device=dev)
        if n and lib.hive_shard_gather(pos.data_ptr(), n, back_st.data_ptr(), back_v.data_ptr(), status.data_ptr(),
                                       outv.data_ptr(), s):
            raise RuntimeError("hive_shard_gather failed")
        return status, outv

    def insert(self, keys, vals):
        """Bulk upsert; statuses as HiveHashTable.insert.  A HiveHashTable shard applies what it
        receives with its bulk insert."""
        t = self.local
        bulk = None if t is None else (lambda _t, k, v: (t.insert(k, v), torch.zeros_like(k)))
        return self.apply(torch.zeros(len(keys), dtype=torch.uint8, device=self.device), keys, vals, bulk)[0]

    def find(self, keys):
        """Bulk lookup: (values, found).  A HiveHashTable shard answers with its bulk find."""
        t = self.local

        def bulk(_t, k, _v):
            v, f = t.find(k)
            return f, v

        # op types and the (unused) values are made where the exchange runs: built on the host they
        # would cross PCIe on every call
        n, d = len(keys), self.device
        st, ov = self.apply(torch.ones(n, dtype=torch.uint8, device=d), keys, torch.zeros(n, dtype=torch.int32, device=d),
                            None if t is None else bulk)
        return ov, st
