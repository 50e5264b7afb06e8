"""Hash-partitioned Hive table over several GPUs (one process per GPU, torch.distributed).

Each rank owns the keys whose owner(key) is its rank and keeps them in its own table.  A batch
submitted on any rank goes through one exchange step:

  1. owner of every op: a multiply-shift range reduction of an independent 32-bit mixer (not
     the table's own hash1/hash2, so each shard's bucket choice stays uniform);
  2. ops grouped by owner (a stable sort), per-destination counts exchanged, then the
     (type, key, value) records exchanged with all_to_all_single (NCCL over NVLink/NVSwitch on
     GPUs, gloo on CPU);
  3. each rank applies what it received to its shard (ops unordered within a batch, as locally);
  4. the (status, value) results travel back with the reverse all_to_all_single and are put
     back in submission order.

All ranks must call apply() together, in the same order (the exchange is a collective).  The
reference is single-GPU; this is the sharding it has no counterpart for.
"""
from __future__ import annotations

from typing import Callable, Optional, Tuple

import numpy as np
import torch
import torch.distributed as dist


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
        if callable(local) and not hasattr(local, "apply"):
            self._apply = local
        else:
            self._apply = lambda t, k, v: local.apply(t, k, v, hints=self.hints)

    def _a2a(self, x: torch.Tensor, send_counts, recv_counts) -> torch.Tensor:
        out = torch.empty((int(sum(recv_counts)),) + tuple(x.shape[1:]), dtype=x.dtype, device=x.device)
        dist.all_to_all_single(out, x, list(recv_counts), list(send_counts), group=self.group)
        return out

    def apply(self, types, keys, vals) -> Tuple[torch.Tensor, torch.Tensor]:
        dev = self.device
        types = torch.as_tensor(types).to(dev).to(torch.int64)
        keys = torch.as_tensor(keys).to(dev).to(torch.int64)
        vals = torch.as_tensor(vals).to(dev).to(torch.int64)
        n = keys.numel()
        dest = owner_of(keys, self.world)
        order = torch.argsort(dest, stable=True)
        send = torch.bincount(dest, minlength=self.world).to(torch.int64)
        recv = torch.empty_like(send)
        dist.all_to_all_single(recv, send, group=self.group)
        send_l, recv_l = send.tolist(), recv.tolist()
        # one record per op: [type, key, value]
        rec = torch.stack([types[order], keys[order] & 0xFFFFFFFF, vals[order] & 0xFFFFFFFF], dim=1).contiguous()
        got = self._a2a(rec, send_l, recv_l)
        gt = got[:, 0].to(torch.uint8)
        gk = got[:, 1].to(torch.int32)
        gv = got[:, 2].to(torch.int32)
        if got.shape[0]:
            st, ov = self._apply(gt, gk, gv)
            res = torch.stack([st.to(torch.int64), ov.to(torch.int64) & 0xFFFFFFFF], dim=1).contiguous()
        else:
            res = torch.empty((0, 2), dtype=torch.int64, device=dev)
        back = self._a2a(res, recv_l, send_l)
        status = torch.empty(n, dtype=torch.uint8, device=dev)
        outv = torch.empty(n, dtype=torch.int64, device=dev)
        status[order] = back[:, 0].to(torch.uint8)
        outv[order] = back[:, 1]
        return status, outv.to(torch.int32)

    def insert(self, keys, vals):
        return self.apply(torch.zeros(len(keys), dtype=torch.uint8), keys, vals)[0]

    def find(self, keys):
        st, ov = self.apply(torch.ones(len(keys), dtype=torch.uint8), keys, torch.zeros(len(keys), dtype=torch.int32))
        return ov, st
