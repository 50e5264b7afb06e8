"""The sharded table's exchange logic with world_size 2 and 3 on CPU (gloo): each rank's shard is
an oracle replay map standing in for its GPU table; results of every op on every rank must equal
one global replay, and every key must live on exactly its owner rank."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import oracle
    from hivehashtable_b200.sharded import ShardedHiveTable, owner_of

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        shard = oracle.ReplayMap()

        def local(t, k, v):
            st, ov = shard.apply(t.numpy().astype(np.uint8), k.numpy().view(np.uint32), v.numpy().view(np.uint32))
            return torch.from_numpy(st), torch.from_numpy(ov.view(np.int32))

        tbl = ShardedHiveTable(local, torch.device("cpu"))
        # rank r submits its own keys (some overlapping other ranks' keys), then mixed ops
        keys, absent, _ = oracle.gen_keys(100 + rank, 3000, 500)
        shared, _, _ = oracle.gen_keys(7, 200, 0)  # every rank upserts these: concurrent writers
        ins_k = np.concatenate([keys, shared]).astype(np.uint32)
        ins_v = oracle.values_for(ins_k) ^ np.uint32(rank)
        st = tbl.insert(torch.from_numpy(ins_k.view(np.int32)), torch.from_numpy(ins_v.view(np.int32)))
        # all own keys are new; the shared ones are new on exactly one rank's op or updates
        assert (st.numpy()[:3000] == 1).all()
        dist.barrier()
        # lookups of own keys, absent keys and the other ranks' first keys
        others = [oracle.gen_keys(100 + r, 3000, 0)[0][:50] for r in range(world)]
        look = np.concatenate([keys[:1000], absent, *others]).astype(np.uint32)
        v, f = tbl.find(torch.from_numpy(look.view(np.int32)))
        f, v = f.numpy(), v.numpy().view(np.uint32)
        assert f[:1000].all() and not f[1000:1500].any() and f[1500:].all()
        np.testing.assert_array_equal(v[:1000], oracle.values_for(keys[:1000]) ^ np.uint32(rank))
        for r in range(world):
            got = v[1500 + 50 * r: 1550 + 50 * r]
            np.testing.assert_array_equal(got, oracle.values_for(others[r]) ^ np.uint32(r))
        # every key on this shard is owned by this rank
        k_here, _ = shard.dump()
        own = owner_of(torch.from_numpy(k_here.view(np.int32)), world).numpy()
        assert (own == rank).all()
        q.put((rank, len(shard)))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_sharded_exchange_gloo(world):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=180)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    sizes = dict(q.get() for _ in range(world))
    # 3000 own keys per rank + the 200 shared keys, each stored once
    assert sum(sizes.values()) == 3000 * world + 200


def test_owner_is_balanced():
    from hivehashtable_b200.sharded import owner_of

    keys = torch.arange(1, 1 << 18, dtype=torch.int64).to(torch.int32)
    for world in (2, 3, 8):
        c = torch.bincount(owner_of(keys, world), minlength=world).double()
        assert (c.max() / c.mean()) < 1.02
