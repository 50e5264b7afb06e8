"""The sharded table with real B200 shards: each rank holds a HiveHashTable on cuda:0.

* world size 1 over NCCL: the exchange runs through NCCL's all_to_all on the GPU (with itself);
* world size 2 over gloo, two processes on the one GPU: each rank's shard is its own table (the
  tables are independent; no kernel waits on another rank's), the exchange moves CPU tensors.

Every op's result equals one global std::unordered_map replay of the batches in order (keys are
unique within a batch, so each result is fixed), and every key lives on its owner rank only.
"""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

pytestmark = pytest.mark.gpu


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _batches(seed, n_batches, size):
    """Mixed batches with unique keys per batch: inserts of new keys, upserts, lookups (present and
    absent), deletes and increments of live keys."""
    import oracle

    pre, pool, _ = oracle.gen_keys(seed, 4 * size, n_batches * size * 2)
    rs = np.random.RandomState(seed)
    live = sorted(set(pre.tolist()))
    out, pi = [], 0
    for _ in range(n_batches):
        new = pool[pi: pi + size // 2]
        pi += size // 2
        la = np.array(live, dtype=np.uint32)
        sel = la[rs.choice(la.size, size=size // 2, replace=False)]
        absent = pool[pi: pi + size // 8]
        pi += size // 8
        keys = np.concatenate([new, sel, absent]).astype(np.uint32)
        types = np.concatenate([np.zeros(new.size), rs.randint(0, 4, size=sel.size), np.ones(absent.size)])
        types = types.astype(np.uint8)
        vals = rs.randint(1, 2**32 - 1, size=keys.size).astype(np.uint32)
        perm = rs.permutation(keys.size)
        keys, types, vals = keys[perm], types[perm], vals[perm]
        out.append((types, keys, vals))
        gone = set(keys[types == 2].tolist())
        live = sorted((set(live) - gone) | set(keys[types == 0].tolist()))  # each key once
    return pre, out


def _run_and_check(tbl, shard, rank, world, seed):
    import oracle
    from hivehashtable_b200.sharded import owner_of

    pre, batches = _batches(seed, 6, 4000)
    m = oracle.ReplayMap()
    # rank r submits its slice of every batch (op i when i % world == r), so together the ranks
    # submit each batch once; every rank replays the whole batch and checks its own slice
    pre_v = oracle.values_for(pre)
    mine = np.arange(pre.size) % world == rank
    st = tbl.insert(torch.from_numpy(pre[mine].view(np.int32)), torch.from_numpy(pre_v[mine].view(np.int32)))
    m.insert(pre, pre_v)
    assert (st.cpu().numpy() == 1).all()
    for b, (types, keys, vals) in enumerate(batches):
        part = np.arange(keys.size) % world == rank
        st, ov = tbl.apply(torch.from_numpy(types[part]), torch.from_numpy(keys[part].view(np.int32)),
                           torch.from_numpy(vals[part].view(np.int32)))
        est, eov = m.apply(types, keys, vals)
        np.testing.assert_array_equal(np.where(st.cpu().numpy() == 3, 1, st.cpu().numpy()), est[part],
                                      err_msg=f"rank {rank} batch {b}")
        np.testing.assert_array_equal(ov.cpu().numpy().view(np.uint32), eov[part], err_msg=f"rank {rank} batch {b}")
    gk, gv = shard.dump()
    own = owner_of(torch.from_numpy(gk.view(np.int32)), world).numpy()
    assert (own == rank).all()
    rk, rv = m.dump()
    mine = owner_of(torch.from_numpy(rk.view(np.int32)), world).numpy() == rank
    np.testing.assert_array_equal(gk, rk[mine])
    np.testing.assert_array_equal(gv, rv[mine])
    v = shard.verify()
    assert v["tag_mismatch"] == v["misplaced"] == v["duplicate"] == 0, v
    shard.check()
    return int(gk.size)


def test_sharded_nccl_world_size_one(cuda):
    from datetime import timedelta

    from hivehashtable_b200 import HiveHashTable
    from hivehashtable_b200.sharded import ShardedHiveTable

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(_free_port())
    torch.cuda.set_device(0)
    dist.init_process_group("nccl", rank=0, world_size=1, timeout=timedelta(seconds=120),
                            device_id=torch.device("cuda", 0))
    try:
        with HiveHashTable(1 << 16) as shard:
            tbl = ShardedHiveTable(shard, torch.device("cuda", 0))
            assert _run_and_check(tbl, shard, 0, 1, 41) > 0
            torch.cuda.synchronize()
    finally:
        dist.destroy_process_group()


def _gloo_worker(rank, world, port, q):
    from hivehashtable_b200 import HiveHashTable
    from hivehashtable_b200.sharded import ShardedHiveTable

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    torch.cuda.set_device(0)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        with HiveHashTable(1 << 15) as shard:
            tbl = ShardedHiveTable(shard, torch.device("cpu"))
            q.put((rank, _run_and_check(tbl, shard, rank, world, 43)))
    finally:
        dist.destroy_process_group()


def test_sharded_two_ranks_gloo_real_shards(cuda):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_gloo_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=300)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    sizes = dict(q.get() for _ in range(2))
    assert min(sizes.values()) > 0


@pytest.mark.parametrize("world,n", [(3, 100_003), (8, 1 << 20), (1, 5000)])
def test_exchange_kernels_split_by_owner(cuda, world, n):
    """hive_shard_count / scatter / gather: every op lands in its owner's range (owner as
    sharded.owner_of computes it), pos is a permutation, and gather inverts scatter."""
    import oracle
    from hivehashtable_b200.sharded import owner_of, shard_library

    lib = shard_library()
    keys, _, _ = oracle.gen_keys(51, n, 0)
    kd = torch.from_numpy(keys.view(np.int32)).to(cuda)
    vd = torch.arange(n, dtype=torch.int32, device=cuda)
    td = (torch.arange(n, device=cuda) % 4).to(torch.uint8)
    s = torch.cuda.current_stream(cuda).cuda_stream
    nb = int(lib.hive_shard_blocks(n))
    counts = torch.zeros(world * nb, dtype=torch.int32, device=cuda)
    assert lib.hive_shard_count(kd.data_ptr(), n, world, counts.data_ptr(), s) == 0
    c64 = counts.to(torch.int64)
    starts = torch.cumsum(c64, 0) - c64
    ok, ov, ot = (torch.empty(n, dtype=d, device=cuda) for d in (torch.int32, torch.int32, torch.uint8))
    pos = torch.empty(n, dtype=torch.int64, device=cuda)
    assert lib.hive_shard_scatter(kd.data_ptr(), vd.data_ptr(), td.data_ptr(), n, world, starts.data_ptr(),
                                  ok.data_ptr(), ov.data_ptr(), ot.data_ptr(), pos.data_ptr(), s) == 0
    own = owner_of(kd, world)
    per_rank = torch.bincount(own, minlength=world)
    assert torch.equal(c64.view(world, -1).sum(1), per_rank)
    p = pos.cpu().numpy()
    assert np.array_equal(np.sort(p), np.arange(n))
    bounds = np.concatenate([[0], np.cumsum(per_rank.cpu().numpy())])
    rank_of_place = np.searchsorted(bounds, p, side="right") - 1
    assert np.array_equal(rank_of_place, own.cpu().numpy())
    assert torch.equal(ok[pos], kd) and torch.equal(ov[pos], vd) and torch.equal(ot[pos], td)
    st = torch.empty(n, dtype=torch.uint8, device=cuda)
    back = torch.empty(n, dtype=torch.int32, device=cuda)
    assert lib.hive_shard_gather(pos.data_ptr(), n, ot.data_ptr(), ov.data_ptr(), st.data_ptr(), back.data_ptr(), s) == 0
    assert torch.equal(st, td) and torch.equal(back, vd)
