"""Batched mixed ops: the persistent one-launch path and the plain per-batch path both match the
unordered_map replay op by op, with growth planned between segments."""
import numpy as np
import pytest

import oracle
from hivehashtable_b200 import HiveHashTable, u32
from hivehashtable_b200.batched import BatchedRunner
from hivehashtable_b200.workload import MixedWorkload

pytestmark = pytest.mark.gpu


def _replay_and_check(run, wl, runner, table):
    m = oracle.ReplayMap()
    m.insert(wl.prefill_keys, wl.prefill_vals)
    st_all = runner.status.cpu().numpy()
    ov_all = u32(runner.outv)
    assert not (st_all == 255).any()
    for b in range(wl.n_batches):
        lo, hi = int(wl.offsets[b]), int(wl.offsets[b + 1])
        types, keys, vals = wl.types[lo:hi], wl.keys[lo:hi], wl.vals[lo:hi]
        st, ov = st_all[lo:hi], ov_all[lo:hi]
        placed = (types != 0) | (st != 0)
        est, eov = m.apply(types, keys, vals, apply_mask=placed.astype(np.uint8))
        got = np.where((types == 0) & (st == 3), 1, st)
        np.testing.assert_array_equal(got, est, err_msg=f"{run} batch {b}")
        np.testing.assert_array_equal(ov, eov, err_msg=f"{run} batch {b}")
        assert placed.all(), f"{run} batch {b}: insert not placed"
    gk, gv = table.dump()
    ok, ov = m.dump()
    np.testing.assert_array_equal(gk, ok)
    np.testing.assert_array_equal(gv, ov)
    assert len(m) == wl.final_live
    v = table.verify()
    assert v["tag_mismatch"] == v["misplaced"] == v["duplicate"] == 0, v


@pytest.mark.parametrize("policy", ["Default2Hash", "MurmurCityHash"])
@pytest.mark.parametrize("mode", ["plain", "persistent"])
def test_mixed_batches_match_replay(cuda, policy, mode):
    wl = MixedWorkload(11, 1 << 14, 48, 8.0, 12.0)
    with HiveHashTable(1 << 15, policy) as t:
        r = BatchedRunner(t, wl, max_load=0.85)
        r.prefill()
        res = r.run_plain() if mode == "plain" else r.run_persistent(blocks_per_sm=2)
        assert res.resizes >= 1  # the sequence outgrows 2^15 slots
        _replay_and_check(mode, wl, r, t)
        t.check()


def test_persistent_segments_and_block_shapes(cuda):
    wl = MixedWorkload(5, 1 << 13, 40, 6.0, 11.0)
    for tpb, bps, seg in ((128, 1, 7), (256, 0, 1 << 30), (512, 1, 3)):
        with HiveHashTable(1 << 16) as t:
            r = BatchedRunner(t, wl, max_load=0.85)
            r.prefill()
            res = r.run_persistent(threads_per_block=tpb, blocks_per_sm=bps, max_segment=seg)
            assert len(res.segments) >= (wl.n_batches + seg - 1) // seg if seg < 100 else True
            _replay_and_check("persistent", wl, r, t)
