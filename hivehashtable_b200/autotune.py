"""Autotuner: per GPU, capacity and load factor, the launch knobs (hive_set_tuning) and the
eviction bound that run a bulk insert + lookup fastest on that device.

The reference fixes its launch shape and eviction bound at compile time (THREADS_PER_BLOCK and
MAX_EVICT in src/hive_dispatch.cu and include/hive_hash_table.cuh:21).  Here they are run-time
settings of a table, so the tuner measures them on the device instead:

  knob                 values tried                 what it changes
  tags                 0, 1 (auto), 2               per-slot fingerprints: never / while they fit L2 / always
  region_insert        0, 2                         submission order vs one region-ordered pass
  second_pass_blocks   2, 4, 8                      resident blocks per SM of the deferred pass
  max_evictions        4, 8                         cuckoo victims tried per insert (a table setting)
  stash_depth          8, 4                         canonical-stash slots an insert may use
  l2_window            0, 1                         L2 persistence window over tables that fit it

The bucket width is not tuned: a bucket is one 64 B line, two 32 B sectors that a lane pair reads
with one request, and its per-slot fingerprints are one 8-byte word; every kernel is built on that
layout.  One thread runs one op (a lane pair shares each bucket read), so there is no warps-per-op
setting either.

A tuned setting is applied to new tables: HiveHashTable(..., tuning="cache") or the
HIVE_TUNE_CACHE environment variable (the JSON file autotune() writes) picks the entry of the same
GPU and policy whose capacity is nearest (lookup_cached).

Search: coordinate descent from the defaults, one knob at a time, two rounds at most.  A setting
is accepted only if it places every key the defaults place (no new failed inserts) and every lookup
result matches; the objective is the mean device time of clear + insert + lookup after warm-up.
"""
from __future__ import annotations

import argparse
import json
from pathlib import Path
from typing import Callable, Dict, Optional

DEFAULTS = {"tags": 1, "region_insert": 0, "second_pass_blocks": 8, "max_evictions": 8, "stash_depth": 8,
            "l2_window": 0, "binned": 1}
SPACE = {"tags": [1, 0, 2], "region_insert": [0, 2], "second_pass_blocks": [8, 4, 2], "max_evictions": [8, 4],
         "stash_depth": [8, 4], "l2_window": [0, 1], "binned": [1, 0]}

# measure(setting) -> {"ms": float, "failed": int, "correct": bool}
Measure = Callable[[Dict[str, int]], Dict[str, float]]


def search(measure: Measure, space: Optional[Dict[str, list]] = None, start: Optional[Dict[str, int]] = None,
           rounds: int = 2) -> dict:
    """Coordinate descent over `space` from `start`; returns the best setting and every trial."""
    space = space or SPACE
    best = dict(start or DEFAULTS)
    trials = {}

    def run(setting):
        key = json.dumps(setting, sort_keys=True)
        if key not in trials:
            trials[key] = dict(measure(dict(setting)), setting=dict(setting))
        return trials[key]

    base = run(best)
    best_r = base
    for _ in range(rounds):
        changed = False
        for knob, values in space.items():
            for v in values:
                if v == best[knob]:
                    continue
                cand = dict(best, **{knob: v})
                r = run(cand)
                ok = r["correct"] and r["failed"] <= base["failed"]
                if ok and r["ms"] < best_r["ms"]:
                    best, best_r, changed = cand, r, True
        if not changed:
            break
    return {"best": best, "best_ms": best_r["ms"], "default_ms": base["ms"], "trials": list(trials.values())}


def device_measure(capacity: int, load_factor: float, present: float = 0.5, policy: str = "Default2Hash",
                   seed: int = 7, reps: int = 3, warmup: int = 2) -> Measure:
    """A Measure over one synthetic workload resident on the current GPU."""
    import numpy as np
    import torch

    from . import workload
    from .table import HiveHashTable, as_device_u32

    dev = torch.device("cuda", torch.cuda.current_device())
    n = int(load_factor * capacity)
    kh, vh, lh = workload.bulk_workload(seed, n, present)
    keys, vals, look = as_device_u32(kh, dev), as_device_u32(vh, dev), as_device_u32(lh, dev)
    exp_found = int(round(lh.size * present))
    status = torch.empty(n, dtype=torch.uint8, device=dev)
    fv = torch.empty(lh.size, dtype=torch.int32, device=dev)
    fd = torch.empty(lh.size, dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream(dev)

    def measure(setting):
        knobs = {k: v for k, v in setting.items() if k != "max_evictions"}
        with HiveHashTable(capacity, policy, max_evictions=setting.get("max_evictions", 8), tuning={}) as t:
            t.set_tuning(**knobs)
            times = []
            for it in range(warmup + reps):
                a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                a.record(stream)
                t.clear()
                t.insert(keys, vals, status)
                t.find(look, fv, fd)
                b.record(stream)
                torch.cuda.synchronize()
                if it >= warmup:
                    times.append(a.elapsed_time(b))
            failed = int((status == 0).sum())
            found = int(fd.sum())
            # every placed key must be found with its value; absent keys must miss
            correct = found == exp_found if failed == 0 else found <= exp_found
            if correct and failed == 0:
                v, f = t.find(keys[: 1 << 16])
                correct = bool((f == 1).all()) and bool((v == vals[: 1 << 16]).all())
            t.check()
        return {"ms": float(np.mean(times)), "failed": failed, "correct": bool(correct)}

    return measure


def cache_key(gpu: str, capacity: int, load_factor: float, present: float, policy: str) -> str:
    return f"{gpu}|cap={capacity}|lf={load_factor:.3f}|present={present:.2f}|{policy}"


def autotune(capacity: int, load_factor: float, present: float = 0.5, policy: str = "Default2Hash",
             cache: Optional[Path] = None, **kw) -> dict:
    """Tune on the current GPU (cached in `cache`, a JSON file, when given)."""
    import torch

    gpu = torch.cuda.get_device_name()
    key = cache_key(gpu, capacity, load_factor, present, policy)
    if cache and Path(cache).exists():
        stored = json.loads(Path(cache).read_text())
        if key in stored:
            return stored[key]
    result = search(device_measure(capacity, load_factor, present, policy, **kw))
    result.update({"gpu": gpu, "capacity_slots": capacity, "load_factor": load_factor, "present": present,
                   "policy": policy})
    if cache:
        stored = json.loads(Path(cache).read_text()) if Path(cache).exists() else {}
        stored[key] = result
        Path(cache).write_text(json.dumps(stored, indent=1))
    return result


def lookup_cached(cache: Path, gpu: str, capacity: int, policy: str) -> Optional[Dict[str, int]]:
    """The best setting stored in `cache` for this GPU and policy at the capacity nearest to
    `capacity` (in log2), or None."""
    import math

    if not cache or not Path(cache).exists():
        return None
    stored = json.loads(Path(cache).read_text())
    cands = [r for r in stored.values() if r.get("gpu") == gpu and r.get("policy") == policy and "best" in r]
    if not cands:
        return None
    r = min(cands, key=lambda e: abs(math.log2(e["capacity_slots"]) - math.log2(max(capacity, 1))))
    return dict(r["best"])


def apply(table, setting: Dict[str, int]) -> None:
    """Apply a tuned setting's knobs to a table (max_evictions is given at creation)."""
    table.set_tuning(**{k: v for k, v in setting.items() if k != "max_evictions"})


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--cap-log", type=int, default=26)
    ap.add_argument("--lf", type=float, default=0.9)
    ap.add_argument("--present", type=float, default=0.5)
    ap.add_argument("--policy", default="Default2Hash")
    ap.add_argument("--cache", type=Path, default=None)
    ap.add_argument("--reps", type=int, default=3)
    a = ap.parse_args()
    r = autotune(1 << a.cap_log, a.lf, a.present, a.policy, cache=a.cache, reps=a.reps)
    print(json.dumps({k: v for k, v in r.items() if k != "trials"}))
    for t in r["trials"]:
        print(json.dumps(t))


if __name__ == "__main__":
    main()
