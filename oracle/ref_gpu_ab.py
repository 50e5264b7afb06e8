"""TEST INFRASTRUCTURE: A/B of the reference's own GPU build against the B200 table.

Runs the reference's GPU path (oracle/_ref/libhive_ref_gpu.so: its src/hive_dispatch.cu,
src/hive_memory.cu and src/GPUTimer.cc compiled unchanged for sm_100a by oracle/build.py) and the
B200 table on the same seeded keys (splitmix64 seed 7, value = key + 1 as the reference's kernels
set it, include/hive_kernels.cuh:238) and prints one JSON line, prefixed "REF_AB ", with per-op
success-flag agreement and both sides' kernel times.  Used by tests/test_gpu_reference_ab.py and by
bench.py's reference arm.  Run it in a process of its own: the reference reserves ~60 % of free HBM
when it loads and ends the process on any CUDA error.

usage: python -m oracle.ref_gpu_ab CAP_LOG LOAD_FACTOR PRESENT_FRACTION
"""
import ctypes
import json
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))
LIB = Path(__file__).resolve().parent / "_ref" / "libhive_ref_gpu.so"


def available() -> bool:
    return LIB.exists()


def main():
    cap_log, lf, present = int(sys.argv[1]), float(sys.argv[2]), float(sys.argv[3])
    cap = 1 << cap_log
    n = int(lf * cap)
    from hivehashtable_b200 import workload

    keys, vals, look = workload.bulk_workload(7, n, present)
    refvals = keys + np.uint32(1)  # the reference's value = key + 1

    import torch
    from hivehashtable_b200 import HiveHashTable, as_device_u32

    dev = torch.device("cuda", 0)
    out = {"cap_log": cap_log, "n": n, "present": present}

    # -- B200 table: same keys, value = key + 1, kernel time by CUDA events (best of 3) --
    kd, vd, ld = as_device_u32(keys, dev), as_device_u32(refvals, dev), as_device_u32(look, dev)
    with HiveHashTable(cap) as t:
        ins, fnd = [], []
        for _ in range(3):
            t.clear()
            a, b, c = (torch.cuda.Event(enable_timing=True) for _ in range(3))
            a.record()
            st = t.insert(kd, vd)
            b.record()
            v, f = t.find(ld)
            c.record()
            torch.cuda.synchronize()
            ins.append(a.elapsed_time(b))
            fnd.append(b.elapsed_time(c))
        hive_ins_ok = (st.cpu().numpy() != 0)
        hive_found = f.cpu().numpy().astype(bool)
        out["hive"] = {"insert_ms": min(ins), "lookup_ms": min(fnd),
                       "insert_mops": n / min(ins) / 1e3, "lookup_mops": look.size / min(fnd) / 1e3,
                       "inserted": int(hive_ins_ok.sum()), "found": int(hive_found.sum())}
    del kd, vd, ld
    torch.cuda.empty_cache()

    # -- the reference's own GPU build --
    lib = ctypes.CDLL(str(LIB))
    P, S, I, D = ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int, ctypes.POINTER(ctypes.c_double)
    lib.ref_bulk_insert.argtypes = [P, S, S, I, I, D, P]
    lib.ref_lookup.argtypes = [P, S, P, S, S, I, D, P]
    lib.ref_lookup_present.argtypes = [P, S, S, I, I, D, P]
    ms = ctypes.c_double()
    r_ins = np.zeros(n, dtype=np.uint64)
    lib.ref_bulk_insert(keys.ctypes.data, n, cap, 0, 1, ctypes.byref(ms), r_ins.ctypes.data)
    ref_ins_ms = ms.value
    r_look = np.zeros(look.size, dtype=np.uint64)
    lib.ref_lookup(keys.ctypes.data, n, look.ctypes.data, look.size, cap, 1, ctypes.byref(ms), r_look.ctypes.data)
    ref_look_ms = ms.value
    r_pres = np.zeros(n, dtype=np.uint64)
    lib.ref_lookup_present(keys.ctypes.data, n, cap, 0, 1, ctypes.byref(ms), r_pres.ctypes.data)
    ref_pres_ms = ms.value
    out["reference"] = {"insert_ms": ref_ins_ms, "lookup_ms": ref_look_ms, "lookup_present_ms": ref_pres_ms,
                        "insert_mops": n / ref_ins_ms / 1e3, "lookup_mops": look.size / ref_look_ms / 1e3,
                        "lookup_present_mops": n / ref_pres_ms / 1e3,
                        "inserted": int((r_ins != 0).sum()), "found": int((r_look != 0).sum()),
                        "found_present": int((r_pres != 0).sum())}
    out["insert_flags_equal"] = bool(np.array_equal(r_ins != 0, hive_ins_ok))
    out["lookup_flags_equal"] = bool(np.array_equal(r_look != 0, hive_found))
    out["speedup_insert"] = ref_ins_ms / out["hive"]["insert_ms"]
    out["speedup_lookup"] = ref_look_ms / out["hive"]["lookup_ms"]
    print("REF_AB " + json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
