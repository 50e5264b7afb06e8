"""A/B against the reference's own GPU build for sm_100a (oracle/_ref/libhive_ref_gpu.so, built
from the reference's src/hive_dispatch.cu, src/hive_memory.cu and src/GPUTimer.cc): the same seeded
keys give the same per-op success flags, and both sides' kernel times are printed (REF_AB line)."""
import json
import subprocess
import sys
from pathlib import Path

import pytest

import oracle

pytestmark = pytest.mark.gpu
ROOT = Path(__file__).resolve().parents[1]


@pytest.mark.parametrize("cap_log,lf,present", [(22, 0.9, 0.5), (26, 0.9, 0.5)])
def test_reference_gpu_same_flags(cuda, cap_log, lf, present):
    if not (oracle.REF_DIR / "libhive_ref_gpu.so").exists():
        pytest.skip("reference GPU build not present (needs the reference tree at build time)")
    p = subprocess.run([sys.executable, "-m", "oracle.ref_gpu_ab", str(cap_log), str(lf), str(present)],
                       capture_output=True, text=True, timeout=900, cwd=str(ROOT))
    line = [ln for ln in p.stdout.splitlines() if ln.startswith("REF_AB ")]
    assert p.returncode == 0 and line, p.stdout[-3000:] + p.stderr[-3000:]
    r = json.loads(line[-1][7:])
    print(line[-1])
    n = r["n"]
    assert r["hive"]["inserted"] == n
    # the reference may leave a key unplaced when a bucket's 8-slot stash overflows; every key it
    # placed the B200 table placed too, and lookups agree op by op where both hold every key
    assert r["reference"]["inserted"] <= r["hive"]["inserted"]
    if r["reference"]["inserted"] == n:
        assert r["insert_flags_equal"] and r["lookup_flags_equal"]
        assert r["reference"]["found_present"] == n
