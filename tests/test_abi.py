"""The C ABI libraries load and export every symbol include/hive_c.h and include/hive_shard.h declare
(no GPU needed)."""
import ctypes
import re
import subprocess
from pathlib import Path

import pytest
import torch

from hivehashtable_b200 import build, table

ROOT = Path(__file__).resolve().parents[1]


def _declared(header: Path):
    text = header.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(hive_[a-z_]+)\s*\(", text)))


def _exported(lib: Path):
    out = subprocess.run(["nm", "-D", "--defined-only", str(lib)], capture_output=True, text=True, check=True).stdout
    return {ln.split()[-1] for ln in out.splitlines() if " T " in ln}


def test_core_exports_every_declared_symbol():
    decl = _declared(ROOT / "include" / "hive_c.h")
    assert "hive_insert" in decl and "hive_find" in decl and len(decl) >= 17
    exp = _exported(build.LIB / "libhive_b200.so")
    missing = [d for d in decl if d not in exp]
    assert not missing, missing
    # the Python mirror binds exactly the declared surface
    assert sorted(n for n, _, _ in table.ABI) == decl


def test_core_exports_nothing_else():
    exp = _exported(build.LIB / "libhive_b200.so")
    extra = [e for e in exp if not e.startswith("hive_")]
    assert not extra, extra


def test_strerror_and_argument_checks_without_device():
    lib = table.library()
    for code in range(0, 8):
        assert lib.hive_strerror(code)
    assert lib.hive_strerror(99) == b"unknown status"
    assert lib.hive_create(None, None) == 1
    h = ctypes.c_void_p()
    bad = table._Config(0, 0, 0, 8, -1, 0)
    assert lib.hive_create(ctypes.byref(bad), ctypes.byref(h)) == 1  # capacity 0
    bad = table._Config(64, 0, 5, 8, -1, 0)
    assert lib.hive_create(ctypes.byref(bad), ctypes.byref(h)) == 1  # unknown policy
    bad = table._Config(64, 0, 0, 9, -1, 0)
    assert lib.hive_create(ctypes.byref(bad), ctypes.byref(h)) == 1  # max_evictions > 8
    assert lib.hive_insert(None, None, None, 0, None, None) == 1
    assert lib.hive_destroy(None) == 1


@pytest.mark.skipif(torch.cuda.is_available(), reason="checks the no-device error path")
def test_create_reports_missing_device():
    lib = table.library()
    h = ctypes.c_void_p()
    cfg = table._Config(1024, 0, 0, 8, -1, 0)
    assert lib.hive_create(ctypes.byref(cfg), ctypes.byref(h)) == 7
    with pytest.raises(table.HiveError):
        table.HiveHashTable(1024)


def test_shard_library_exports_its_header():
    decl = _declared(ROOT / "include" / "hive_shard.h")
    assert decl == ["hive_shard_blocks", "hive_shard_count", "hive_shard_gather", "hive_shard_scatter"]
    exp = _exported(build.build_shard())
    assert sorted(e for e in exp if e.startswith("hive_")) == decl
    assert not [e for e in exp if not e.startswith("hive_")]
    from hivehashtable_b200.sharded import shard_library

    lib = shard_library()
    assert lib.hive_shard_blocks(0) == 0 and lib.hive_shard_blocks(4096) == 1 and lib.hive_shard_blocks(4097) == 2
    # argument checks run before any launch, so they need no device
    assert lib.hive_shard_count(None, 10, 2, None, None) == 1
    assert lib.hive_shard_scatter(None, None, None, 10, 2, None, None, None, None, None, None) == 1
    assert lib.hive_shard_gather(None, 10, None, None, None, None, None) == 1
