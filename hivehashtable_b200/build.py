"""Build recipe for the native libraries of hivehashtable_b200 (in-tree, sm_100a only).

Outputs (git-ignored, shipped with the source tree):
  hivehashtable_b200/lib/libhive_b200.so     kernels + the C ABI of include/hive_c.h
  hivehashtable_b200/lib/libhive_compat.so   the reference's C++ API on top of the C ABI
  hivehashtable_b200/lib/libhive_workload.so seeded workload generator (host C++)
  hivehashtable_b200/lib/libhive_serve.so    the served request loop (host C++)
  hivehashtable_b200/lib/libhive_shard.so    the sharded table's exchange kernels
and, for bench.py only (build_probe), lib/libhive_probe.so: the random-access ceiling probes.

Run as ``python -m hivehashtable_b200.build`` or through ``__graft_entry__.build()``.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
LIB = PKG / "lib"
INCLUDE = ROOT / "include"

ARCH_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build hivehashtable_b200")


def _stale(out: Path, deps: list[Path]) -> bool:
    if not out.exists():
        return True
    t = out.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def _run(cmd: list[str]) -> None:
    proc = subprocess.run(cmd, capture_output=True, text=True)
    if proc.returncode != 0:
        sys.stderr.write(proc.stdout + proc.stderr)
        raise RuntimeError("build step failed: " + " ".join(cmd))


def build_core(force: bool = False, verbose_ptxas: bool = False) -> Path:
    out = LIB / "libhive_b200.so"
    deps = [CSRC / "hive_table.cu", CSRC / "hive_device.cuh", INCLUDE / "hive_c.h"]
    if force or _stale(out, deps):
        LIB.mkdir(exist_ok=True)
        cmd = [_nvcc(), *ARCH_FLAGS, "-O3", "-lineinfo", "-std=c++17", "-shared", "-Xcompiler", "-fPIC",
               "-Xcompiler", "-fvisibility=hidden", "-DHIVE_BUILD", f"-I{INCLUDE}", f"-I{CSRC}",
               str(CSRC / "hive_table.cu"), "-o", str(out), "-lcudart"]
        if verbose_ptxas:
            cmd.insert(1, "-Xptxas=-v")
        _run(cmd)
    return out


def build_workload(force: bool = False) -> Path:
    out = LIB / "libhive_workload.so"
    src = CSRC / "hive_workload.cpp"
    if force or _stale(out, [src]):
        LIB.mkdir(exist_ok=True)
        _run(["g++", "-O3", "-std=c++17", "-shared", "-fPIC", "-pthread", str(src), "-o", str(out)])
    return out


def build_compat(force: bool = False) -> Path:
    out = LIB / "libhive_compat.so"
    src = CSRC / "hive_compat.cpp"
    hdrs = [INCLUDE / "hive_hash_table.cuh", INCLUDE / "hive_c.h"]
    core = build_core(force=False)
    if force or _stale(out, [src, core, *hdrs]):
        LIB.mkdir(exist_ok=True)
        _run([_nvcc(), "-O3", "-std=c++17", "-shared", "-Xcompiler", "-fPIC", f"-I{INCLUDE}", f"-I{CSRC / 'compat_types'}",
              str(src), "-o", str(out), f"-L{LIB}", "-lhive_b200", "-Xlinker", "-rpath=$ORIGIN", "-lcudart"])
    return out


def build_probe(force: bool = False) -> Path:
    """bench.py's random-access probes (csrc/hive_probe.cu): a measurement helper of the
    benchmark, not part of the library; built on demand by bench.py."""
    out = LIB / "libhive_probe.so"
    src = CSRC / "hive_probe.cu"
    if force or _stale(out, [src]):
        LIB.mkdir(exist_ok=True)
        _run([_nvcc(), *ARCH_FLAGS, "-O3", "-lineinfo", "-std=c++17", "-shared", "-Xcompiler", "-fPIC",
              "-Xcompiler", "-fvisibility=hidden", str(src), "-o", str(out), "-lcudart"])
    return out


def build_serve(force: bool = False) -> Path:
    out = LIB / "libhive_serve.so"
    src = CSRC / "hive_serve.cpp"
    core = build_core(force=False)
    if force or _stale(out, [src, core, INCLUDE / "hive_c.h", INCLUDE / "hive_serve.h"]):
        LIB.mkdir(exist_ok=True)
        _run([_nvcc(), "-O3", "-std=c++17", "-shared", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
              f"-I{INCLUDE}", str(src), "-o", str(out), f"-L{LIB}", "-lhive_b200", "-Xlinker", "-rpath=$ORIGIN",
              "-lcudart"])
    return out


def build_shard(force: bool = False) -> Path:
    """The sharded table's exchange kernels (csrc/hive_shard.cu, include/hive_shard.h)."""
    out = LIB / "libhive_shard.so"
    src = CSRC / "hive_shard.cu"
    if force or _stale(out, [src, INCLUDE / "hive_shard.h"]):
        LIB.mkdir(exist_ok=True)
        _run([_nvcc(), *ARCH_FLAGS, "-O3", "-lineinfo", "-std=c++17", "-shared", "-Xcompiler", "-fPIC",
              "-Xcompiler", "-fvisibility=hidden", f"-I{INCLUDE}", str(src), "-o", str(out), "-lcudart"])
    return out


def build_all(force: bool = False) -> list[Path]:
    outs = [build_core(force), build_workload(force), build_serve(force), build_shard(force)]
    if (CSRC / "hive_compat.cpp").exists():
        outs.append(build_compat(force))
    return outs


if __name__ == "__main__":
    for p in build_all(force="--force" in sys.argv):
        print(p)
