"""TEST INFRASTRUCTURE: build recipe for the oracle and for the reference-side pins.

  oracle/lib/libhive_oracle.so        the CPU restatement (hive_oracle.cpp), g++
  oracle/_ref/hash_kat_inc            reference include/hash.hpp host hashes   (needs the reference tree)
  oracle/_ref/hash_kat_uhf            reference UniformHashFunction hash_function.cu (plain-C hash2)
  oracle/_ref/libhive_ref_hashdev.so  reference device hash policies, sm_100a

The reference is compiled directly from its sources where they lie (REFERENCE_ROOT: the
HIVE_REFERENCE_ROOT environment variable, else a directory named `reference` beside this
repository); nothing is copied into this repository and the reference's own build system is not
used.  Outputs under oracle/_ref/ are git-ignored but travel with the source tree, so the GPU
tests can use the prebuilt reference library where the reference tree is absent.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
LIB = HERE / "lib"
REF_OUT = HERE / "_ref"
REFERENCE_ROOT = Path(os.environ.get("HIVE_REFERENCE_ROOT", str(HERE.parents[1] / "reference")))
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _nvcc() -> str:
    for c in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if c and Path(c).exists():
            return c
    raise RuntimeError("nvcc not found")


def _run(cmd):
    p = subprocess.run([str(c) for c in cmd], capture_output=True, text=True)
    if p.returncode:
        sys.stderr.write(p.stdout + p.stderr)
        raise RuntimeError("oracle build step failed: " + " ".join(map(str, cmd)))


def _stale(out: Path, deps) -> bool:
    return not out.exists() or any(Path(d).stat().st_mtime > out.stat().st_mtime for d in deps)


def build_oracle(force: bool = False) -> Path:
    out = LIB / "libhive_oracle.so"
    src = HERE / "hive_oracle.cpp"
    if force or _stale(out, [src]):
        LIB.mkdir(exist_ok=True)
        _run(["g++", "-O3", "-std=c++17", "-shared", "-fPIC", "-pthread", src, "-o", out])
    return out


def reference_available() -> bool:
    return (REFERENCE_ROOT / "include" / "hash.hpp").exists()


def build_reference_pins(force: bool = False) -> list[Path]:
    """Compile the reference's hash code into oracle/_ref (only where the reference tree exists)."""
    if not reference_available():
        return []
    REF_OUT.mkdir(exist_ok=True)
    inc = REFERENCE_ROOT / "include"
    uhf = REFERENCE_ROOT / "UniformHashFunction"
    outs = []
    o = REF_OUT / "hash_kat_inc"
    if force or _stale(o, [HERE / "ref" / "hash_kat_inc.cpp", inc / "hash.hpp"]):
        _run([_nvcc(), "-std=c++17", "-O2", "-x", "cu", f"-I{inc}", HERE / "ref" / "hash_kat_inc.cpp", "-o", o])
    outs.append(o)
    o = REF_OUT / "hash_kat_uhf"
    if force or _stale(o, [HERE / "ref" / "hash_kat_uhf.cpp", uhf / "src" / "hash_function.cu"]):
        _run([_nvcc(), "-std=c++17", "-O2", f"-I{uhf / 'include'}", "-x", "cu", HERE / "ref" / "hash_kat_uhf.cpp",
              "-x", "cu", uhf / "src" / "hash_function.cu", "-o", o])
    outs.append(o)
    o = REF_OUT / "libhive_ref_hashdev.so"
    if force or _stale(o, [HERE / "ref" / "hash_dev_kat.cu", inc / "hash.hpp", inc / "HashPolicies.cuh"]):
        _run([_nvcc(), *ARCH, "-std=c++17", "-O3", "-shared", "-Xcompiler", "-fPIC", f"-I{inc}",
              HERE / "ref" / "hash_dev_kat.cu", "-o", o])
    outs.append(o)
    return outs


def build_reference_gpu(force: bool = False) -> list[Path]:
    """The reference's own GPU path (src/hive_dispatch.cu, src/hive_memory.cu, src/GPUTimer.cc,
    unchanged, with its include/ tree) for sm_100a, plus the extern "C" harness ref/ref_ab.cu, into
    oracle/_ref/libhive_ref_gpu.so.  Flags follow the reference Makefile's release build
    (Makefile:7-13, :33-39): -O3 -lineinfo --extended-lambda."""
    if not reference_available():
        return []
    REF_OUT.mkdir(exist_ok=True)
    o = REF_OUT / "libhive_ref_gpu.so"
    srcs = [REFERENCE_ROOT / "src" / "hive_dispatch.cu", REFERENCE_ROOT / "src" / "hive_memory.cu",
            REFERENCE_ROOT / "src" / "GPUTimer.cc", HERE / "ref" / "ref_ab.cu"]
    cccl = Path(_nvcc()).resolve().parent.parent / "include" / "cccl"
    if force or _stale(o, srcs):
        cmd = [_nvcc(), *ARCH, "-std=c++17", "-O3", "-lineinfo", "--extended-lambda", "-shared", "-Xcompiler",
               "-fPIC", f"-I{REFERENCE_ROOT}", f"-I{REFERENCE_ROOT / 'include'}", f"-I{cccl}"]
        for s in srcs:
            cmd += ["-x", "cu", s]
        _run(cmd + ["-o", o, "-lcudart"])
    return [o]


DROPIN_DRIVERS = {
    "dropin_hive_table_benchmark": "benchmark/hive_table_benchmark.cpp",
    "dropin_hive_lookup_only_benchmark": "benchmark/hive_lookup_only_benchmark.cpp",
    "dropin_ycsb_benchmark": "benchmark/ycsb_benchmark.cpp",
}


def build_dropin_drivers(force: bool = False) -> list[Path]:
    """The reference's own CLI drivers and workload harness (benchmark/*.cpp,
    src/hashTableBenchmark.cc, src/GPUTimer.cc), unchanged, compiled against this repository's
    include/hive_hash_table.cuh and linked to libhive_compat.so + libhive_b200.so instead of the
    reference's src/hive_dispatch.cu and src/hive_memory.cu.  Demonstrates the drop-in boundary."""
    if not reference_available():
        return []
    repo = HERE.parent
    pkg_lib = repo / "hivehashtable_b200" / "lib"
    if str(repo) not in sys.path:
        sys.path.insert(0, str(repo))
    from hivehashtable_b200 import build as pbuild

    pbuild.build_core()
    pbuild.build_compat()
    REF_OUT.mkdir(exist_ok=True)
    cccl = Path(_nvcc()).resolve().parent.parent / "include" / "cccl"
    common = [REFERENCE_ROOT / "src" / "hashTableBenchmark.cc", REFERENCE_ROOT / "src" / "GPUTimer.cc"]
    outs = []
    for name, drv in DROPIN_DRIVERS.items():
        o = REF_OUT / name
        deps = [REFERENCE_ROOT / drv, *common, repo / "include" / "hive_hash_table.cuh", pkg_lib / "libhive_compat.so"]
        if force or _stale(o, deps):
            cmd = [_nvcc(), *ARCH, "-std=c++17", "-O2", f"-I{repo / 'include'}", f"-I{REFERENCE_ROOT / 'include'}",
                   f"-I{cccl}"]
            for src in [REFERENCE_ROOT / drv, *common]:
                cmd += ["-x", "cu", src]
            cmd += ["-o", o, f"-L{pkg_lib}", "-lhive_compat", "-lhive_b200", f"-Xlinker=-rpath={pkg_lib}",
                    "-Xlinker=-rpath=$ORIGIN/../../hivehashtable_b200/lib", "-lcudart"]
            _run(cmd)
        outs.append(o)
    return outs


def build_all(force: bool = False) -> list[Path]:
    return [build_oracle(force), *build_reference_pins(force), *build_reference_gpu(force),
            *build_dropin_drivers(force)]


if __name__ == "__main__":
    for p in build_all(force="--force" in sys.argv):
        print(p)
