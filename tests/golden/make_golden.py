"""Regenerates the golden fixtures of tests/golden/ (run from the repository root).

  hash_kats_inc.npz   the reference's include/hash.hpp host hashes (hash1, murmurhash % M,
                      cityhash % M) evaluated by oracle/_ref/hash_kat_inc, built from the reference
                      tree by oracle/build.py
  hash_kats_uhf.npz   the reference's plain-C hashes of UniformHashFunction/src/hash_function.cu
                      (hash1, hash2, cityhash, murmurhash, all mod PRIME_N) from oracle/_ref/hash_kat_uhf
  generators.npz      the seeded generators (keys, values, shuffles, lookup sets) for the five
                      workload seeds, from the oracle
  bulk_small.npz      a small end-to-end case (seed 42): 4096 inserts into 5120 slots, then 4096
                      lookups with half present; expected results from the unordered_map replay

The reference has no tests, golden vectors or fixtures of its own, so the hash fixtures are the
outputs of the reference's code itself, and the rest freezes the oracle.
"""
from __future__ import annotations

import subprocess
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

import oracle  # noqa: E402
from oracle import build as obuild  # noqa: E402

OUT = Path(__file__).resolve().parent
N_KAT = 1024
SEEDS = (42, 7, 11, 13, 17)


def _run(exe: Path, n: int) -> list[str]:
    return subprocess.run([str(exe), str(n)], capture_output=True, text=True, check=True).stdout.splitlines()


def hash_kats() -> None:
    obuild.build_reference_pins()
    lines = _run(oracle.REF_DIR / "hash_kat_inc", N_KAT)
    mods = np.array([int(x) for x in lines[0].split()[1:]], dtype=np.uint64)
    rows = np.array([[int(x) for x in ln.split()] for ln in lines[1:]], dtype=np.uint64)
    nm = mods.size
    np.savez_compressed(OUT / "hash_kats_inc.npz", mods=mods.astype(np.uint32), keys=rows[:, 0].astype(np.uint32),
                        hash1=rows[:, 1].astype(np.uint32), murmur=rows[:, 2:2 + nm].astype(np.uint32),
                        city=rows[:, 2 + nm:2 + 2 * nm].astype(np.uint32))
    lines = _run(oracle.REF_DIR / "hash_kat_uhf", N_KAT)
    rows = np.array([[int(x) for x in ln.split()] for ln in lines], dtype=np.uint64).astype(np.uint32)
    np.savez_compressed(OUT / "hash_kats_uhf.npz", prime=np.uint32(294967291), keys=rows[:, 0], hash1=rows[:, 1],
                        hash2=rows[:, 2], city=rows[:, 3], murmur=rows[:, 4])


def generators() -> None:
    out = {}
    for s in SEEDS:
        present, absent, st = oracle.gen_keys(s, 64, 16)
        out[f"present_{s}"] = present
        out[f"absent_{s}"] = absent
        out[f"values_{s}"] = oracle.values_for(present)
        sh = np.arange(64, dtype=np.uint32)
        st2 = oracle.shuffle(sh, st)
        out[f"shuffle_{s}"] = sh
        look, st3 = oracle.lookup_set(present, absent, 24, 8, st2)
        out[f"lookup_{s}"] = look
        out[f"states_{s}"] = np.array([st, st2, st3], dtype=np.uint64)
    np.savez_compressed(OUT / "generators.npz", **out)


def bulk_small() -> None:
    n = 4096
    cap = -(-n * 10 // 8)  # ceil(n / 0.8)
    keys, absent, st = oracle.gen_keys(42, n, n // 2)
    vals = oracle.values_for(keys)
    look, _ = oracle.lookup_set(keys, absent, n // 2, n // 2, st)
    m = oracle.ReplayMap()
    ins = m.insert(keys, vals)
    fv, ff = m.find(look)
    np.savez_compressed(OUT / "bulk_small.npz", capacity=np.uint64(cap), keys=keys, values=vals, insert_status=ins,
                        lookup_keys=look, found=ff, found_values=fv)


if __name__ == "__main__":
    hash_kats()
    generators()
    bulk_small()
    for p in sorted(OUT.glob("*.npz")):
        print(p.name, p.stat().st_size)
