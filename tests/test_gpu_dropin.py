"""The reference's own CLI drivers (benchmark/*.cpp + src/hashTableBenchmark.cc, unchanged) built
against include/hive_hash_table.cuh and linked to libhive_compat.so + libhive_b200.so by
oracle/build.py: they run on the GPU and report the success counts the workload implies."""
import re
import subprocess

import pytest

import oracle

pytestmark = pytest.mark.gpu


def _run(name, *args, timeout=600):
    exe = oracle.REF_DIR / name
    if not exe.exists():
        pytest.skip(f"{exe.name} not built (needs the reference tree at build time)")
    p = subprocess.run([str(exe), *map(str, args)], capture_output=True, text=True, timeout=timeout)
    assert p.returncode == 0, p.stdout[-2000:] + p.stderr[-2000:]
    return p.stdout + p.stderr


def _count(out, label):
    return [int(x) for x in re.findall(label + r":\s*(\d+)", out)]


def test_table_benchmark_all_inserts(cuda):
    # unique keys 1..n at LF 0.9 of 2^16 slots; every insert of the last iteration succeeds
    out = _run("dropin_hive_table_benchmark", "--table_size", 16, "--load_factor", 0.9, "--insert_ratio", 1,
               "--lookup_ratio", 0, "--delete_ratio", 0, "--num_iterations", 2, "--distribution", "unique")
    n = int(0.9 * (1 << 16))
    assert _count(out, "Successful Inserts")[-1] == n
    assert "Throughput" in out


def test_table_benchmark_mixed_defaults(cuda):
    # the driver's default 50/40/10 mix over "uniform" keys (with repeats), timed after a clear:
    # lookups and deletes race with the inserts of their keys in the same launch, and ops within
    # one launch are unordered (as in the reference), so only the inserts have a fixed outcome
    n = int(0.9 * (1 << 16))
    out = _run("dropin_hive_table_benchmark", "--table_size", 16, "--load_factor", 0.9, "--num_iterations", 1,
               "--hash_policy", "MurmurCityHash")
    assert _count(out, "Successful Inserts")[-1] == int(n * 0.5)
    assert "Average Time over 1 iterations" in out


def test_lookup_only_benchmark(cuda):
    out = _run("dropin_hive_lookup_only_benchmark", "--table_size", 16, "--load_factor", 0.7,
               "--num_iterations", 2, "--data_layout", "HybridSoA-AoS")
    n = int(0.7 * (1 << 16))
    looks = _count(out, "Successful Lookups")
    # present fractions 100, 75, 50, 25, 0 %
    assert len(looks) == 5
    for got, frac in zip(looks, (1.0, 0.75, 0.5, 0.25, 0.0)):
        assert abs(got - frac * n) <= 1, (got, frac * n)


def test_ycsb_benchmark(cuda):
    out = _run("dropin_ycsb_benchmark", "--table_size", 16, "--num_iterations", 2)
    assert "Throughput" in out and _count(out, "Successful Lookups")
