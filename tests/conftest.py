"""Shared test setup: the `gpu` marker, library builds and common fixtures.

`-m "not gpu"` runs on a CPU-only machine (oracle pins, generators, host logic, ABI exports);
`-m gpu` runs the CUDA path against the oracle on a B200.
"""
from __future__ import annotations

import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); runs the kernels through the C ABI")


def _ensure_built():
    from hivehashtable_b200 import build as pbuild
    from oracle import build as obuild

    core = pbuild.LIB / "libhive_b200.so"
    wl = pbuild.LIB / "libhive_workload.so"
    compat = pbuild.LIB / "libhive_compat.so"
    if not core.exists():
        pbuild.build_core()
    if not wl.exists():
        pbuild.build_workload()
    if (pbuild.CSRC / "hive_compat.cpp").exists() and not compat.exists():
        pbuild.build_compat()
    if not (obuild.LIB / "libhive_oracle.so").exists():
        obuild.build_oracle()


_ensure_built()


@pytest.fixture(scope="session")
def cuda():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda", 0)
