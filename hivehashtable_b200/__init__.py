"""hivehashtable_b200 -- a B200-native Hive hash table (32-bit keys and values, 8-slot buckets,
two-choice bucketed cuckoo hashing with an overflow stash).

The kernels and the C ABI live in lib/libhive_b200.so (source: csrc/, header: include/hive_c.h);
the reference's C++ host API is rebuilt in lib/libhive_compat.so.  This package is the Python
mirror used by the tests and the benchmark.
"""
from .table import (  # noqa: F401
    HINT_NO_DELETES,
    HINT_UNIQUE_KEYS,
    OP_DELETE,
    OP_INCREMENT,
    OP_INSERT,
    OP_LOOKUP,
    OP_NONE,
    POLICIES,
    ST_ERROR,
    ST_FAIL,
    ST_INSERTED,
    ST_STASHED,
    ST_UPDATED,
    HiveError,
    HiveHashTable,
    as_device_u32,
    as_host_u32,
    library,
    u32,
)

__all__ = ["HiveHashTable", "HiveError", "library", "POLICIES"]
