// utils.h -- the op and layout types of the reference's host API, restated so libhive_compat.so
// can be built without the reference tree.  Names, enumerator order and record layout must equal
// the reference's include/utils.h:10-37 (they are part of the ABI: mangled names and the 16-byte
// Operation record).  Only used when building libhive_compat.so; callers compile against their
// own utils.h.
#pragma once
#include <cstdint>

enum class OperationType { INSERT, LOOKUP, DELETE, ATOMIC_INC, NONE };

struct Operation {
    OperationType type;
    uint64_t key;
};

enum class HashTableDataLayout {
    HYBRID_SOA_AOS,
    ARRAY_OF_ALIGNED_STRUCTS,
    ARRAY_OF_ALIGNED_STRUCTS_LEAD_METADATA,
    WARPSPEED
};

enum class YCSBWorkLoadType { WORKLOAD_A, WORKLOAD_B, WORKLOAD_C, WORKLOAD_D, WORKLOAD_F, NONE };

static_assert(sizeof(Operation) == 16, "Operation must be the reference's 16-byte record");
