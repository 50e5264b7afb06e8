// ref_ab.cu -- TEST INFRASTRUCTURE: an extern "C" harness over the reference's own GPU path.
//
// oracle/build.py links this file with the reference's src/hive_dispatch.cu, src/hive_memory.cu and
// src/GPUTimer.cc (compiled from the reference tree, unchanged, for sm_100a) into
// oracle/_ref/libhive_ref_gpu.so.  Tests feed it the same seeded keys as the B200 table and compare
// per-op success flags; its timings are the reference's own (a cudaEvent pair around one kernel,
// after its 5 warm-ups and clear: src/hive_dispatch.cu:64-164).
//
// The reference sizes its buffers from cudaMemGetInfo when the library loads
// (include/hive_hash_table_struct.cuh:38-48), so the library needs a GPU to load and nothing else
// may hold most of the device memory meanwhile.
#include <cstdint>
#include <string>
#include <vector>

#include "hive_hash_table.cuh"

namespace {
std::vector<Operation> as_ops(const uint32_t* keys, size_t n, OperationType type) {
    std::vector<Operation> ops(n);
    for (size_t i = 0; i < n; ++i) ops[i] = Operation{type, (uint64_t)keys[i]};
    return ops;
}
}  // namespace

// Bulk insert through hash_table_kernel_dispatch (all-insert batch -> hive_insert_kernel).
// policy: 0 Default2Hash, 1 MurmurCityHash.  results: n uint64 0/1 flags.  Returns 0.
extern "C" int ref_bulk_insert(const uint32_t* keys, size_t n, size_t table_size, int policy, int iterations,
                               double* ms, uint64_t* results) {
    std::vector<Operation> ops = as_ops(keys, n, OperationType::INSERT);
    double t = 0.0;
    hash_table_kernel_dispatch(ops.data(), n, table_size, 256, (n + 255) / 256, (size_t)iterations, t, results, false,
                               HashTableDataLayout::HYBRID_SOA_AOS, policy == 1 ? "MurmurCityHash" : "Default2Hash");
    *ms = t;
    return 0;
}

// Prefill with `prefill` keys, then time a lookup batch through hash_table_kernel_dispatch_YCSB
// (hive_mixed_kernel LOOKUP path), as the reference's own lookup sweep does
// (src/hashTableBenchmark.cc:275-432).  Default2Hash only (the YCSB path is not templated).
extern "C" int ref_lookup(const uint32_t* prefill, size_t n_prefill, const uint32_t* look, size_t n_look,
                          size_t table_size, int iterations, double* ms, uint64_t* results) {
    std::vector<Operation> pre = as_ops(prefill, n_prefill, OperationType::INSERT);
    std::vector<Operation> ops = as_ops(look, n_look, OperationType::LOOKUP);
    double t = 0.0;
    hash_table_kernel_dispatch_YCSB(pre.data(), ops.data(), n_prefill, n_look, table_size, 256, (size_t)iterations, t,
                                    results, false, HashTableDataLayout::HYBRID_SOA_AOS);
    *ms = t;
    return 0;
}

// All-lookup batch of present keys through hash_table_kernel_dispatch (prefill with the same keys,
// then hive_lookup_kernel).
extern "C" int ref_lookup_present(const uint32_t* keys, size_t n, size_t table_size, int policy, int iterations,
                                  double* ms, uint64_t* results) {
    std::vector<Operation> ops = as_ops(keys, n, OperationType::LOOKUP);
    double t = 0.0;
    hash_table_kernel_dispatch(ops.data(), n, table_size, 256, (n + 255) / 256, (size_t)iterations, t, results, false,
                               HashTableDataLayout::HYBRID_SOA_AOS, policy == 1 ? "MurmurCityHash" : "Default2Hash");
    *ms = t;
    return 0;
}
