// hive_hash_table.cuh -- drop-in replacement for the reference's C++ host API
// (SabbirPulok/HiveHashTable include/hive_hash_table.cuh:50-144), implemented by
// libhive_compat.so on top of the C ABI in hive_c.h.
//
// Put this directory before the reference's include/ directory on the include path: the
// reference's drivers (benchmark/*.cpp, src/hashTableBenchmark.cc) then compile unchanged and link
// against -lhive_compat -lhive_b200 instead of src/hive_dispatch.cu + src/hive_memory.cu.
// The op and layout types come from the reference's own utils.h (include/utils.h:10-37), so the
// mangled names match the reference's.
//
// Host-only: no device code is declared here.  The three layouts of the reference map to the one
// B200 table layout; HashTableDataLayout::WARPSPEED (a competitor table) is not provided.
#pragma once

#include <cstddef>
#include <cstdint>
#include <string>

#include "hive_c.h"
#include "utils.h"

using key_type = uint32_t;
using value_type = uint32_t;
using kv_type = uint64_t;

// Host/device mirrors of a table, with the public fields of the reference's structs
// (include/hive_hash_table_struct.cuh:62-271).  `impl` is the B200 table; the array pointers are
// left null because the B200 layout has no freeMask/lock arrays.
struct HiveHashTable {
    static constexpr size_t SLOTS = 8;
    void* buckets = nullptr;
    uint32_t* freeMask = nullptr;
    uint32_t* lock = nullptr;
    size_t num_buckets = 0;
    size_t max_num_buckets = 0;
    size_t max_evictions = 8;
    uint32_t index_mask = 0;
    uint32_t split_ptr = 0;
    hive_table* impl = nullptr;
};

template <typename KVType>
struct HiveHashTableAoaS {
    static constexpr size_t SLOTS = 8;
    void* buckets = nullptr;
    size_t num_buckets = 0;
    size_t max_num_buckets = 0;
    size_t max_evictions = 8;
    uint32_t index_mask = 0;
    uint32_t split_ptr = 0;
    hive_table* impl = nullptr;
};

template <typename KVType>
struct HiveHashTableAoaS_LeadMetaData {
    static constexpr size_t SLOTS = 8;
    void* buckets = nullptr;
    size_t num_buckets = 0;
    size_t max_num_buckets = 0;
    size_t max_evictions = 8;
    uint32_t index_mask = 0;
    uint32_t split_ptr = 0;
    hive_table* impl = nullptr;
};

// Mixed operations over one table (src/hive_dispatch.cu:815-872).
void hash_table_kernel_dispatch(Operation* h_ops, size_t num_ops, size_t table_size, size_t threads_per_block,
                                size_t num_blocks, size_t numIterations, double& elapsed_time, uint64_t* h_results,
                                bool verify, HashTableDataLayout layout, std::string hash_policy = "Default2Hash");

// Prefill, then a timed workload (src/hive_dispatch.cu:317-549).
void hash_table_kernel_dispatch_YCSB(Operation* h_prefill_ops, Operation* h_workload_ops, size_t num_prefill_ops,
                                     size_t num_workload_ops, size_t table_size, size_t threads_per_block,
                                     size_t numIterations, double& elapsed_time, uint64_t* h_results, bool verify,
                                     HashTableDataLayout layout);

// Mixed-kernel launcher over the SoA layout (src/hive_dispatch.cu:874-1176).
void hive_launch_mix_ops_kernel(Operation* h_ops, size_t num_ops, size_t table_size, size_t threads_per_block,
                                size_t num_blocks, size_t numIterations, double& elapsed_time, uint64_t* h_results,
                                bool verify);

// Table memory management (src/hive_memory.cu:29-307).  table_device is caller-cudaMalloc'ed
// device memory of sizeof(table) bytes, as in the reference; it receives a copy of the mirror.
void hiveHashTableCreate(HiveHashTable& table_host, HiveHashTable* table_device, size_t num_buckets,
                         size_t max_num_buckets);
void hiveHashTableCreate(HiveHashTableAoaS<kv_type>& table_host, HiveHashTableAoaS<kv_type>* table_device,
                         size_t num_buckets, size_t max_num_buckets);
void hiveHashTableCreate(HiveHashTableAoaS_LeadMetaData<kv_type>& table_host,
                         HiveHashTableAoaS_LeadMetaData<kv_type>* table_device, size_t num_buckets,
                         size_t max_num_buckets);
void hiveHashTableDestroy(HiveHashTable& table_host, HiveHashTable* table_device);
void hiveHashTableDestroy(HiveHashTableAoaS<kv_type>& table_host, HiveHashTableAoaS<kv_type>* table_device);
void hiveHashTableDestroy(HiveHashTableAoaS_LeadMetaData<kv_type>& table_host,
                          HiveHashTableAoaS_LeadMetaData<kv_type>* table_device);
void hiveHashTableClear(HiveHashTable* table_device);
void hiveHashTableClear(HiveHashTableAoaS<kv_type>* table_device);
void hiveHashTableClear(HiveHashTableAoaS_LeadMetaData<kv_type>* table_device);
