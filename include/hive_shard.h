/* hive_shard.h -- the exchange kernels of the hash-partitioned Hive table (libhive_shard.so).
 *
 * The reference is single-GPU (SabbirPulok/HiveHashTable has no multi-GPU code); these calls have
 * no counterpart there.  A batch on one rank is split by owner rank, exchanged with one
 * all-to-all (NCCL), applied to each rank's own table, and its results returned in submission
 * order.  The owner of a key is (fmix32(key ^ 0x9E3779B9) * world) >> 32: a mixer independent of
 * the table's bucket hashes, so each shard's buckets stay uniformly loaded.
 *
 * All pointers are device pointers; calls are ordered on `stream` (a cudaStream_t) and return 0,
 * or 1 for an invalid argument or a failed launch. */
#ifndef HIVE_SHARD_H
#define HIVE_SHARD_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* The library is built with hidden visibility; exactly the entry points below are exported. */
#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif

#define HIVE_SHARD_MAX_RANKS 1024
#define HIVE_SHARD_TILE 4096 /* ops per block of the count and scatter passes */

/* Blocks of the count and scatter passes for a batch of n ops. */
uint64_t hive_shard_blocks(uint64_t n);

/* counts[r * blocks + b] = ops of block b (ops [b * HIVE_SHARD_TILE, (b + 1) * HIVE_SHARD_TILE))
 * owned by rank r, for r < world; counts holds world * hive_shard_blocks(n) words. */
int hive_shard_count(const uint32_t* keys, uint64_t n, uint32_t world, uint32_t* counts, void* stream);

/* With starts = the exclusive prefix sum of counts in the same rank-major order, every op's key,
 * value and type (vals / types may be NULL, with their outputs) are written at their place in
 * destination order (rank 0's ops first), and pos[i] = op i's place. */
int hive_shard_scatter(const uint32_t* keys, const uint32_t* vals, const uint8_t* types, uint64_t n, uint32_t world,
                       const uint64_t* starts, uint32_t* out_keys, uint32_t* out_vals, uint8_t* out_types,
                       uint64_t* pos, void* stream);

/* status[i] = src_status[pos[i]], vals[i] = src_vals[pos[i]] (either pair may be NULL). */
int hive_shard_gather(const uint64_t* pos, uint64_t n, const uint8_t* src_status, const uint32_t* src_vals,
                      uint8_t* status, uint32_t* vals, void* stream);

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif

#ifdef __cplusplus
}
#endif

#endif /* HIVE_SHARD_H */
