/* hive_c.h -- C ABI of the B200 Hive hash table (32-bit keys, 32-bit values).
 *
 * Every entry point takes plain pointers and sizes, returns an int status (HIVE_OK = 0), and
 * never exits the process.  Key/value/status arrays are DEVICE pointers owned by the caller;
 * work is enqueued on `stream` (a cudaStream_t passed as void*, NULL = legacy default stream)
 * and is stream-ordered: outputs are valid once the stream has reached the call.  Calls that
 * return a host value (hive_size, hive_dump's count, hive_counters, hive_check) synchronise
 * `stream` first.  A table handle is not thread-safe; use one host thread per handle.
 *
 * Key 0 is reserved as the empty sentinel (reference include/utils.h:39-47): inserting it fails,
 * looking it up or deleting it finds nothing.  Any other 32-bit key is valid.
 *
 * Each declaration cites the reference interface (SabbirPulok/HiveHashTable, path:line) that it
 * replaces.  The reference's C++ entry points (hash_table_kernel_dispatch & co.) are rebuilt on
 * top of this ABI in hivehashtable_b200/csrc/hive_compat.cpp.
 */
#ifndef HIVE_C_H
#define HIVE_C_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* The library is built with hidden visibility; exactly the entry points below are exported. */
#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif

/* ---- status codes -------------------------------------------------------------------------- */
#define HIVE_OK 0
#define HIVE_ERR_INVALID_ARG 1   /* null handle/pointer, bad policy, size out of range        */
#define HIVE_ERR_CUDA 2          /* a CUDA runtime call failed (see hive_last_cuda_error)     */
#define HIVE_ERR_OOM 3           /* device allocation failed                                   */
#define HIVE_ERR_LOCK_TIMEOUT 4  /* a bucket-lock wait expired inside a kernel (sticky)        */
#define HIVE_ERR_RETRY_LIMIT 5   /* a CAS retry budget ran out inside a kernel (sticky)        */
#define HIVE_ERR_CAPACITY 6      /* resize refused, or hive_load entries that found no room    */
#define HIVE_ERR_NO_DEVICE 7     /* no CUDA device / the library was not built for it         */

/* ---- hash policies (reference include/HashPolicies.cuh:10-17, :29-36) ------------------------ */
#define HIVE_POLICY_DEFAULT2HASH 0   /* {hash1 (Wang), hash2 (Jenkins)} */
#define HIVE_POLICY_MURMURCITYHASH 1 /* {murmurhash, cityhash}          */

/* ---- per-op status bytes written by insert / erase / apply ----------------------------------- */
#define HIVE_ST_FAIL 0      /* not placed (stash full, key 0) / not found                      */
#define HIVE_ST_INSERTED 1  /* new key placed in a bucket; find/erase/increment: success       */
#define HIVE_ST_UPDATED 2   /* existing key's value overwritten (upsert)                       */
#define HIVE_ST_STASHED 3   /* new key placed in the overflow stash                            */
#define HIVE_ST_ERROR 255   /* a bounded wait expired for this op                              */

/* ---- op codes of hive_apply_ops (same numbering as reference OperationType, include/utils.h:10-16) */
#define HIVE_OP_INSERT 0
#define HIVE_OP_LOOKUP 1
#define HIVE_OP_DELETE 2
#define HIVE_OP_INCREMENT 3 /* the reference's ATOMIC_INC */
#define HIVE_OP_NONE 4

/* hints for hive_apply_ops / hive_apply_reference_ops */
#define HIVE_HINT_NO_DELETES 1u   /* caller guarantees the batch holds no DELETE op                */
#define HIVE_HINT_LOOKUPS_ONLY 2u /* batch holds only LOOKUP/NONE ops and no other call modifies the
                                     table meanwhile: lookups take the read-only load path and any
                                     other op type is answered 0 without running               */
#define HIVE_HINT_UNIQUE_KEYS 4u  /* caller guarantees each key appears at most once in the batch
                                     (as a coalescing server or a deduplicated batch does): on a
                                     table that has had deletes, inserts then find an existing
                                     copy and a free slot from the per-slot fingerprints and
                                     claim without the canonical bucket's lock (without the hint
                                     a new key is claimed only under that lock, which serialises
                                     the inserts of one key).  A batch that breaks the promise
                                     may keep two copies of a key                            */

/* ---- counters (hive_counters) ---------------------------------------------------------------- */
#define HIVE_CTR_SLOW_PATH 0    /* inserts whose canonical bucket was full                     */
#define HIVE_CTR_EVICTIONS 1    /* keys moved by cuckoo eviction                               */
#define HIVE_CTR_STASH_PUSH 2   /* keys placed in the stash                                    */
#define HIVE_CTR_FAILED 3       /* inserts that could not be placed                            */
#define HIVE_CTR_LOCK_TIMEOUT 4 /* bucket-lock waits that expired                              */
#define HIVE_CTR_RETRY_OUT 5    /* CAS retry budgets that ran out                              */
#define HIVE_CTR_DUP_FIXED 6    /* always 0: inserts of one key claim under one lock, no copies */
#define HIVE_CTR_LOCK_WAITS 7   /* bucket-lock attempts that found the lock taken (contention) */
#define HIVE_CTR_ERROR 15       /* sticky error bits                                           */
#define HIVE_NUM_COUNTERS 16

typedef struct hive_table hive_table; /* opaque */

typedef struct hive_config {
    uint64_t capacity_slots;     /* slots at creation; buckets = ceil(capacity_slots / 8)        */
    uint64_t max_capacity_slots; /* slots reserved for growth by hive_resize (0 = capacity)      */
    int32_t policy;              /* HIVE_POLICY_*                                                */
    int32_t max_evictions;       /* cuckoo victims tried per insert, 0..8 (reference default 8)  */
    int32_t device;              /* CUDA device ordinal; -1 = the current device                 */
    uint32_t reserved;           /* must be 0                                                    */
} hive_config;

typedef struct hive_info {
    uint64_t num_buckets;     /* buckets in use (n_lo + split)                                */
    uint64_t capacity_slots;  /* num_buckets * 8                                              */
    uint64_t max_buckets;     /* buckets allocated                                            */
    uint32_t base_buckets;    /* N0: buckets at level 0                                       */
    uint32_t level;           /* linear-hashing level L (n_lo = N0 << L)                      */
    uint32_t split;           /* buckets [0, split) already split at this level               */
    int32_t policy;
    int32_t max_evictions;
    uint32_t flags;           /* bit 0: deletes or a resize ran since the last clear          */
    int32_t device;
    uint32_t reserved;
} hive_info;

/* Create a table with `capacity_slots` slots of zeroed HBM and room for max_capacity_slots.
 * Replaces hiveHashTableCreate (include/hive_hash_table.cuh:92-113, src/hive_memory.cu:29-171),
 * which sizes buckets from table_size / 8 the same way (src/hive_dispatch.cu:630-631). */
int hive_create(const hive_config* cfg, hive_table** out);

/* Free all device memory of the table.  Replaces hiveHashTableDestroy
 * (include/hive_hash_table.cuh:115-128, src/hive_memory.cu:174-307). */
int hive_destroy(hive_table* t);

/* Empty the table (and its stash, locks, counters) and undo any resize.  Replaces
 * hiveHashTableClear (include/hive_hash_table.cuh:141-143, src/hive_memory.cu:203-240). */
int hive_clear(hive_table* t, void* stream);

/* Bulk upsert of n (key, value) pairs; status[i] = HIVE_ST_*.  status may be NULL.
 * Replaces hive_insert_kernel launched by run_hash_table_benchmark
 * (include/hive_kernels.cuh:205-266, src/hive_dispatch.cu:134-148), with explicit values
 * instead of the reference's value = key + 1 (include/hive_kernels.cuh:238).  The table keeps a
 * queue for the ops that need a second pass, about 12.75 bytes per op of the largest batch, grown
 * with cudaMalloc (stream-synchronising) the first time a batch is larger than any before. */
int hive_insert(hive_table* t, const uint32_t* keys, const uint32_t* values, uint64_t n,
                uint8_t* status, void* stream);

/* hive_insert without any device allocation.  No counterpart in the reference.
 *
 * hive_insert keeps its second-pass queue (about 13 bytes per op) in device memory that it allocates,
 * and grows with cudaMalloc the first time a batch is larger than any before.  Some callers
 * cannot allow that: a service that hands all device memory to its own pool up front, a
 * latency-bound loop where cudaMalloc/cudaFree would stall the device, code under an allocator
 * that forbids raw device allocations.  This entry point uses instead a fixed queue compiled
 * into the library (HIVE_NOALLOC_MAX_OPS entries, 4 MiB plus a 256-byte header, resident on every
 * GPU that loads the library until the process exits) and makes no allocation of any kind.
 *   - n > HIVE_NOALLOC_MAX_OPS is rejected with HIVE_ERR_TOO_LARGE before any work is queued.
 *   - The first call on each device looks up the queue's device address (cudaGetSymbolAddress)
 *     with that device current, and keeps it for the later calls on that device.
 *   - All calls share the one queue: calls whose work overlaps on the GPU (other streams, other
 *     threads, other tables) race and must be ordered by the caller.  Each call resets the queue
 *     count on `stream` before using it; the queue keeps the last call's contents otherwise.
 * Results and semantics are those of hive_insert. */
#define HIVE_NOALLOC_MAX_OPS (1u << 20)
#define HIVE_ERR_TOO_LARGE 8 /* batch larger than HIVE_NOALLOC_MAX_OPS */
int hive_insert_noalloc(hive_table* t, const uint32_t* keys, const uint32_t* values, uint64_t n,
                        uint8_t* status, void* stream);

/* hive_insert with keys, values and status in HOST memory (page-locked for overlap; pageable
 * works but its copies do not overlap).  The batch is copied in chunks of 2^22 ops on an internal
 * copy stream and each chunk's first pass runs on `stream` as soon as it lands; the later passes
 * finish the batch and the statuses are copied back on a second copy stream, so the result
 * equals hive_insert's on the same batch.  Returns once the work is queued; `status` and the
 * inputs belong to the call until `stream` completes.  Device staging arrays (18 bytes per op
 * of the largest host batch) are kept by the table.  Replaces the host-side steps of
 * hash_table_kernel_dispatch_t: ops copied to the device (src/hive_dispatch.cu:583), the kernel,
 * results copied back (src/hive_dispatch.cu:1096), done serially there. */
int hive_insert_host(hive_table* t, const uint32_t* keys, const uint32_t* values, uint64_t n,
                     uint8_t* status, void* stream);

/* hive_find with keys, values and found in HOST memory: chunked upload, lookup and download
 * overlapped as in hive_insert_host.  Either output may be NULL.  Same ordering rules. */
int hive_find_host(hive_table* t, const uint32_t* keys, uint64_t n, uint32_t* values, uint8_t* found,
                   void* stream);

/* Bulk lookup: values[i] = value of keys[i] (0 if absent), found[i] = 0/1.  Either output may be
 * NULL.  Must not overlap on the GPU with a call that modifies the same table.
 * Replaces hive_lookup_kernel (include/hive_kernels.cuh:76-117), which discards the value. */
int hive_find(hive_table* t, const uint32_t* keys, uint64_t n, uint32_t* values, uint8_t* found,
              void* stream);

/* Bulk delete of every copy of each key; status[i] = 1 removed, 0 absent.  status may be NULL.
 * Replaces the DELETE case of hive_mixed_kernel (include/hive_kernels.cuh:177-181,
 * include/hive_hash_delete.cuh:168-194). */
int hive_erase(hive_table* t, const uint32_t* keys, uint64_t n, uint8_t* status, void* stream);

/* Mixed batch, ops unordered within the call: types[i] = HIVE_OP_*, values used by INSERT.
 * status[i] = HIVE_ST_* (lookup/delete/increment: 1 success, 0 miss); out_values[i] = value
 * found (LOOKUP) or value after the increment (INCREMENT), else 0.  out_values/status may be
 * NULL.  hints: HIVE_HINT_*.
 * Replaces hive_mixed_kernel (include/hive_kernels.cuh:119-192) with structure-of-arrays input. */
int hive_apply_ops(hive_table* t, const uint8_t* types, const uint32_t* keys, const uint32_t* values,
                   uint64_t n, uint8_t* status, uint32_t* out_values, uint32_t hints, void* stream);

/* A sequence of mixed batches in ONE persistent (cooperative) launch: batch b is ops
 * [offsets[b], offsets[b+1]) of types/keys/values (device arrays, offsets a device array of
 * n_batches + 1 entries); ops within a batch are unordered, batches are applied in order (a grid
 * barrier separates them).  Outputs as hive_apply_ops, indexed by global op position.
 * max_batch_ops >= the largest batch.  blocks_per_sm: 0 = as many as fit.  The table geometry is
 * fixed for the launch: grow it (hive_resize) before a sequence that would overfill it.
 * Replaces the reference's host loop of one hive_mixed_kernel launch per batch
 * (src/hive_dispatch.cu:119-226) with one launch per sequence. */
int hive_apply_batches(hive_table* t, const uint8_t* types, const uint32_t* keys, const uint32_t* values,
                       const uint64_t* offsets, uint32_t n_batches, uint64_t max_batch_ops, uint8_t* status,
                       uint32_t* out_values, uint32_t hints, int threads_per_block, int blocks_per_sm,
                       void* stream);

/* hive_apply_ops while the same launch splits the next `split_buckets` buckets of the table's
 * current level (linear hashing: bucket b moves the keys that now address b + n_lo), so the
 * table grows while its ops run.  Lookups of keys whose bucket is being split read both its old
 * and its new home; ops that would write into those buckets, and inserts that need the locked
 * path, finish after the split, in the same launch.  Results are those of hive_apply_ops; the
 * geometry (hive_get_info) has advanced by min(split_buckets, buckets left in the level) when the
 * call returns.  Grows the allocation first (synchronously) when it lacks room.  A cooperative
 * launch.  Replaces the reference's grow between launches (hive_hash_grow,
 * include/hive_hash_resize.cuh:138-215, triggered at src/hive_dispatch.cu:181-211), which moves
 * buckets only while no op runs. */
int hive_apply_ops_split(hive_table* t, const uint8_t* types, const uint32_t* keys, const uint32_t* values,
                         uint64_t n, uint8_t* status, uint32_t* out_values, uint32_t hints, uint64_t split_buckets,
                         void* stream);

/* Mixed batch in the reference's own record layout: ops points to n 16-byte records
 * {int32 type (OperationType); 4 bytes padding; uint64 key} (include/utils.h:18-21);
 * value = (uint32)key + 1 (include/hive_kernels.cuh:156); results[i] = 1 on success else 0,
 * as uint64 (include/hive_kernels.cuh:187-190).  results may be NULL.
 * Replaces hive_mixed_kernel / hive_insert_kernel / hive_lookup_kernel as launched by
 * run_hash_table_benchmark (src/hive_dispatch.cu:119-162). */
int hive_apply_reference_ops(hive_table* t, const void* ops, uint64_t n, uint64_t* results,
                             uint32_t hints, void* stream);

/* Number of live entries (buckets + stash).  Synchronises `stream`.  Replaces
 * count_occupancy_kernel (include/hive_kernels.cuh:303-325), which counts freeMask bits. */
int hive_size(hive_table* t, uint64_t* n_out, void* stream);

/* Copy up to `cap` packed entries ((value << 32) | key, arbitrary order) to the device array kv;
 * *n_out = total number of entries (may exceed cap).  Synchronises `stream`.  No reference
 * counterpart: the reference has no way to read its table back (its compact_stash_kernel,
 * include/hive_stash_table.cuh:33-64, does this for the stash only). */
int hive_dump(hive_table* t, uint64_t* kv, uint64_t cap, uint64_t* n_out, void* stream);

/* Restore a table from n packed entries in the device array kv, in hive_dump's format and any
 * order: empties the table (keeping its current number of buckets), grows it to the next full
 * linear-hashing level when n exceeds load factor 0.9 of the slots of its unsplit level
 * (8 * n_lo, n_lo = base_buckets << level), and inserts every entry.  Keys must be unique, as a dump's are (a repeated key keeps
 * one of its values).  *n_unplaced (may be NULL) = entries not placed: key 0, or no room left;
 * the call then returns HIVE_ERR_CAPACITY and the table holds the others.  Synchronises `stream`.
 * No reference counterpart: the reference keeps no checkpoint of its table. */
int hive_load(hive_table* t, const uint64_t* kv, uint64_t n, uint64_t* n_unplaced, void* stream);

/* Grow or shrink to ceil(target_slots / 8) buckets by linear-hashing split/merge, stream-ordered
 * between other calls (synchronises `stream`).  Growth beyond the reserved capacity reallocates.
 * A shrink stops at the creation size and is refused with HIVE_ERR_CAPACITY (table unchanged)
 * when the live entries would exceed load factor 0.9 of the slots of the target's unsplit level
 * (8 * n_lo: mid-level, those buckets take twice a split bucket's share of the keys).
 * Replaces hive_hash_grow / hive_hash_shrink (include/hive_hash_resize.cuh:138-215, :340-420). */
int hive_resize(hive_table* t, uint64_t target_slots, void* stream);

/* Diagnostic: the two candidate buckets of each key (device arrays) under the table's current
 * geometry.  Replaces HashPolicy::get_bucket(0|1, key, num_buckets)
 * (include/HashPolicies.cuh:13-16, :32-35). */
int hive_bucket_of(hive_table* t, const uint32_t* keys, uint64_t n, uint32_t* b0, uint32_t* b1, void* stream);

/* Table geometry.  Host only, no device work. */
int hive_get_info(const hive_table* t, hive_info* out);

/* Copy the HIVE_NUM_COUNTERS device counters to host memory `out`.  Synchronises `stream`.
 * Replaces the per-stage InsertBreakdown timing of -DBREAKDOWN_INSERT
 * (include/hive_hash_table_struct.cuh:274-294, src/hive_dispatch.cu:268-312) with event counts. */
int hive_counters(hive_table* t, uint64_t* out, void* stream);

/* Synchronise `stream` and report a sticky in-kernel error: HIVE_ERR_LOCK_TIMEOUT or
 * HIVE_ERR_RETRY_LIMIT if any op hit its bound since the last clear, else HIVE_OK.
 * The reference has no counterpart (its lock spins are unbounded,
 * include/hive_hash_table_struct.cuh:101-117). */
int hive_check(hive_table* t, void* stream);

/* Structural check of the table on the device (synchronises `stream`): out[HIVE_VERIFY_*] counts
 * slots whose per-slot fingerprint byte is not their key's, keys outside both of their buckets
 * (stash entries outside their canonical bucket's stash), extra copies of a key (twice in one
 * bucket, or in more than one of its two buckets and its canonical stash), and --
 * on a table with no delete or resize since the last clear -- free slots with a nonzero
 * fingerprint.  All zero on a sound table.  Replaces the reference's post-run table checks
 * (count_occupancy_kernel, src/hive_dispatch.cu:169-176; freeMask copy-back,
 * src/hive_dispatch.cu:1023-1036), which count occupancy only. */
#define HIVE_VERIFY_TAG_MISMATCH 0
#define HIVE_VERIFY_MISPLACED 1
#define HIVE_VERIFY_DUPLICATE 2
#define HIVE_VERIFY_STALE_TAG 3
#define HIVE_VERIFY_COUNT 4
int hive_verify(hive_table* t, uint64_t* out, void* stream);

/* ---- launch tuning (hive_set_tuning / hive_get_tuning) ----------------------------------------
 * Knobs of how a batch is run, never of what it computes: every setting gives the results of
 * the one-at-a-time replay.  They replace the reference's compile-time launch constants
 * (THREADS_PER_BLOCK / blocks-per-SM in src/hive_dispatch.cu) and are what an autotuner sets. */
#define HIVE_TUNE_REGION_INSERT 0    /* large inserts in bucket-region order (a counting sort
                                        first, statuses permuted back): 1 in sub-batches with an
                                        H0-only first pass; 2 in one pass claiming H0 then H1,
                                        evicting from H1 before the stash; 0 (default): in
                                        submission order                                        */
#define HIVE_TUNE_REGION_FIND 1      /* the same for hive_find; default 0                       */
#define HIVE_TUNE_SUBBATCHES 2       /* sub-batches of a region-ordered insert, 1..8; 0 (default)
                                        = chosen from the share of the capacity the batch adds   */
#define HIVE_TUNE_SECOND_PASS_BLOCKS 3 /* resident blocks per SM of the second insert pass, 1..8;
                                          default 8 (the autotuner's choice at 2^26 slots, LF 0.9:
                                          4.10 against 4.21 ms per insert + lookup with 4)      */
#define HIVE_TUNE_BULK_RETAG 4       /* per-slot fingerprint upkeep of hive_insert*: 0 per op; 1
                                        (default) per op for batches under one op per eight
                                        buckets, else one rebuild of the fingerprints after the
                                        batch; 2 always the rebuild                              */
#define HIVE_TUNE_TAGS 5             /* per-slot fingerprints: 0 never (lookups read whole buckets);
                                        1 (default) while their words (8 bytes per bucket) fit
                                        64 MiB, i.e. up to 2^23 buckets, where they stay in L2;
                                        2 always                                                */
#define HIVE_TUNE_L2_WINDOW 6        /* L2 persistence window over the table's memory for the
                                        table's launches (a stream access-policy window set for
                                        the call and restored after it): 0 (default) never; 1
                                        when the table's memory fits the device's persisting-L2
                                        limit (about 2^22 slots and below on B200); 2 always,
                                        covering as much as the limit allows.  Measured at 2^22
                                        slots (LF 0.9, L2 flushed between batches): 2% slower
                                        with the window, so it is off unless asked for           */
#define HIVE_TUNE_STASH_DEPTH 7      /* slots of a canonical bucket's overflow stash that inserts
                                        may use, 1..8 (default 8, the reference's 8-slot stash,
                                        include/hive_stash_table.cuh:20-27): fewer keep stash
                                        reads shorter and leave more keys unplaced near LF 1     */
#define HIVE_TUNE_BINNED 8           /* binned bulk insert into a table without deletes: the ops
                                        are partitioned by the 1024-bucket bin of their canonical
                                        bucket and each bin's slots are updated in shared memory
                                        (one read and one write of every bucket per batch instead
                                        of a random read and CAS per op); the ops whose canonical
                                        bucket is full continue as in the unbinned insert.  0
                                        never; 1 (default) for batches of at least 2^20 ops and
                                        one op per bucket into a table whose slots span at least
                                        three times the L2 (2^26 slots and up on B200); 2
                                        whenever the table allows it.  Measured at 2^26 slots,
                                        LF 0.9: 2.89 ms against 3.26 ms for the unbinned insert;
                                        at 2^25 slots 1.89 against 1.62 ms                      */
#define HIVE_NUM_TUNES 9

/* Set knob `key` to `value`.  HIVE_ERR_INVALID_ARG for an unknown key or a value out of range. */
int hive_set_tuning(hive_table* t, int32_t key, int64_t value);

/* Read knob `key` into *value. */
int hive_get_tuning(const hive_table* t, int32_t key, int64_t* value);

/* Test hook for the bounded lock wait: held = 1 sets bucket `bucket`'s eviction lock as an
 * evictor holding it would, held = 0 clears it (stream-ordered).  An insert that needs a held lock
 * waits about 65 ms (2^16 attempts with a backoff), then returns HIVE_ST_ERROR for that op and
 * sets the sticky HIVE_ERR_LOCK_TIMEOUT that hive_check reports.  No counterpart in the reference,
 * whose lock spins are unbounded (include/hive_hash_table_struct.cuh:101-117). */
int hive_debug_hold_lock(hive_table* t, uint64_t bucket, int held, void* stream);

/* Message for a status code; never NULL. */
const char* hive_strerror(int status);

/* The cudaError_t (as int) of the last failing CUDA call on this thread, 0 if none. */
int hive_last_cuda_error(void);

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif

#ifdef __cplusplus
}
#endif

#endif /* HIVE_C_H */
