/* hive_serve.h -- the served request loop over a Hive table (libhive_serve.so).
 *
 * No counterpart in the reference: its nearest path is the YCSB driver, one closed-loop bulk
 * launch per workload (src/hashTableBenchmark.cc:434-570 via src/hive_dispatch.cu:317-549).
 *
 * hive_serve_run replays an open-loop request stream against a table.  Request r arrives at
 * arrival_s[r] seconds after the call starts (non-decreasing); types[r] is HIVE_OP_LOOKUP or
 * HIVE_OP_INSERT (an upsert), keys[r]/vals[r] its key and value.  The loop admits arrived
 * requests, coalesces each batch by key, keeps up to `depth` batches in flight (continuous
 * batching; depth 1 = one synchronous batch at a time) and grows the table when free device
 * memory allows.  With grow_start > 0 growth is incremental: once the load could pass grow_start,
 * each batch first splits a bounded run of buckets (linear hashing, stream-ordered before the
 * batch, no drain), sized so that the doubling ends before the load reaches max_load.  Without
 * it, or if the load would still pass max_load, the loop drains and doubles the table at once.
 * Outputs per request: out_status (lookup: found 0/1; upsert: placed 1 / not placed 0), out_vals
 * (lookup: the value, else 0), done_s (seconds after the start when its result was on the host).  Every result equals that of a one-at-a-time
 * replay in arrival order.  All arrays are host memory.
 */
#ifndef HIVE_SERVE_H
#define HIVE_SERVE_H

#include <stdint.h>

#include "hive_c.h"

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif

typedef struct hive_serve_config {
    uint32_t depth;      /* batches in flight, 1..64 (1 = plain synchronous loop)             */
    uint32_t max_batch;  /* requests per batch                                               */
    double max_load;     /* grow before a batch could pass this load factor (0 = never grow) */
    uint64_t live_keys;  /* keys already in the table when the run starts                   */
    double grow_start;   /* begin incremental growth at this load factor (0 = off; < max_load) */
} hive_serve_config;

typedef struct hive_serve_stats {
    uint64_t batches;
    uint64_t device_lookups; /* distinct keys looked up on the device                        */
    uint64_t device_upserts; /* distinct keys written on the device                          */
    uint64_t resizes;        /* doublings completed (incremental or at once)                  */
    uint64_t refused;        /* possible new keys of batches that found no memory to grow    */
    double wall_s;           /* call start to last completion                                */
    uint64_t grow_steps;     /* bounded split steps run between batches by incremental growth */
    uint64_t drains;         /* growths that had to drain the pipeline first                 */
    double form_s;           /* host time forming batches (admission and coalescing)         */
    double launch_s;         /* host time queueing copies and table calls                    */
    double answer_s;         /* host time answering finished batches                         */
    double idle_s;           /* host time with nothing to do: waiting for arrivals or batches */
} hive_serve_stats;

int hive_serve_run(hive_table* t, const hive_serve_config* cfg, const uint8_t* types, const uint32_t* keys,
                   const uint32_t* vals, const double* arrival_s, uint64_t n, uint32_t* out_vals,
                   uint8_t* out_status, double* done_s, hive_serve_stats* stats);

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif

#ifdef __cplusplus
}
#endif

#endif /* HIVE_SERVE_H */
