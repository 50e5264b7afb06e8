// hive_table.cu -- kernels and the C ABI (include/hive_c.h) of the B200 Hive hash table.
//
// One thread owns one operation: it loads a whole 64 B bucket with two 256-bit loads, matches
// all 8 slots in registers and commits with one 64-bit CAS, so a warp keeps 32 independent
// random bucket reads in flight (the reference serialises 4 ops per 4-lane tile,
// include/hive_kernels.cuh:205-266).  Grids are one thread per op in 256-thread blocks.

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <new>

#include <cooperative_groups.h>

#include "hive_c.h"
#include "hive_device.cuh"

using hive::u64;
namespace cg = cooperative_groups;

namespace {

thread_local int g_last_cuda_error = 0;

constexpr int kBlock = 256;
constexpr double kMaxShrinkLoad = 0.9;
constexpr uint64_t kLoadChunk = 1ull << 22;  // entries per insert of hive_load

inline int cuda_fail(cudaError_t e) {
    g_last_cuda_error = (int)e;
    return e == cudaErrorMemoryAllocation ? HIVE_ERR_OOM : HIVE_ERR_CUDA;
}

#define HIVE_CUDA(call)                              \
    do {                                             \
        cudaError_t e_ = (call);                     \
        if (e_ != cudaSuccess) return cuda_fail(e_); \
    } while (0)

inline u64 fastmod_magic(uint32_t d) { return ~0ull / (u64)d + 1ull; }

inline unsigned grid_for(uint64_t n) { return (unsigned)((n + kBlock - 1) / kBlock); }

// Keeps the table's device current for the duration of a call and restores the caller's.
struct DeviceGuard {
    int prev = -1;
    bool ok = true;
    explicit DeviceGuard(int dev) {
        if (cudaGetDevice(&prev) != cudaSuccess) { ok = false; return; }
        if (prev != dev && cudaSetDevice(dev) != cudaSuccess) ok = false;
    }
    ~DeviceGuard() {
        int cur = -1;
        if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
    }
};

}  // namespace

struct hive_table {
    int device = 0;
    int policy = 0;
    hive::Table t{};
    uint64_t nb_cap = 0;     // buckets allocated
    uint32_t n0 = 0;         // level-0 bucket count
    uint32_t level = 0;
    void* block = nullptr;   // single allocation holding every array
    size_t block_bytes = 0;
    u64* scratch = nullptr;  // device words: [0] size/dump count, [1] deferred-op count, [2, 6) verify,
                             // [6] third-pass op count
    uint32_t* defer_q = nullptr;  // deferred-op queue (one index per op of the largest batch)
    uint64_t defer_cap = 0;
    void* rbuf = nullptr;         // region-ordering buffers (13 bytes per op of the largest batch)
    uint64_t rcap = 0;
    void* bbuf = nullptr;         // binned-insert buffers (24 bytes per op of the largest batch)
    uint64_t bcap = 0;
    int num_sms = 148;
    int l2_bytes = 126 << 20;  // the device's L2 (cudaDevAttrL2CacheSize)
    int64_t tune[HIVE_NUM_TUNES] = {0, 0, 0, 8, 1, 1, 0, 8, 1};  // HIVE_TUNE_* knobs
    bool tags_valid = true;  // the tag words match the slots (a zeroed table's do)
    void* ovf = nullptr;     // shrink: overflow entries of one merge step (kept between calls)
    size_t ovf_cap = 0;      // entries
    // host-buffer pipeline (hive_insert_host / hive_find_host): copy streams, events and device
    // staging arrays (insert keys, values, statuses; find keys, values, flags: 18 bytes per op)
    cudaStream_t pipe_h2d = nullptr, pipe_d2h = nullptr;
    cudaEvent_t ev_in = nullptr, ev_out = nullptr, ev_ins_free = nullptr, ev_find_free = nullptr;
    void* hbuf = nullptr;
    uint64_t hcap = 0;
};

namespace {

inline uint64_t num_buckets(const hive_table* h) { return (uint64_t)h->t.n_lo + h->t.split; }

// ---- L2 persistence window (HIVE_TUNE_L2_WINDOW, off by default) ---------------------------------
// A table whose memory fits in L2 (126 MB on B200; the persisting part of it is a per-process
// limit, reserved here the first time a window is used on a device) can be kept there against the
// streaming inputs and outputs of its batches: for the duration of a call, the caller's stream
// carries an access-policy window over the table's memory block with persisting hits, and the
// stream's previous window is put back when the call has queued its launches.  Measured at 2^22
// slots (a 36 MiB table, batches of 3.8 M ops, L2 flushed between batches) the window made the
// insert 1.4 % and the lookup 4 % slower: such a table and batch fit in L2 without it.
constexpr int kMaxWindowDevices = 64;
size_t g_persist_reserved[kMaxWindowDevices] = {};
std::mutex g_persist_mutex;

struct L2Window {
    cudaStream_t s = nullptr;
    bool active = false;
    cudaStreamAttrValue prev{};

    L2Window(const hive_table* h, cudaStream_t stream) : s(stream) {
        const int64_t mode = h->tune[HIVE_TUNE_L2_WINDOW];
        if (mode == 0 || h->device < 0 || h->device >= kMaxWindowDevices) return;
        int max_persist = 0, max_window = 0;
        // a failed query or setting leaves the call without a window (and clears its error)
        if (cudaDeviceGetAttribute(&max_persist, cudaDevAttrMaxPersistingL2CacheSize, h->device) != cudaSuccess ||
            cudaDeviceGetAttribute(&max_window, cudaDevAttrMaxAccessPolicyWindowSize, h->device) != cudaSuccess) {
            cudaGetLastError();
            return;
        }
        if (max_persist <= 0 || max_window <= 0) return;
        const size_t bytes = h->block_bytes;
        if (mode == 1 && bytes > (size_t)max_persist) return;
        {
            std::lock_guard<std::mutex> lock(g_persist_mutex);
            size_t& reserved = g_persist_reserved[h->device];
            const size_t want = std::min(bytes, (size_t)max_persist);
            if (reserved < want) {
                if (cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, want) != cudaSuccess) {
                    cudaGetLastError();
                    return;
                }
                reserved = want;
            }
        }
        if (cudaStreamGetAttribute(s, cudaStreamAttributeAccessPolicyWindow, &prev) != cudaSuccess) {
            cudaGetLastError();
            return;
        }
        cudaStreamAttrValue w{};
        w.accessPolicyWindow.base_ptr = h->block;
        w.accessPolicyWindow.num_bytes = std::min(bytes, (size_t)max_window);
        w.accessPolicyWindow.hitRatio =
            (float)std::min(1.0, (double)max_persist / (double)w.accessPolicyWindow.num_bytes);
        w.accessPolicyWindow.hitProp = cudaAccessPropertyPersisting;
        w.accessPolicyWindow.missProp = cudaAccessPropertyStreaming;
        active = cudaStreamSetAttribute(s, cudaStreamAttributeAccessPolicyWindow, &w) == cudaSuccess;
        if (!active) cudaGetLastError();
    }
    ~L2Window() {
        if (active) cudaStreamSetAttribute(s, cudaStreamAttributeAccessPolicyWindow, &prev);
    }
};

void set_geometry(hive_table* h, uint32_t level, uint32_t split) {
    h->level = level;
    h->t.n_lo = h->n0 << level;
    h->t.split = split;
    h->t.m_lo = fastmod_magic(h->t.n_lo);
    h->t.m_hi = fastmod_magic(h->t.n_lo << 1);
}

size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

constexpr size_t kCounterBytes = (size_t)hive::kCounterStripes * hive::kCounterStride * 8;
static_assert(hive::kCounterStride >= HIVE_NUM_COUNTERS, "a counter stripe holds every counter");

struct Carve {
    size_t slots, stash, sbits, lbits, fbits, ctr, tags, scratch, total;
};
Carve carve(uint64_t nb_cap) {
    Carve c;
    size_t words = (size_t)((nb_cap + 31) / 32);
    c.slots = 0;
    c.stash = align256(c.slots + (size_t)nb_cap * 64);
    c.sbits = align256(c.stash + (size_t)nb_cap * 64);
    c.lbits = align256(c.sbits + words * 4);
    c.fbits = align256(c.lbits + ((size_t)nb_cap + 3) / 4 * 4);  // lock bytes
    c.ctr = align256(c.fbits + words * 4);
    c.tags = align256(c.ctr + kCounterBytes);
    c.scratch = align256(c.tags + (size_t)nb_cap * 8);
    c.total = align256(c.scratch + 64);  // 8 scratch words
    return c;
}

void bind_arrays(hive_table* h, void* block, uint64_t nb_cap) {
    Carve c = carve(nb_cap);
    char* base = (char*)block;
    h->block = block;
    h->block_bytes = c.total;
    h->nb_cap = nb_cap;
    h->t.slots = (u64*)(base + c.slots);
    h->t.stash = (u64*)(base + c.stash);
    h->t.stash_bits = (uint32_t*)(base + c.sbits);
    h->t.locks = (uint32_t*)(base + c.lbits);
    h->t.full_bits = (uint32_t*)(base + c.fbits);
    h->t.counters = (u64*)(base + c.ctr);
    h->t.tags = (u64*)(base + c.tags);
    h->scratch = (u64*)(base + c.scratch);
}

// ---------------------------------------------------------------------------------------------
// Kernels
// ---------------------------------------------------------------------------------------------

// The queue of ops deferred by a first pass to the second (insert stages C/D): op indices and
// their count.  q == nullptr disables deferral.  permute: visit the queue in a permuted order.
struct Defer {
    uint32_t* q;
    u64* n;
    uint32_t permute = 0;
    // Bulk inserts: the deferred op's packed (value << 32) | key beside its index, so the second
    // pass reads its ops from the queue sequentially instead of gathering them from the batch;
    // the first pass then also writes HIVE_ST_INSERTED as the deferred op's provisional status
    // and the second pass writes only statuses that differ from it (an eviction, the common
    // outcome, leaves the byte alone: a scattered 1-byte write costs a DRAM read and write).
    u64* kv = nullptr;
    u64 cap = ~0ull;  // entries the queue holds (a later count may pass it: see k_insert_deferred)
    // Bulk inserts: where the second pass hands on the ops it does not finish (their index, packed
    // kv and count): those whose H0 lock was taken and those whose eviction found no victim.
    uint32_t* sq = nullptr;
    u64* skv = nullptr;
    u64* sn = nullptr;
    u64 scap = 0;
};

// The second pass visits queue position defer_slot(j, cnt) at step j.  In submission order the
// queue is already in random bucket order and is visited in order: consecutive queue entries hold
// increasing op indices, so the keys, values and statuses they name are read and written nearly
// sequentially (a permuted visit made them random accesses, the pass's largest cost), and with
// Defer::kv the keys and values come from the queue itself.  A
// region-ordered batch's queue is in bucket order; it is visited through a bijection of [0, cnt)
// (multiplication by a prime larger than any queue) so that its deferred ops are finished in an
// order unrelated to their buckets: finished in bucket order, the last buckets' overflow would
// meet alternate buckets already filled by all earlier overflow and exhaust their stashes.
// (j < cnt < 2^32, so j * (p mod cnt) < 2^64; gcd(p mod cnt, cnt) = gcd(p, cnt) = 1.)
__device__ __forceinline__ u64 defer_slot(u64 j, u64 cnt, uint32_t permute) {
    return permute ? (j * (4294967311ull % cnt)) % cnt : j;
}

// Appends index i (and, with Defer::kv, the op's packed kv) for every lane whose st is kStDefer,
// one atomic per warp.  Every lane of the warp must call it.
__device__ __forceinline__ void defer_push(const Defer& d, bool deferred, uint64_t i, u64 kv = 0) {
    const unsigned m = __ballot_sync(0xffffffffu, deferred);
    if (!m) return;
    const unsigned lane = threadIdx.x & 31;
    const int leader = __ffs(m) - 1;
    u64 base = 0;
    if ((int)lane == leader) base = atomicAdd(d.n, (u64)__popc(m));
    base = __shfl_sync(0xffffffffu, base, leader);
    if (deferred) {
        const u64 pos = base + __popc(m & ((1u << lane) - 1u));
        d.q[pos] = (uint32_t)i;
        if (d.kv) d.kv[pos] = kv;
    }
}

// defer_push for a whole block (every thread of the block calls it once): the block's deferred ops
// are gathered in shared memory and appended to the queue with one atomic per block.  The queue
// counter is one word, and a warp atomic on it for each warp holding a deferred op (1.4 M of them
// in a bulk insert of 60 M ops) serialises on its L2 slice.
__device__ __forceinline__ void block_defer_push(const Defer& d, bool deferred, uint64_t i, u64 kv) {
    __shared__ uint32_t n_q;
    __shared__ u64 q_at;
    __shared__ uint32_t q_idx[kBlock];
    __shared__ u64 q_kv[kBlock];
    if (threadIdx.x == 0) n_q = 0;
    __syncthreads();
    const unsigned m = __ballot_sync(0xffffffffu, deferred);
    if (m) {
        const unsigned lane = threadIdx.x & 31;
        const int leader = __ffs(m) - 1;
        uint32_t at = 0;
        if ((int)lane == leader) at = atomicAdd(&n_q, (uint32_t)__popc(m));
        at = __shfl_sync(0xffffffffu, at, leader);
        if (deferred) {
            const uint32_t pos = at + __popc(m & ((1u << lane) - 1u));
            q_idx[pos] = (uint32_t)i;
            q_kv[pos] = kv;
        }
    }
    __syncthreads();
    const uint32_t c = n_q;
    if (!c) return;  // the same for every thread of the block
    if (threadIdx.x == 0) q_at = atomicAdd(d.n, (u64)c);
    __syncthreads();
    if (threadIdx.x < c) {
        d.q[q_at + threadIdx.x] = q_idx[threadIdx.x];
        if (d.kv) d.kv[q_at + threadIdx.x] = q_kv[threadIdx.x];
    }
}

// First pass (kDefer) or the whole protocol in one pass (!kDefer, batches too large to queue)
// over ops [lo, hi) of the batch; deferred ops are queued by their index in the batch, so the
// first passes of several chunks of one batch feed one second pass.
template <int P, bool kDefer, int kMode>
__global__ void __launch_bounds__(kBlock, (kDefer && hive::mode_base(kMode) == hive::kModeMono) ? 8 : 1)
    k_insert(hive::Table t, const uint32_t* __restrict__ keys, const uint32_t* __restrict__ vals, uint64_t lo,
             uint64_t hi, uint8_t* __restrict__ status, Defer d) {
    const uint64_t i = lo + (uint64_t)blockIdx.x * kBlock + threadIdx.x;
    const bool active = i < hi;
    uint8_t st = hive::kStFail;
    constexpr bool kCoop = kDefer && hive::mode_base(kMode) == hive::kModeMono && (kMode & hive::kModeUntagged) &&
                           !(kMode & hive::kModePrimary);
    if constexpr (kCoop) {
        // Bulk first pass, one op per thread: each bucket read is one request shared by a lane
        // pair (every lane of the warp takes part, so nothing here returns early).
        const uint32_t k = active ? __ldcs(keys + i) : 0u;
        const uint32_t v = active ? __ldcs(vals + i) : 0u;
        const bool live = k != 0u;
        const u64 kv = hive::pack(k, v);
        const uint32_t b0 = live ? hive::bucket_addr(t, hive::Policy<P>::h0(k)) : 0u;
        const uint32_t b1 = live ? hive::bucket_addr(t, hive::Policy<P>::h1(k)) : 0u;
        const uint32_t m0 = hive::warp_bucket_masks(t.slots, live, b0, k);
        if (live) st = hive::claim_from_masks(t, b0, k, kv, m0);
        const bool need1 = live && !st && b1 != b0;
        const uint32_t m1 = hive::warp_bucket_masks(t.slots, need1, b1, k);
        if (need1) st = hive::claim_from_masks(t, b1, k, kv, m1);
        if (live && !st) st = hive::kStDefer;
        block_defer_push(d, st == hive::kStDefer, i, kv);
    } else if (active) {
        st = hive::insert_one<P, kDefer, kMode>(t, __ldcs(keys + i), __ldcs(vals + i));
    }
    if constexpr (kDefer && !kCoop) {
        // a deferred op's key and value are read again (L2 hits: the lines were just streamed in)
        // rather than kept live across the insert
        u64 kv = 0;
        if (st == hive::kStDefer && d.kv) kv = hive::pack(__ldcg(keys + i), __ldcg(vals + i));
        defer_push(d, st == hive::kStDefer, i, kv);
    }
    // a deferred op's provisional status (Defer::kv) is kStInserted
    if (active && status && (st != hive::kStDefer || d.kv)) __stcs(status + i, st == hive::kStDefer ? hive::kStInserted : st);
}

// Second pass: the deferred inserts, grid-stride over the queue.  kKV: the queue carries the ops'
// packed kv (Defer::kv) and the statuses are provisionally kStInserted; else the ops are gathered
// from the batch by index and every status is written.  With Defer::sq (and kFlagHandOn on
// the view) an op whose H0 lock was taken or whose eviction found no victim is handed on to that
// queue for a third pass (this kernel again, over the handed-on ops); one that finds the queue
// full is finished here.
template <int P, bool kKV>
__global__ void __launch_bounds__(kBlock, 4) k_insert_deferred(hive::Table t, const uint32_t* __restrict__ keys,
                                                            const uint32_t* __restrict__ vals,
                                                            uint8_t* __restrict__ status, Defer d) {
    const u64 n = *d.n;
    const u64 cnt = n < d.cap ? n : d.cap;
    const u64 stride = (u64)gridDim.x * kBlock;
    if constexpr (kKV) {
        // (An L2 prefetch of the next op's buckets and lock word while this op runs was measured
        // slower: the lines were evicted before use and the pass's DRAM traffic grew by a third.)
        // Warp-uniform trip count: the hand-on is a warp-wide append.  An op that finds the
        // third-pass queue full runs again at once with the hand-on off (one call site, so the
        // insert path is inlined once).
        const unsigned lane = threadIdx.x & 31;
        hive::Table tv = t;
        const uint32_t flags0 = t.flags;
        for (u64 j0 = (u64)blockIdx.x * kBlock + (threadIdx.x & ~31u); j0 < cnt; j0 += stride) {
            const u64 j = j0 + lane;
            const bool active = j < cnt;
            const u64 q = active ? defer_slot(j, cnt, d.permute) : 0;
            const u64 e = active ? __ldcs(d.kv + q) : 0ull;
            uint8_t st = hive::kStInserted;
            bool run = active;
            tv.flags = flags0;
            for (;;) {
                if (run) st = hive::insert_deferred_one<P>(tv, hive::key_of(e), hive::val_of(e));
                if (!d.sq) break;
                const bool hand_on = run && st == hive::kStDefer;
                const unsigned m = __ballot_sync(0xffffffffu, hand_on);
                if (!m) break;
                const int leader = __ffs(m) - 1;
                u64 base = 0;
                if ((int)lane == leader) base = atomicAdd(d.sn, (u64)__popc(m));
                base = __shfl_sync(0xffffffffu, base, leader);
                const u64 pos = base + __popc(m & ((1u << lane) - 1u));
                if (hand_on && pos < d.scap) {
                    d.sq[pos] = __ldcs(d.q + q);
                    d.skv[pos] = e;
                }
                run = hand_on && pos >= d.scap;
                if (!__any_sync(0xffffffffu, run)) break;
                tv.flags = (flags0 & ~hive::kFlagHandOn) | hive::kFlagResumed;
            }
            // a handed-on op's status is written by the third pass
            if (status && active && st != hive::kStInserted && st != hive::kStDefer) status[__ldcs(d.q + q)] = st;
        }
    } else {
        for (u64 j = (u64)blockIdx.x * kBlock + threadIdx.x; j < cnt; j += stride) {
            const uint32_t i = d.q[defer_slot(j, cnt, d.permute)];
            const uint8_t st = hive::insert_deferred_one<P>(t, keys[i], vals[i]);
            if (status) status[i] = st;
        }
    }
}

// The general locked path out of line, for the rare op of the converged pass below that finds
// the third-pass queue full (kFlagResumed: it was counted on the slow path already).
template <int P>
__device__ __noinline__ uint8_t insert_deferred_general(const hive::Table& t, uint32_t k, uint32_t v) {
    hive::Table tr = t;
    tr.flags = (t.flags & ~hive::kFlagHandOn) | hive::kFlagResumed;
    return hive::insert_deferred_one<P>(tr, k, v);
}

// Second pass of a bulk insert into a table without holes and without tag upkeep, with the
// third-pass queue present: every lane of a warp takes its queued op through the warp-converged
// locked path (insert_locked_converged); ops it does not finish go to the third-pass queue, which
// the general pass (k_insert_deferred) finishes.  Statuses: kStInserted is already written
// (provisional), an update writes kStUpdated, a handed-on op's status is written by the third pass.
template <int P>
__global__ void __launch_bounds__(kBlock, 4) k_insert_converged(hive::Table t, uint8_t* __restrict__ status, Defer d) {
    const u64 n = *d.n;
    const u64 cnt = n < d.cap ? n : d.cap;
    const u64 stride = (u64)gridDim.x * kBlock;
    const unsigned lane = threadIdx.x & 31;
    for (u64 j0 = (u64)blockIdx.x * kBlock + (threadIdx.x & ~31u); j0 < cnt; j0 += stride) {
        const u64 j = j0 + lane;
        const bool active = j < cnt;
        const u64 qj = active ? defer_slot(j, cnt, d.permute) : 0ull;
        const u64 e = active ? __ldcs(d.kv + qj) : 0ull;
        uint8_t st = hive::insert_locked_converged<P>(t, active, hive::key_of(e), hive::val_of(e));
        const bool hand_on = active && st == hive::kStDefer;
        const unsigned m = __ballot_sync(0xffffffffu, hand_on);
        if (m) {
            const int leader = __ffs(m) - 1;
            u64 base = 0;
            if ((int)lane == leader) base = atomicAdd(d.sn, (u64)__popc(m));
            base = __shfl_sync(0xffffffffu, base, leader);
            const u64 pos = base + __popc(m & ((1u << lane) - 1u));
            if (hand_on && pos < d.scap) {
                d.sq[pos] = __ldcs(d.q + qj);
                d.skv[pos] = e;
            } else if (hand_on) {
                st = insert_deferred_general<P>(t, hive::key_of(e), hive::val_of(e));
            }
        }
        if (status && active && st != hive::kStInserted && st != hive::kStDefer) status[__ldcs(d.q + qj)] = st;
    }
}

// The second pass and, for ops it handed on, the third.
template <int P>
void launch_second_pass(unsigned grid, cudaStream_t s, const hive::Table& t, const uint32_t* keys,
                        const uint32_t* vals, uint8_t* status, const Defer& d) {
    if (!d.kv) {
        k_insert_deferred<P, false><<<grid, kBlock, 0, s>>>(t, keys, vals, status, d);
        return;
    }
    hive::Table t2 = t;
    if (d.sq) t2.flags |= hive::kFlagHandOn;
    if (d.sq && (t.flags & hive::kFlagUntagged) && !(t.flags & (hive::kFlagHoles | hive::kFlagPrimaryFirst)))
        k_insert_converged<P><<<grid, kBlock, 0, s>>>(t2, status, d);
    else
        k_insert_deferred<P, true><<<grid, kBlock, 0, s>>>(t2, keys, vals, status, d);
    if (!d.sq) return;
    Defer d3{d.sq, d.sn};
    d3.kv = d.skv;
    d3.cap = d.scap;
    hive::Table t3 = t;
    t3.flags |= hive::kFlagResumed;
    const unsigned g3 = (unsigned)std::min<uint64_t>(grid, (d.scap + kBlock - 1) / kBlock);
    k_insert_deferred<P, true><<<g3, kBlock, 0, s>>>(t3, keys, vals, status, d3);
}

// ---------------------------------------------------------------------------------------------
// Binned bulk insert.  A large bulk batch into a table without holes touches every bucket several
// times (7.2 ops per bucket at 2^26 slots and LF 0.9); one op at a time, each touch is a random
// read and CAS in HBM, which a B200 serves at about 26 G/s however the reads are issued (the
// dirty sectors' random write-backs set the rate).  Binned, each bucket crosses HBM twice per
// batch.  The ops are partitioned by the bin of their canonical bucket H0 (kBinBuckets
// consecutive buckets, 64 KiB of slots): a histogram of the bins, then two partition passes, by
// super-bin (kSuperBins bins) and then by bin, each staging a tile of ops in shared memory grouped
// by destination so that every destination's run is written contiguously (one pass straight into
// thousands of bins would scatter every op's 12 bytes, which runs at the random-write rate).
// One block per bin then loads the bin's slots into shared memory, runs the H0 stage of each of
// its ops there (update the key or claim the lowest free slot, with shared-memory atomics) and
// writes the slots back.  Ops whose H0 is full go on to H1 in a second launch (one random read
// and CAS each, as the unbinned first pass does) and from there to the locked passes.  Every H0
// claim of the batch precedes every H1 claim: each primary keeps its H0 slot, and the H1 stage
// meets buckets that hold their primaries.
// ---------------------------------------------------------------------------------------------
constexpr int kBinShift = 10;
constexpr uint32_t kBinBuckets = 1u << kBinShift;  // 64 KiB of slots per bin
constexpr int kSuperShift = 6;
constexpr uint32_t kSuperBins = 1u << kSuperShift;  // bins per super-bin
constexpr uint32_t kMaxBins = 16384;                // 2^24 buckets; the histogram in 64 KiB of shared memory
constexpr uint32_t kMaxSupers = kMaxBins / kSuperBins;
constexpr int kBinBlock = 512;
constexpr uint64_t kHistTile = (uint64_t)kBinBlock * 128;  // ops per block of the histogram
constexpr uint32_t kPartPer = 8;                            // ops per thread of a partition pass
constexpr uint32_t kPartTile = kBinBlock * kPartPer;        // ops staged per block of a partition pass
constexpr uint64_t kBinMinOps = 1ull << 20;
constexpr int kLoadBatch = 16;  // elements a thread loads before using any of them

// Device buffers of a binned insert (Bins).  The partition passes go keys/values -> (akv, aidx)
// in super-bin order -> (rkv, ridx) in bin order; the H0 stage writes each bin's ops that go on
// to H1 into the bin's own range of (okv, oidx), which reuses (akv, aidx), with their count in
// ocnt[bin].  starts[b] = ops in bins before b (starts[nbins] = all binned ops); cursors: the
// partition passes' next free place per super-bin (supcur) and per bin (bincur); tiles: the
// second partition pass's tiles (lo, hi, super-bin), their count in ntiles.
struct Bins {
    uint32_t nbins = 0, nsupers = 0;
    u64 *akv = nullptr, *rkv = nullptr, *okv = nullptr;
    uint32_t *aidx = nullptr, *ridx = nullptr, *oidx = nullptr;
    uint32_t *counts = nullptr, *starts = nullptr, *bincur = nullptr, *supcur = nullptr, *ocnt = nullptr;
    uint4* tiles = nullptr;
    uint32_t* ntiles = nullptr;
    uint32_t max_tiles = 0;
};

template <int P>
__device__ __forceinline__ uint32_t bin_of(const hive::Table& t, uint32_t k) {
    return hive::bucket_addr(t, hive::Policy<P>::h0(k)) >> kBinShift;
}

// counts[bin] += ops of the tile whose H0 lies in the bin (key 0 is never binned).
template <int P>
__global__ void __launch_bounds__(kBinBlock) k_bin_count(hive::Table t, const uint32_t* __restrict__ keys, uint64_t n,
                                                          uint32_t nbins, uint32_t* __restrict__ counts) {
    extern __shared__ uint32_t hist[];
    for (uint32_t b = threadIdx.x; b < nbins; b += kBinBlock) hist[b] = 0;
    __syncthreads();
    const uint64_t lo = (uint64_t)blockIdx.x * kHistTile, hi = lo + kHistTile < n ? lo + kHistTile : n;
    for (uint64_t i0 = lo + threadIdx.x; i0 < hi; i0 += kLoadBatch * kBinBlock) {
        uint32_t kk[kLoadBatch];  // all of the batch's loads first: several misses in flight per thread
#pragma unroll
        for (int q = 0; q < kLoadBatch; ++q) {
            const uint64_t i = i0 + (uint64_t)q * kBinBlock;
            kk[q] = i < hi ? __ldcs(keys + i) : 0u;
        }
#pragma unroll
        for (int q = 0; q < kLoadBatch; ++q)
            if (kk[q]) atomicAdd(hist + bin_of<P>(t, kk[q]), 1u);
    }
    __syncthreads();
    for (uint32_t b = threadIdx.x; b < nbins; b += kBinBlock)
        if (hist[b]) atomicAdd(counts + b, hist[b]);
}

// Exclusive scan of 1024 per-thread sums across the block (1024 threads); returns the sum of the
// threads before this one.
__device__ __forceinline__ uint32_t block_exclusive_scan_1024(uint32_t v, uint32_t* warp_sums) {
    const unsigned lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t incl = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= (unsigned)o) incl += y;
    }
    if (lane == 31) warp_sums[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = warp_sums[lane];
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= (unsigned)o) w += y;
        }
        warp_sums[lane] = w;
    }
    __syncthreads();
    return incl - v + (warp ? warp_sums[warp - 1] : 0u);
}

// One block of 1024 threads: starts and bin cursors from the counts, super-bin cursors, and the
// second partition pass's tiles (each super-bin's range cut into kPartTile-op tiles).
__global__ void __launch_bounds__(1024) k_bin_scan(Bins b) {
    __shared__ uint32_t warp_sums[32];
    const uint32_t per = (b.nbins + 1023) / 1024;
    const uint32_t b0 = threadIdx.x * per;
    uint32_t sum = 0;
    for (uint32_t x = b0; x < b0 + per && x < b.nbins; ++x) sum += b.counts[x];
    uint32_t run = block_exclusive_scan_1024(sum, warp_sums);
    for (uint32_t x = b0; x < b0 + per && x < b.nbins; ++x) {
        b.starts[x] = run;
        b.bincur[x] = run;
        run += b.counts[x];
    }
    if (threadIdx.x == 1023) b.starts[b.nbins] = run;
    __syncthreads();
    // tiles of the second pass: super-bin s (thread s) covers [starts[64 s], starts[min(64 (s + 1), nbins)])
    const uint32_t s = threadIdx.x;
    uint32_t lo = 0, hi = 0, nt = 0;
    if (s < b.nsupers) {
        lo = b.starts[s * kSuperBins];
        hi = b.starts[min((s + 1) * kSuperBins, b.nbins)];
        b.supcur[s] = lo;
        nt = (hi - lo + kPartTile - 1) / kPartTile;
    }
    __syncthreads();  // warp_sums is reused
    const uint32_t t0 = block_exclusive_scan_1024(nt, warp_sums);
    for (uint32_t j = 0; j < nt; ++j) {
        const uint32_t a = lo + j * kPartTile;
        b.tiles[t0 + j] = make_uint4(a, min(a + kPartTile, hi), s, 0u);
    }
    if (threadIdx.x == 1023) *b.ntiles = t0 + nt;
}

// Shared memory of a partition pass: the tile's ops grouped by destination, and per destination
// (up to kMaxPartDigits) its count, its first place in the group order and its first place in the
// output.
constexpr uint32_t kMaxPartDigits = kMaxSupers > kSuperBins ? kMaxSupers : kSuperBins;
struct PartSmem {
    u64 kv[kPartTile];
    uint32_t idx[kPartTile];
    uint8_t dig[kPartTile];
    uint32_t cnt[kMaxPartDigits], lstart[kMaxPartDigits], gbase[kMaxPartDigits];
    uint32_t warp_sums[32];
};

// One tile of a partition pass.  Each thread holds kPartPer ops of the tile in registers (kv,
// idx, destination d, -1 for none) and sm.cnt is zeroed.  Every op takes its rank in its group
// from a shared-memory counter; each destination's run of the output is reserved with one
// atomic on cursors[cur_base + d]; the ops are staged in shared memory in group order and the
// groups written out contiguously.
__device__ __forceinline__ void part_tile(PartSmem& sm, uint32_t ndig, const u64 (&kv)[kPartPer],
                                          const uint32_t (&idx)[kPartPer], int (&d)[kPartPer],
                                          uint32_t* cursors, uint32_t cur_base, u64* __restrict__ out_kv,
                                          uint32_t* __restrict__ out_idx) {
    // d[q] becomes (destination << 16) | rank (a tile holds fewer than 2^16 ops)
#pragma unroll
    for (int q = 0; q < (int)kPartPer; ++q)
        if (d[q] >= 0) d[q] = (d[q] << 16) | (int)atomicAdd(sm.cnt + d[q], 1u);
    __syncthreads();
    // exclusive scan of the counts (ndig <= kBinBlock threads) and the global reservations
    const uint32_t c = threadIdx.x < ndig ? sm.cnt[threadIdx.x] : 0u;
    const unsigned lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t incl = c;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= (unsigned)o) incl += y;
    }
    if (lane == 31) sm.warp_sums[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = lane < kBinBlock / 32 ? sm.warp_sums[lane] : 0u;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= (unsigned)o) w += y;
        }
        if (lane < kBinBlock / 32) sm.warp_sums[lane] = w;
    }
    __syncthreads();
    const uint32_t ex = incl - c + (warp ? sm.warp_sums[warp - 1] : 0u);
    if (threadIdx.x < ndig) {
        sm.lstart[threadIdx.x] = ex;
        sm.gbase[threadIdx.x] = c ? atomicAdd(cursors + cur_base + threadIdx.x, c) : 0u;
    }
    if (threadIdx.x == kBinBlock - 1) sm.warp_sums[31] = ex + c;  // the tile's op count (ndig <= kBinBlock)
    __syncthreads();
#pragma unroll
    for (int q = 0; q < (int)kPartPer; ++q) {
        if (d[q] < 0) continue;
        const uint32_t g = (uint32_t)d[q] >> 16;
        const uint32_t p = sm.lstart[g] + ((uint32_t)d[q] & 0xFFFFu);
        sm.kv[p] = kv[q];
        sm.idx[p] = idx[q];
        sm.dig[p] = (uint8_t)g;
    }
    __syncthreads();
    const uint32_t total = sm.warp_sums[31];
    for (uint32_t p = threadIdx.x; p < total; p += kBinBlock) {
        const uint32_t g = sm.dig[p];
        const uint32_t at = sm.gbase[g] + (p - sm.lstart[g]);
        __stcg(out_kv + at, sm.kv[p]);
        __stcg(out_idx + at, sm.idx[p]);
    }
}

// First partition pass: keys and values -> (akv, aidx) grouped by super-bin; statuses
// provisionally kStInserted (key 0: kStFail, an insert of key 0 is refused).
template <int P>
__global__ void __launch_bounds__(kBinBlock, 3) k_bin_part_super(hive::Table t, const uint32_t* __restrict__ keys,
                                                                  const uint32_t* __restrict__ vals, uint64_t n,
                                                                  Bins b, uint8_t* __restrict__ status) {
    extern __shared__ __align__(16) unsigned char part_raw[];
    PartSmem& sm = *reinterpret_cast<PartSmem*>(part_raw);
    for (uint32_t x = threadIdx.x; x < b.nsupers; x += kBinBlock) sm.cnt[x] = 0;
    const uint64_t lo = (uint64_t)blockIdx.x * kPartTile;
    u64 kv[kPartPer];
    uint32_t idx[kPartPer];
    int d[kPartPer];
    uint32_t kk[kPartPer], vv[kPartPer];
#pragma unroll
    for (int q = 0; q < (int)kPartPer; ++q) {  // every load of the tile first
        const uint64_t i = lo + (uint64_t)q * kBinBlock + threadIdx.x;
        kk[q] = i < n ? __ldcs(keys + i) : 0u;
        vv[q] = i < n ? __ldcs(vals + i) : 0u;
    }
#pragma unroll
    for (int q = 0; q < (int)kPartPer; ++q) {
        const uint64_t i = lo + (uint64_t)q * kBinBlock + threadIdx.x;
        if (i < n && status) __stcs(status + i, kk[q] ? hive::kStInserted : hive::kStFail);
        d[q] = i < n && kk[q] ? (int)(bin_of<P>(t, kk[q]) >> kSuperShift) : -1;
        kv[q] = hive::pack(kk[q], vv[q]);
        idx[q] = (uint32_t)i;
    }
    __syncthreads();  // counters zeroed
    part_tile(sm, b.nsupers, kv, idx, d, b.supcur, 0u, b.akv, b.aidx);
}

// Second partition pass: one tile of one super-bin's range of (akv, aidx) -> (rkv, ridx) grouped
// by bin.  Blocks beyond the tile count do nothing.
template <int P>
__global__ void __launch_bounds__(kBinBlock, 3) k_bin_part_bin(hive::Table t, Bins b) {
    extern __shared__ __align__(16) unsigned char part_raw[];
    PartSmem& sm = *reinterpret_cast<PartSmem*>(part_raw);
    if (blockIdx.x >= *b.ntiles) return;
    const uint4 tile = b.tiles[blockIdx.x];
    const uint32_t lo = tile.x, m = tile.y - tile.x, sup = tile.z;
    const uint32_t first = sup * kSuperBins;
    const uint32_t ndig = min(kSuperBins, b.nbins - first);
    for (uint32_t x = threadIdx.x; x < ndig; x += kBinBlock) sm.cnt[x] = 0;
    u64 kv[kPartPer];
    uint32_t idx[kPartPer];
    int d[kPartPer];
#pragma unroll
    for (int q = 0; q < (int)kPartPer; ++q) {
        const uint32_t e = q * kBinBlock + threadIdx.x;
        kv[q] = e < m ? __ldcs(b.akv + lo + e) : 0ull;
        idx[q] = e < m ? __ldcs(b.aidx + lo + e) : 0u;
    }
#pragma unroll
    for (int q = 0; q < (int)kPartPer; ++q)
        d[q] = q * kBinBlock + threadIdx.x < m ? (int)(bin_of<P>(t, hive::key_of(kv[q])) - first) : -1;
    __syncthreads();  // counters zeroed
    part_tile(sm, ndig, kv, idx, d, b.bincur, first, b.rkv, b.ridx);
}

// The bin's slots in shared memory.  A bucket is 64 bytes, half a row of the 32 four-byte banks,
// so lanes reading slot j of random buckets would all meet in two bank groups; the 16-byte chunks
// of bucket g are therefore stored rotated by XOR with bits 1-2 of g (chunk q at g * 4 +
// (q ^ slab_swizzle(g)) in 16-byte units), which spreads a warp's reads over all the banks.
__device__ __forceinline__ uint32_t slab_swizzle(uint32_t g) { return (g >> 1) & 3u; }
__device__ __forceinline__ uint32_t slab_chunk(uint32_t g, uint32_t q) { return g * 4u + (q ^ slab_swizzle(g)); }

// The H0 stage of one op against bucket g of the bin's slots (slab): an exchange if the bucket
// holds k, else a CAS of the lowest free slot.  Slots only fill during the launch, so a failed CAS
// means one more slot is taken and the loop ends within kSlots + 1 rounds; the bound is a guard.
// Returns kStUpdated, kStInserted, 0 (bucket full) or kStError.
__device__ __forceinline__ uint8_t bin_claim(u64* slab, uint32_t g, uint32_t k, u64 kv) {
    const uint32_t sw = slab_swizzle(g);
    u64* bucket = slab + (size_t)g * hive::kSlots;
    const uint32_t base = (uint32_t)__cvta_generic_to_shared(bucket);
    const auto slot = [&](int j) { return bucket + (((uint32_t)(j >> 1) ^ sw) * 2u + (uint32_t)(j & 1)); };
#pragma unroll 1
    for (int r = 0; r <= hive::kSlots; ++r) {
        uint32_t free_m = 0, match_m = 0;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            u64 x0, x1;
            asm volatile("ld.volatile.shared.v2.u64 {%0, %1}, [%2];"
                         : "=l"(x0), "=l"(x1)
                         : "r"(base + (((uint32_t)q ^ sw) << 4))
                         : "memory");
            free_m |= ((uint32_t)(x0 == 0ull) | ((uint32_t)(x1 == 0ull) << 1)) << (2 * q);
            match_m |= ((uint32_t)(hive::key_of(x0) == k) | ((uint32_t)(hive::key_of(x1) == k) << 1)) << (2 * q);
        }
        if (match_m) {
            atomicExch((unsigned long long*)slot(__ffs(match_m) - 1), (unsigned long long)kv);
            return hive::kStUpdated;
        }
        if (!free_m) return 0;
        const int j = __ffs(free_m) - 1;
        const u64 obs = atomicCAS((unsigned long long*)slot(j), 0ull, (unsigned long long)kv);
        if (obs == 0ull) return hive::kStInserted;
        if (hive::key_of(obs) == k) {
            atomicExch((unsigned long long*)slot(j), (unsigned long long)kv);
            return hive::kStUpdated;
        }
    }
    return hive::kStError;
}

// One op of the H0 stage (every lane of the warp calls it, `live` or not): the claim, then the
// op's way on -- into the bin's range of the H1 queue (n_over: a shared-memory counter) or, when
// H1 is H0, to the deferred queue -- and an update's status.
template <int P>
__device__ __forceinline__ void bin_h0_op(const hive::Table& t, const Bins& b, u64* slab, uint32_t b_lo, uint32_t lo,
                                          uint32_t* n_over, bool live, u64 kv, uint32_t i,
                                          uint8_t* __restrict__ status, const Defer& d) {
    const unsigned lane = threadIdx.x & 31;
    const uint32_t k = hive::key_of(kv);
    uint8_t st = 0;
    uint32_t b0 = 0, b1 = 0;
    if (live) {
        b0 = hive::bucket_addr(t, hive::Policy<P>::h0(k));
        st = bin_claim(slab, b0 - b_lo, k, kv);
        if (!st) b1 = hive::bucket_addr(t, hive::Policy<P>::h1(k));  // only ops that go on need H1
        if (st == hive::kStError) {
            hive::count(t, hive::kCtrRetryOut);
            hive::raise_error(t, hive::kErrRetryOut);
        }
    }
    const bool over = live && !st && b1 != b0;
    const unsigned m = __ballot_sync(0xffffffffu, over);
    if (m) {
        const int leader = __ffs(m) - 1;
        uint32_t at = 0;
        if ((int)lane == leader) at = atomicAdd(n_over, (uint32_t)__popc(m));
        at = __shfl_sync(0xffffffffu, at, leader);
        if (over) {
            const uint32_t pos = lo + at + __popc(m & ((1u << lane) - 1u));
            b.okv[pos] = kv;
            b.oidx[pos] = i;
        }
    }
    defer_push(d, live && !st && b1 == b0, i, kv);
    if (live && status && (st == hive::kStUpdated || st == hive::kStError)) status[i] = st;
}

// One block per bin: its slots into shared memory, the H0 stage of each of its ops, the slots and
// their full hints back.
template <int P>
__global__ void __launch_bounds__(kBinBlock) k_bin_h0(hive::Table t, Bins b, uint8_t* __restrict__ status, Defer d) {
    extern __shared__ __align__(16) u64 slab[];
    __shared__ uint32_t n_over;
    const uint32_t nb = t.n_lo + t.split;
    const uint32_t b_lo = blockIdx.x << kBinShift;
    const uint32_t nbk = nb - b_lo < kBinBuckets ? nb - b_lo : kBinBuckets;
    const uint4* src = reinterpret_cast<const uint4*>(t.slots + (size_t)b_lo * hive::kSlots);
    uint4* sv = reinterpret_cast<uint4*>(slab);
    const uint32_t nvec = nbk * 4u;  // 16-byte chunks
    if (threadIdx.x == 0) n_over = 0;
    for (uint32_t v0 = threadIdx.x; v0 < nvec; v0 += 4 * kBinBlock) {
        uint4 x[4];
#pragma unroll
        for (int q = 0; q < 4; ++q)
            if (v0 + q * kBinBlock < nvec) x[q] = __ldcs(src + v0 + q * kBinBlock);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const uint32_t v = v0 + q * kBinBlock;
            if (v < nvec) sv[slab_chunk(v >> 2, v & 3u)] = x[q];
        }
    }
    __syncthreads();
    const uint32_t lo = b.starts[blockIdx.x], hi = b.starts[blockIdx.x + 1];
    // two ops per lane per round, both loaded before either is used
    for (u64 base = (u64)lo + (threadIdx.x & ~31u); base < hi; base += 2 * kBinBlock) {
        const u64 r0 = base + (threadIdx.x & 31), r1 = r0 + kBinBlock;
        const bool l0 = r0 < hi, l1 = r1 < hi;
        const u64 kv0 = l0 ? __ldcs(b.rkv + r0) : 0ull, kv1 = l1 ? __ldcs(b.rkv + r1) : 0ull;
        const uint32_t i0 = l0 ? __ldcs(b.ridx + r0) : 0u, i1 = l1 ? __ldcs(b.ridx + r1) : 0u;
        bin_h0_op<P>(t, b, slab, b_lo, lo, &n_over, l0, kv0, i0, status, d);
        bin_h0_op<P>(t, b, slab, b_lo, lo, &n_over, l1, kv1, i1, status, d);
    }
    __syncthreads();
    if (threadIdx.x == 0) b.ocnt[blockIdx.x] = n_over;
    // full hints (a bin starts on a multiple of 32 buckets, so each warp owns whole words).  Each
    // lane reads its bucket's four 16-byte chunks in swizzled order, which keeps the 8 lanes of a
    // shared-memory phase on 8 different bank groups (8-byte reads of consecutive buckets put
    // every other lane on the same banks: a 16-way conflict).
    const uint4* cv = reinterpret_cast<const uint4*>(slab);
    for (uint32_t g = threadIdx.x; g < ((nbk + 31) & ~31u); g += kBinBlock) {
        bool full = g < nbk;
        if (full) {
#pragma unroll
            for (uint32_t q = 0; q < 4; ++q) {
                const uint4 c = cv[slab_chunk(g, q)];
                full = full && (c.x | c.y) && (c.z | c.w);
            }
        }
        const unsigned fm = __ballot_sync(0xffffffffu, full);
        if ((threadIdx.x & 31) == 0 && fm) atomicOr(t.full_bits + ((b_lo + g) >> 5), fm);
    }
    uint4* dst = reinterpret_cast<uint4*>(t.slots + (size_t)b_lo * hive::kSlots);
    for (uint32_t v = threadIdx.x; v < nvec; v += kBinBlock) __stcs(dst + v, sv[slab_chunk(v >> 2, v & 3u)]);
}

// The H1 stage of the ops whose H0 was full, one block per bin over the bin's range of the H1
// queue: one lane-pair read of H1 per op and a claim or update there, as in the unbinned first
// pass.  Ops that find H1 full are deferred to the locked passes: staged in the bin's range of
// (rkv, ridx), free once the H0 stage has run, then appended to the deferred queue with one atomic
// per block (a warp atomic each on the one queue counter serialised on its L2 slice).
template <int P>
__global__ void __launch_bounds__(kBlock) k_bin_h1(hive::Table t, Bins b, uint8_t* __restrict__ status, Defer d) {
    __shared__ uint32_t n_def;
    __shared__ u64 q_base;
    const uint32_t lo = b.starts[blockIdx.x], hi = lo + b.ocnt[blockIdx.x];
    const unsigned lane = threadIdx.x & 31;
    if (threadIdx.x == 0) n_def = 0;
    __syncthreads();
    for (u64 base = (u64)lo + (threadIdx.x & ~31u); base < hi; base += kBlock) {
        const u64 r = base + lane;
        const bool live = r < hi;
        const u64 kv = live ? __ldcs(b.okv + r) : 0ull;
        const uint32_t i = live ? __ldcs(b.oidx + r) : 0u;
        const uint32_t k = hive::key_of(kv);
        const uint32_t b1 = live ? hive::bucket_addr(t, hive::Policy<P>::h1(k)) : 0u;
        const uint32_t m1 = hive::warp_bucket_masks(t.slots, live, b1, k);
        const uint8_t st = live ? hive::claim_from_masks(t, b1, k, kv, m1) : (uint8_t)0;
        const bool defer = live && !st;
        const unsigned m = __ballot_sync(0xffffffffu, defer);
        if (m) {
            const int leader = __ffs(m) - 1;
            uint32_t at = 0;
            if ((int)lane == leader) at = atomicAdd(&n_def, (uint32_t)__popc(m));
            at = __shfl_sync(0xffffffffu, at, leader);
            if (defer) {
                const uint32_t pos = lo + at + __popc(m & ((1u << lane) - 1u));
                b.rkv[pos] = kv;
                b.ridx[pos] = i;
            }
        }
        if (live && status && st == hive::kStUpdated) status[i] = st;
    }
    __syncthreads();
    const uint32_t cnt = n_def;
    if (!cnt) return;
    if (threadIdx.x == 0) q_base = atomicAdd(d.n, (u64)cnt);
    __syncthreads();
    for (uint32_t j = threadIdx.x; j < cnt; j += kBlock) {
        d.q[q_base + j] = b.ridx[lo + j];
        d.kv[q_base + j] = b.rkv[lo + j];
    }
}

// ---------------------------------------------------------------------------------------------
// Region ordering for large bulk batches.  A batch with about one op per bucket or more touches
// every bucket several times; processed in arrival order each touch is a random HBM access.
// Reordered by region (2^rshift consecutive buckets, >= 2 MiB of table), the blocks in flight at
// any moment cover a few regions, so after a region's first touches its buckets are served by
// L2 and each table line crosses HBM about once per batch.  The reorder is a counting sort by
// region over (key, value, index): one histogram pass, a scan of the region counts, one scatter
// pass (sequential traffic), and at the end one scatter of the per-op outputs back to the
// caller's order.
// ---------------------------------------------------------------------------------------------
// Regions of 2^15 .. 2^20 buckets (2 .. 64 MiB of slots), about 8 per table.  A region is the
// span the blocks in flight share: small regions crowd ~7 concurrent claimers onto each bucket
// (2 MiB regions ran a 2^26-slot insert at 7.6 ms against 4.9 ms with 64 MiB ones), while a 64 MiB
// region still stays in L2.
constexpr int kMinRegionShift = 15;
constexpr int kMaxRegionShift = 20;
constexpr int kMaxRegions = 1024;
constexpr int kRegionTile = kBlock * 8;   // ops per block in the histogram and scatter passes

// Sort bin of op i: its sub-batch (a contiguous share of the caller's order, i * nsub / n) major,
// its region minor.  Sub-batches let a batch that adds much of the table's capacity fill it in
// nsub rounds -- each a first pass and a deferred pass -- as an online insert order would, rather
// than handling all of its overflow at the end when every bucket holds its final primaries.
__device__ __forceinline__ uint32_t region_bin(const hive::Table& t, uint32_t h0, uint64_t i, uint64_t n, int nreg,
                                               int rshift, int nsub) {
    const uint32_t sub = nsub > 1 ? (uint32_t)((i * (uint64_t)nsub) / n) : 0u;
    return sub * (uint32_t)nreg + (hive::bucket_addr(t, h0) >> rshift);
}

template <int P>
__global__ void __launch_bounds__(kBlock) k_region_hist(hive::Table t, const uint32_t* __restrict__ keys, uint64_t n,
                                                        int nreg, int rshift, int nsub, uint32_t* __restrict__ counts) {
    const int nbin = nreg * nsub;
    __shared__ uint32_t hist[kMaxRegions];
    for (int r = threadIdx.x; r < nbin; r += kBlock) hist[r] = 0;
    __syncthreads();
    const uint64_t base = (uint64_t)blockIdx.x * kRegionTile;
    for (int q = threadIdx.x; q < kRegionTile; q += kBlock) {
        const uint64_t i = base + q;
        if (i < n) atomicAdd(&hist[region_bin(t, hive::Policy<P>::h0(__ldg(keys + i)), i, n, nreg, rshift, nsub)], 1u);
    }
    __syncthreads();
    for (int r = threadIdx.x; r < nbin; r += kBlock)
        if (hist[r]) atomicAdd(counts + r, hist[r]);
}

// Exclusive scan of the region counts into cursors (one block; nreg <= kMaxRegions).
__global__ void __launch_bounds__(kMaxRegions) k_region_scan(const uint32_t* __restrict__ counts, int nreg,
                                                             uint32_t* __restrict__ cursors) {
    __shared__ uint32_t s[kMaxRegions];
    const int r = threadIdx.x;
    const uint32_t c = r < nreg ? counts[r] : 0u;
    s[r] = c;
    __syncthreads();
    for (int o = 1; o < kMaxRegions; o <<= 1) {
        const uint32_t y = r >= o ? s[r - o] : 0u;
        __syncthreads();
        s[r] += y;
        __syncthreads();
    }
    if (r < nreg) cursors[r] = s[r] - c;
}

// Scatter (key, value, index) of each op to its region's next free positions.  vals may be null.
template <int P>
__global__ void __launch_bounds__(kBlock) k_region_scatter(hive::Table t, const uint32_t* __restrict__ keys,
                                                           const uint32_t* __restrict__ vals, uint64_t n, int nreg,
                                                           int rshift, int nsub, uint32_t* __restrict__ cursors,
                                                           uint32_t* __restrict__ rkeys,
                                                           uint32_t* __restrict__ rvals, uint32_t* __restrict__ ridx) {
    __shared__ uint32_t hist[kMaxRegions];
    __shared__ uint32_t start[kMaxRegions];
    constexpr int kPer = kRegionTile / kBlock;
    const int nbin = nreg * nsub;
    for (int r = threadIdx.x; r < nbin; r += kBlock) hist[r] = 0;
    __syncthreads();
    const uint64_t base = (uint64_t)blockIdx.x * kRegionTile;
    uint32_t k[kPer], reg[kPer], rank[kPer];
#pragma unroll
    for (int q = 0; q < kPer; ++q) {
        const uint64_t i = base + (uint64_t)q * kBlock + threadIdx.x;
        reg[q] = 0xFFFFFFFFu;
        if (i < n) {
            k[q] = __ldcs(keys + i);
            reg[q] = region_bin(t, hive::Policy<P>::h0(k[q]), i, n, nreg, rshift, nsub);
            rank[q] = atomicAdd(&hist[reg[q]], 1u);
        }
    }
    __syncthreads();
    for (int r = threadIdx.x; r < nbin; r += kBlock)
        if (hist[r]) start[r] = atomicAdd(cursors + r, hist[r]);
    __syncthreads();
#pragma unroll
    for (int q = 0; q < kPer; ++q) {
        if (reg[q] == 0xFFFFFFFFu) continue;
        const uint64_t i = base + (uint64_t)q * kBlock + threadIdx.x;
        const uint32_t pos = start[reg[q]] + rank[q];
        rkeys[pos] = k[q];
        if (rvals) rvals[pos] = __ldcs(vals + i);
        ridx[pos] = (uint32_t)i;
    }
}

// Outputs back to the caller's order.
__global__ void __launch_bounds__(kBlock) k_unpermute_u8(const uint32_t* __restrict__ ridx,
                                                         const uint8_t* __restrict__ src, uint64_t n,
                                                         uint8_t* __restrict__ dst) {
    const uint64_t j = (uint64_t)blockIdx.x * kBlock + threadIdx.x;
    if (j < n) dst[__ldcs(ridx + j)] = __ldcs(src + j);
}
__global__ void __launch_bounds__(kBlock) k_unpermute_find(const uint32_t* __restrict__ ridx,
                                                           const uint32_t* __restrict__ sv, const uint8_t* __restrict__ sf,
                                                           uint64_t n, uint32_t* __restrict__ dv, uint8_t* __restrict__ df) {
    const uint64_t j = (uint64_t)blockIdx.x * kBlock + threadIdx.x;
    if (j >= n) return;
    const uint32_t i = __ldcs(ridx + j);
    if (dv) dv[i] = __ldcs(sv + j);
    if (df) df[i] = __ldcs(sf + j);
}

template <int P>
__global__ void __launch_bounds__(kBlock) k_find(hive::Table t, const uint32_t* __restrict__ keys, uint64_t n,
                                                 uint32_t* __restrict__ vals, uint8_t* __restrict__ found) {
    const uint64_t i = (uint64_t)blockIdx.x * kBlock + threadIdx.x;
    if (i >= n) return;
    const uint32_t k = __ldcs(keys + i);
    uint32_t v = 0;
    const bool f = hive::find_one<P, true>(t, k, &v);
    if (vals) __stcs(vals + i, f ? v : 0u);
    if (found) __stcs(found + i, (uint8_t)f);
}

template <int P>
__global__ void __launch_bounds__(kBlock) k_erase(hive::Table t, const uint32_t* __restrict__ keys, uint64_t n,
                                                  uint8_t* __restrict__ status) {
    const uint64_t i = (uint64_t)blockIdx.x * kBlock + threadIdx.x;
    if (i >= n) return;
    const bool r = hive::erase_one<P>(t, __ldcs(keys + i));
    if (status) __stcs(status + i, (uint8_t)r);
}

template <int P, bool kDefer, int kMode>
__device__ __forceinline__ uint8_t apply_one(const hive::Table& t, uint8_t type, uint32_t k, uint32_t v,
                                             uint32_t* out) {
    *out = 0;
    switch (type) {
        case HIVE_OP_INSERT:
            return hive::insert_one<P, kDefer, kMode>(t, k, v);
        case HIVE_OP_LOOKUP: {
            uint32_t fv = 0;
            bool f = hive::find_one<P, false>(t, k, &fv);
            *out = f ? fv : 0u;
            return (uint8_t)f;
        }
        case HIVE_OP_DELETE:
            return (uint8_t)hive::erase_one<P>(t, k);
        case HIVE_OP_INCREMENT: {
            uint32_t nv = 0;
            bool f = hive::increment_one<P>(t, k, &nv);
            *out = f ? nv : 0u;
            return (uint8_t)f;
        }
        default:
            return 0;
    }
}

template <int P, bool kDefer, int kMode>
__global__ void __launch_bounds__(kBlock) k_apply(hive::Table t, const uint8_t* __restrict__ types,
                                                  const uint32_t* __restrict__ keys,
                                                  const uint32_t* __restrict__ vals, uint64_t n,
                                                  uint8_t* __restrict__ status, uint32_t* __restrict__ outv, Defer d) {
    const uint64_t i = (uint64_t)blockIdx.x * kBlock + threadIdx.x;
    const bool active = i < n;
    uint32_t o = 0;
    uint8_t st = 0;
    if (active)
        st = apply_one<P, kDefer, kMode>(t, __ldcs(types + i), __ldcs(keys + i), vals ? __ldcs(vals + i) : 0u, &o);
    // Only inserts defer.  Their queue entries carry key and value (Defer::kv), and the later
    // insert passes (k_insert_deferred) write only statuses that differ from the provisional
    // kStInserted; a deferred insert's out value is 0.
    u64 kv = 0;
    if (kDefer && st == hive::kStDefer && d.kv) kv = hive::pack(__ldcg(keys + i), vals ? __ldcg(vals + i) : 0u);
    if (kDefer) defer_push(d, st == hive::kStDefer, i, kv);
    if (!active) return;
    if (st == hive::kStDefer) {
        if (!d.kv) return;
        st = hive::kStInserted;
    }
    if (status) __stcs(status + i, st);
    if (outv) __stcs(outv + i, o);
}

// A sequence of mixed batches in one cooperative launch.  Per batch: a first pass over its ops
// (warp-uniform grid-stride, so every lane of a warp takes part in each deferral append), a grid
// barrier, the deferred inserts, a grid barrier.  Two queue counts alternate between batches:
// batch b appends to count[b & 1], and its deferred pass zeroes count[(b + 1) & 1], which no one
// uses until the next barrier.  Every block reaches every barrier (no early exit), and the
// cooperative launch guarantees all blocks are resident, so each barrier completes.
template <int P, int kMode>
__global__ void k_apply_batches(hive::Table t, const uint8_t* __restrict__ types, const uint32_t* __restrict__ keys,
                                const uint32_t* __restrict__ vals, const u64* __restrict__ offsets, uint32_t nbatch,
                                uint8_t* __restrict__ status, uint32_t* __restrict__ outv, uint32_t* q, u64* qn) {
    cg::grid_group grid = cg::this_grid();
    const u64 tid = (u64)blockIdx.x * blockDim.x + threadIdx.x;
    const u64 stride = (u64)gridDim.x * blockDim.x;
    const unsigned lane = threadIdx.x & 31;
    for (uint32_t b = 0; b < nbatch; ++b) {
        const u64 lo = offsets[b], hi = offsets[b + 1];
        const Defer d{q, qn + (b & 1)};
        for (u64 base = lo + (tid - lane); base < hi; base += stride) {
            const u64 i = base + lane;
            const bool active = i < hi;
            uint32_t o = 0;
            uint8_t st = 0;
            if (active) st = apply_one<P, true, kMode>(t, types[i], keys[i], vals ? vals[i] : 0u, &o);
            defer_push(d, st == hive::kStDefer, i);
            if (active && st != hive::kStDefer) {
                if (status) status[i] = st;
                if (outv) outv[i] = o;
            }
        }
        grid.sync();
        const u64 cnt = *d.n;
        if (tid == 0) qn[(b + 1) & 1] = 0;
        for (u64 j = tid; j < cnt; j += stride) {
            const uint32_t i = q[defer_slot(j, cnt, 0)];
            const uint8_t st = hive::insert_deferred_one<P>(t, keys[i], vals ? vals[i] : 0u);
            if (status) status[i] = st;
            if (outv) outv[i] = 0u;
        }
        grid.sync();
    }
}

// Reference Operation records: {int32 type; pad; uint64 key} (include/utils.h:18-21).
__device__ __forceinline__ unsigned long long ref_result(uint8_t st) {
    return (unsigned long long)(st != hive::kStFail && st != hive::kStError);
}

template <int P, bool kDefer, int kMode>
__global__ void __launch_bounds__(kBlock) k_apply_ref(hive::Table t, const ulonglong2* __restrict__ ops, uint64_t n,
                                                      unsigned long long* __restrict__ results, Defer d) {
    const uint64_t i = (uint64_t)blockIdx.x * kBlock + threadIdx.x;
    const bool active = i < n;
    uint8_t st = 0;
    if (active) {
        const ulonglong2 rec = __ldcs(ops + i);
        const int32_t type = (int32_t)(uint32_t)rec.x;
        const uint32_t k = (uint32_t)rec.y;
        uint32_t o;
        st = (type >= 0 && type <= 3) ? apply_one<P, kDefer, kMode>(t, (uint8_t)type, k, k + 1u, &o) : 0;
    }
    if (kDefer) defer_push(d, st == hive::kStDefer, i);
    if (active && st != hive::kStDefer && results) __stcs(results + i, ref_result(st));
}

template <int P>
__global__ void __launch_bounds__(kBlock, 4) k_apply_ref_deferred(hive::Table t, const ulonglong2* __restrict__ ops,
                                                               unsigned long long* __restrict__ results, Defer d) {
    const u64 cnt = *d.n;
    for (u64 j = (u64)blockIdx.x * kBlock + threadIdx.x; j < cnt; j += (u64)gridDim.x * kBlock) {
        const uint32_t i = d.q[defer_slot(j, cnt, d.permute)];
        const uint32_t k = (uint32_t)ops[i].y;
        const uint8_t st = hive::insert_deferred_one<P>(t, k, k + 1u);
        if (results) results[i] = ref_result(st);
    }
}

// Lookup-only batches of reference records (HIVE_HINT_LOOKUPS_ONLY): read-only load path, as the
// reference's hive_lookup_kernel (include/hive_kernels.cuh:76-117).
template <int P>
__global__ void __launch_bounds__(kBlock) k_apply_ref_ro(hive::Table t, const ulonglong2* __restrict__ ops,
                                                         uint64_t n, unsigned long long* __restrict__ results) {
    const uint64_t i = (uint64_t)blockIdx.x * kBlock + threadIdx.x;
    if (i >= n) return;
    const ulonglong2 rec = __ldcs(ops + i);
    uint32_t v;
    const bool f = (int32_t)(uint32_t)rec.x == HIVE_OP_LOOKUP && hive::find_one<P, true>(t, (uint32_t)rec.y, &v);
    if (results) __stcs(results + i, (unsigned long long)f);
}

template <int P>
__global__ void k_bucket_of(hive::Table t, const uint32_t* __restrict__ keys, uint64_t n, uint32_t* b0,
                            uint32_t* b1) {
    const uint64_t i = (uint64_t)blockIdx.x * kBlock + threadIdx.x;
    if (i >= n) return;
    const uint32_t k = keys[i];
    if (b0) b0[i] = hive::bucket_addr(t, hive::Policy<P>::h0(k));
    if (b1) b1[i] = hive::bucket_addr(t, hive::Policy<P>::h1(k));
}

// Zero the stash buckets whose flag is set; one thread per flag word.
__global__ void k_clear_stash(hive::Table t, uint64_t words) {
    const uint64_t w = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (w >= words) return;
    uint32_t bits = t.stash_bits[w];
    while (bits) {
        const int b = __ffs(bits) - 1;
        bits &= bits - 1;
        ulonglong4* p = reinterpret_cast<ulonglong4*>(t.stash + (w * 32 + b) * hive::kSlots);
        p[0] = make_ulonglong4(0, 0, 0, 0);
        p[1] = make_ulonglong4(0, 0, 0, 0);
    }
}

__device__ __forceinline__ uint32_t occupied(const hive::Bucket& B) {
    uint32_t c = 0;
#pragma unroll
    for (int j = 0; j < hive::kSlots; ++j) c += B.s[j] != 0ull;
    return c;
}

// Live entries in buckets [0, nb) and their stashes; warp-reduced, one atomic per warp.
__global__ void k_count(hive::Table t, uint64_t nb, u64* out) {
    const uint64_t b = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t c = 0;
    if (b < nb) {
        hive::Bucket B;
        hive::load_bucket_ro(t.slots + b * hive::kSlots, B);
        c = occupied(B);
        if ((t.stash_bits[b >> 5] >> (b & 31)) & 1u) {
            hive::load_bucket_ro(t.stash + b * hive::kSlots, B);
            c += occupied(B);
        }
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
    if ((threadIdx.x & 31) == 0 && c) atomicAdd(out, (u64)c);
}

// Compacts every live entry into kv[0, cap); *cnt ends as the total.
__global__ void k_dump(hive::Table t, uint64_t nb, u64* __restrict__ kv, uint64_t cap, u64* cnt) {
    const uint64_t b = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    hive::Bucket B, S;
    uint32_t c = 0;
    bool st = false;
    if (b < nb) {
        hive::load_bucket_ro(t.slots + b * hive::kSlots, B);
        c = occupied(B);
        st = (t.stash_bits[b >> 5] >> (b & 31)) & 1u;
        if (st) {
            hive::load_bucket_ro(t.stash + b * hive::kSlots, S);
            c += occupied(S);
        }
    }
    const unsigned lane = threadIdx.x & 31;
    uint32_t incl = c;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= (unsigned)o) incl += y;
    }
    const uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
    u64 base = 0;
    if (lane == 31 && total) base = atomicAdd(cnt, (u64)total);
    base = __shfl_sync(0xffffffffu, base, 31);
    u64 pos = base + incl - c;
    if (b < nb) {
#pragma unroll
        for (int j = 0; j < hive::kSlots; ++j)
            if (B.s[j]) {
                if (pos < cap) kv[pos] = B.s[j];
                ++pos;
            }
        if (st) {
#pragma unroll
            for (int j = 0; j < hive::kSlots; ++j)
                if (S.s[j]) {
                    if (pos < cap) kv[pos] = S.s[j];
                    ++pos;
                }
        }
    }
}

// Splits packed entries ((value << 32) | key) into the key and value arrays an insert takes.
__global__ void __launch_bounds__(kBlock) k_unpack(const u64* __restrict__ kv, uint64_t n, uint32_t* __restrict__ keys,
                                                   uint32_t* __restrict__ vals) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        const u64 e = kv[i];
        keys[i] = (uint32_t)e;
        vals[i] = (uint32_t)(e >> 32);
    }
}

// *cnt += the ops of status[0, n) that were not placed (HIVE_ST_FAIL or HIVE_ST_ERROR).
__global__ void __launch_bounds__(kBlock) k_count_unplaced(const uint8_t* __restrict__ status, uint64_t n, u64* cnt) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const bool bad = i < n && (status[i] == HIVE_ST_FAIL || status[i] == HIVE_ST_ERROR);
    const unsigned m = __ballot_sync(0xffffffffu, bad);
    if ((threadIdx.x & 31) == 0 && m) atomicAdd(cnt, (u64)__popc(m));
}

// Copies of k in bucket (or stash bucket) p.
__device__ __forceinline__ u64 copies_in(const u64* p, uint32_t k) {
    hive::Bucket B;
    hive::load_bucket_ro(p, B);
    return (u64)__popc(hive::match_mask(B, k));
}

// Structural check of buckets [0, nb) and their stashes; out[HIVE_VERIFY_*] counts violations:
// a slot whose tag byte is not its key's fingerprint, a key in neither of its buckets (a stash
// entry not under its canonical bucket), a key with more than one copy (twice in one bucket, or
// in more than one of its H0, its H1 and H0's stash: each extra copy counted once, by the copy
// in the earlier of those places), and -- only when the table has no holes (strict) -- a free
// slot with a nonzero tag byte.
template <int P>
__global__ void k_verify(hive::Table t, uint64_t nb, bool strict, u64* out) {
    const uint64_t b = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nb) return;
    hive::Bucket B;
    hive::load_bucket_ro(t.slots + b * hive::kSlots, B);
    const u64 T = t.tags[b];
    const bool tags = !(t.flags & hive::kFlagUntagged);  // a table without tags: no tag checks
    u64 bad[HIVE_VERIFY_COUNT] = {0, 0, 0, 0};
    for (int j = 0; j < hive::kSlots; ++j) {
        const u64 kv = B.s[j];
        const uint32_t byte = (uint32_t)(T >> (8 * j)) & 0xFFu;
        if (!kv) {
            bad[HIVE_VERIFY_STALE_TAG] += tags && strict && byte != 0;
            continue;
        }
        const uint32_t k = hive::key_of(kv);
        bad[HIVE_VERIFY_TAG_MISMATCH] += tags && byte != hive::tag_of(k);
        const uint32_t c0 = hive::bucket_addr(t, hive::Policy<P>::h0(k));
        const uint32_t c1 = hive::bucket_addr(t, hive::Policy<P>::h1(k));
        bad[HIVE_VERIFY_MISPLACED] += c0 != b && c1 != b;
        for (int q = 0; q < j; ++q) bad[HIVE_VERIFY_DUPLICATE] += hive::key_of(B.s[q]) == k;
        if (c0 == b && c1 != b) bad[HIVE_VERIFY_DUPLICATE] += copies_in(t.slots + (size_t)c1 * hive::kSlots, k);
        if ((c0 == b || c1 == b) && ((t.stash_bits[c0 >> 5] >> (c0 & 31)) & 1u))
            bad[HIVE_VERIFY_DUPLICATE] += copies_in(t.stash + (size_t)c0 * hive::kSlots, k);
    }
    if ((t.stash_bits[b >> 5] >> (b & 31)) & 1u) {
        hive::load_bucket_ro(t.stash + b * hive::kSlots, B);
        for (int j = 0; j < hive::kSlots; ++j)
            if (B.s[j]) {
                const uint32_t k = hive::key_of(B.s[j]);
                bad[HIVE_VERIFY_MISPLACED] += hive::bucket_addr(t, hive::Policy<P>::h0(k)) != b;
                for (int q = 0; q < j; ++q) bad[HIVE_VERIFY_DUPLICATE] += hive::key_of(B.s[q]) == k;
            }
    }
    for (int c = 0; c < HIVE_VERIFY_COUNT; ++c)
        if (bad[c]) atomicAdd(out + c, bad[c]);
}

// Tag words of buckets [0, nb) recomputed from their slots (after an untagged bulk insert): one
// coalesced pass, 64 B read and 8 B written per bucket.
__global__ void __launch_bounds__(kBlock) k_retag(hive::Table t, uint64_t nb) {
    const uint64_t b = (uint64_t)blockIdx.x * kBlock + threadIdx.x;
    if (b >= nb) return;
    hive::Bucket B;
    hive::load_bucket_ro(t.slots + b * hive::kSlots, B);
    t.tags[b] = hive::tag_word(B.s);
}

// ---------------------------------------------------------------------------------------------
// Resize: linear hashing.  Split moves the keys of buckets [s, s + cnt) that now address
// b + n_lo; merge folds buckets [s - cnt + n_lo, s + n_lo) back into [s - cnt, s).  Both run
// between other kernels on the stream, so each bucket pair has a single owner thread.
// (The reference's host loop is include/hive_hash_resize.cuh:138-215 / :340-420; its kernels are
// not reused because of the defects listed there: slots 4-7 never split, modulus = index_mask.)
// ---------------------------------------------------------------------------------------------

template <int P>
__device__ __forceinline__ uint32_t resident_hash(const hive::Table& t, uint32_t k, uint32_t b, bool* via0) {
    const uint32_t h0 = hive::Policy<P>::h0(k);
    if (hive::bucket_addr(t, h0) == b) {
        *via0 = true;
        return h0;
    }
    *via0 = false;
    return hive::Policy<P>::h1(k);
}

// told: geometry before the split (split = s); tnew: after (split = s + cnt).
template <int P>
__global__ void k_split(hive::Table told, hive::Table tnew, uint32_t s, uint32_t cnt) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= cnt) return;
    const uint32_t b = s + i, nbk = b + told.n_lo;
    u64* src = told.slots + (size_t)b * hive::kSlots;
    u64* dst = told.slots + (size_t)nbk * hive::kSlots;
    hive::Bucket B;
    hive::load_bucket(src, B);
    // new contents of b (keep) and of b + n_lo (moved), written with their tag words at the end
    u64 keep[hive::kSlots], moved[hive::kSlots];
    int nk = 0, nd = 0;
#pragma unroll
    for (int j = 0; j < hive::kSlots; ++j) {
        keep[j] = 0ull;
        moved[j] = 0ull;
    }
#pragma unroll
    for (int j = 0; j < hive::kSlots; ++j) {
        const u64 kv = B.s[j];
        if (!kv) continue;
        bool via0;
        const uint32_t h = resident_hash<P>(told, hive::key_of(kv), b, &via0);
        if (hive::bucket_addr(tnew, h) == nbk) moved[nd++] = kv;
        else keep[nk++] = kv;
    }
    // Stash entries of canonical bucket b: re-place them by their new canonical bucket, into a
    // free slot when there is one, else into that bucket's stash.
    if ((told.stash_bits[b >> 5] >> (b & 31)) & 1u) {
        u64* sb = told.stash + (size_t)b * hive::kSlots;
        u64* sn = told.stash + (size_t)nbk * hive::kSlots;
        hive::Bucket S;
        hive::load_bucket(sb, S);
        int keep_s = 0, moved_s = 0;
        u64 ks[hive::kSlots];
        for (int j = 0; j < hive::kSlots; ++j) {
            const u64 kv = S.s[j];
            if (!kv) continue;
            const uint32_t c = hive::bucket_addr(tnew, hive::Policy<P>::h0(hive::key_of(kv)));
            if (c == b && nk < hive::kSlots) {
                keep[nk++] = kv;
            } else if (c == nbk && nd < hive::kSlots) {
                moved[nd++] = kv;
            } else if (c == b) {
                ks[keep_s++] = kv;
            } else {
                sn[moved_s++] = kv;
            }
        }
        for (int j = 0; j < hive::kSlots; ++j) sb[j] = j < keep_s ? ks[j] : 0ull;
        if (!keep_s) atomicAnd(told.stash_bits + (b >> 5), ~(1u << (b & 31)));
        if (moved_s) atomicOr(told.stash_bits + (nbk >> 5), 1u << (nbk & 31));
    }
#pragma unroll
    for (int j = 0; j < hive::kSlots; ++j) {
        src[j] = keep[j];
        dst[j] = moved[j];
    }
    told.tags[b] = hive::tag_word(keep);
    told.tags[nbk] = hive::tag_word(moved);
    if (nk == hive::kSlots) hive::mark_full(told, b);
    else hive::mark_not_full(told, b);
    if (nd == hive::kSlots) hive::mark_full(told, nbk);
}

// Split of bucket b of the window [told.split, told.win_end) while other ops of the launch read
// the table (k_apply_split).  Readers of a window key read its old home b before its new home
// nbk = b + n_lo and b's stash before nbk's (find_one_migrating), so the entries that move are
// written to their new places first and only then, after a fence, removed from the old ones.
// Entries that stay keep their positions (a reader reads a bucket in two halves), and stash
// entries stay stash entries (a stash entry moved into a slot could be passed by a reader that
// reads the slots before the stash).  No op of the launch writes into the window.
template <int P>
__device__ void split_bucket_live(const hive::Table& told, const hive::Table& tnew, uint32_t b) {
    const uint32_t nbk = b + told.n_lo;
    u64* src = told.slots + (size_t)b * hive::kSlots;
    u64* dst = told.slots + (size_t)nbk * hive::kSlots;
    const bool tags = !(told.flags & hive::kFlagUntagged);
    hive::Bucket B;
    hive::load_bucket(src, B);
    u64 moved[hive::kSlots];
    uint32_t out = 0;  // bit j: slot j of b moves
    int nd = 0;
#pragma unroll
    for (int j = 0; j < hive::kSlots; ++j) moved[j] = 0ull;
#pragma unroll
    for (int j = 0; j < hive::kSlots; ++j) {
        const u64 kv = B.s[j];
        if (!kv) continue;
        bool via0;
        const uint32_t h = resident_hash<P>(told, hive::key_of(kv), b, &via0);
        if (hive::bucket_addr(tnew, h) == nbk) {
            moved[nd++] = kv;
            out |= 1u << j;
        }
    }
    const bool has_stash = (told.stash_bits[b >> 5] >> (b & 31)) & 1u;
    hive::Bucket S;
    uint32_t sout = 0;
    int nms = 0, nks = 0;
    u64* sb = told.stash + (size_t)b * hive::kSlots;
    u64* sn = told.stash + (size_t)nbk * hive::kSlots;
    if (has_stash) {
        hive::load_bucket(sb, S);
        for (int j = 0; j < hive::kSlots; ++j) {
            const u64 kv = S.s[j];
            if (!kv) continue;
            if (hive::bucket_addr(tnew, hive::Policy<P>::h0(hive::key_of(kv))) == nbk) sout |= 1u << j;
            else ++nks;
        }
    }
    // 1. the new homes: nbk's slots and stash (and its flag, before any entry leaves b's stash)
#pragma unroll
    for (int j = 0; j < hive::kSlots; ++j) dst[j] = moved[j];
    if (sout) {
        for (int j = 0; j < hive::kSlots; ++j) sn[j] = (sout >> j) & 1u ? S.s[j] : 0ull;
        atomicOr(told.stash_bits + (nbk >> 5), 1u << (nbk & 31));
    }
    if (tags) told.tags[nbk] = hive::tag_word(moved);
    if (nd == hive::kSlots) hive::mark_full(told, nbk);
    __threadfence();
    // 2. the old home loses what moved
    u64 keep[hive::kSlots];
    int nk = 0;
#pragma unroll
    for (int j = 0; j < hive::kSlots; ++j) {
        keep[j] = (out >> j) & 1u ? 0ull : B.s[j];
        nk += keep[j] != 0ull;
        if ((out >> j) & 1u) src[j] = 0ull;
    }
    if (sout) {
        for (int j = 0; j < hive::kSlots; ++j)
            if ((sout >> j) & 1u) sb[j] = 0ull;
        if (!nks) atomicAnd(told.stash_bits + (b >> 5), ~(1u << (b & 31)));
    }
    if (tags) told.tags[b] = hive::tag_word(keep);
    if (nk == hive::kSlots) hive::mark_full(told, b);
    else hive::mark_not_full(told, b);
}

// A batch of mixed ops while the same launch splits the window [tmig.split, tmig.win_end) (a
// cooperative launch: every block is resident).  Phase 1: threads split the window's buckets,
// one bucket each, while all threads run the batch's ops against the table as it is being split
// (tmig): lookups read both homes of a window key; ops that would write into the window, and
// inserts that need the locked path, are queued.  Grid barrier.  Phase 2: the queued ops, against
// the split geometry (tnew), with the whole protocol.  Ops of one launch are unordered, so running
// some after the barrier changes no result.
template <int P, int kMode>
__global__ void k_apply_split(hive::Table tmig, hive::Table tnew, const uint8_t* __restrict__ types,
                              const uint32_t* __restrict__ keys, const uint32_t* __restrict__ vals, uint64_t n,
                              uint8_t* __restrict__ status, uint32_t* __restrict__ outv, uint32_t* q, u64* qn) {
    cg::grid_group grid = cg::this_grid();
    const u64 tid = (u64)blockIdx.x * blockDim.x + threadIdx.x;
    const u64 stride = (u64)gridDim.x * blockDim.x;
    const unsigned lane = threadIdx.x & 31;
    const uint32_t w_lo = tmig.split, w_cnt = tmig.win_end - tmig.split;
    for (u64 x = tid; x < w_cnt; x += stride) split_bucket_live<P>(tmig, tnew, w_lo + (uint32_t)x);
    const Defer d{q, qn};
    for (u64 base = tid - lane; base < n; base += stride) {
        const u64 i = base + lane;
        const bool active = i < n;
        uint32_t o = 0;
        uint8_t st = 0;
        bool later = false;
        if (active) {
            const uint8_t type = types[i];
            const uint32_t k = keys[i];
            if (type != HIVE_OP_LOOKUP && hive::touches_window<P>(tmig, k)) {
                later = true;
            } else {
                st = apply_one<P, true, kMode>(tmig, type, k, vals ? vals[i] : 0u, &o);
                later = st == hive::kStDefer;
            }
        }
        defer_push(d, later, i);
        if (active && !later) {
            if (status) status[i] = st;
            if (outv) outv[i] = o;
        }
    }
    grid.sync();
    const u64 cnt = *qn;
    for (u64 j = tid; j < cnt; j += stride) {
        const uint32_t i = q[j];
        uint32_t o = 0;
        const uint8_t st = apply_one<P, false, hive::kModeRuntime>(tnew, types[i], keys[i], vals ? vals[i] : 0u, &o);
        if (status) status[i] = st;
        if (outv) outv[i] = o;
    }
}

// told: geometry before (buckets [lo, lo + cnt) + n_lo are folded); tnew: after.
// Entries that find no room are appended to ovf for re-insertion.
template <int P>
__global__ void k_merge(hive::Table told, hive::Table tnew, uint32_t lo, uint32_t cnt, u64* ovf, u64* novf) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= cnt) return;
    const uint32_t b = lo + i, src_b = b + told.n_lo;
    u64* src = told.slots + (size_t)src_b * hive::kSlots;
    u64* ss = told.stash + (size_t)src_b * hive::kSlots;
    const bool has_stash = (told.stash_bits[src_b >> 5] >> (src_b & 31)) & 1u;
    for (int part = 0; part < (has_stash ? 2 : 1); ++part) {
        u64* from = part ? ss : src;
        hive::Bucket B;
        hive::load_bucket(from, B);
        for (int j = 0; j < hive::kSlots; ++j) {
            const u64 kv = B.s[j];
            if (!kv) continue;
            from[j] = 0ull;
            // Under the new geometry every key of src_b addresses b through the same hash.
            bool placed = false;
            u64* dstp = tnew.slots + (size_t)b * hive::kSlots;
            for (int q = 0; q < hive::kSlots && !placed; ++q)
                if (hive::cas64(dstp + q, 0ull, kv) == 0ull) placed = true;
            if (!placed) ovf[atomicAdd(novf, 1ull)] = kv;
        }
    }
    if (has_stash) atomicAnd(told.stash_bits + (src_b >> 5), ~(1u << (src_b & 31)));
    hive::mark_not_full(told, src_b);
    hive::Bucket D;
    hive::load_bucket(tnew.slots + (size_t)b * hive::kSlots, D);
    if (!hive::empty_mask(D)) hive::mark_full(told, b);
    told.tags[b] = hive::tag_word(D.s);
    told.tags[src_b] = 0ull;
}

// Re-insert overflow entries produced by k_merge through the normal insert protocol.
template <int P>
__global__ void k_reinsert(hive::Table t, const u64* __restrict__ kv, const u64* __restrict__ n, uint8_t* fail) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= *n) return;
    const u64 e = kv[i];
    const uint8_t st = hive::insert_one<P>(t, hive::key_of(e), hive::val_of(e));
    if (st == hive::kStFail || st == hive::kStError) *fail = 1;
}

template <template <int> class K>
struct ByPolicy;

int launch_check() {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e);
    return HIVE_OK;
}

int reset(hive_table* h, cudaStream_t s) {
    const uint64_t nb = num_buckets(h);
    const uint64_t words = (h->nb_cap + 31) / 32;
    HIVE_CUDA(cudaMemsetAsync(h->t.slots, 0, (size_t)nb * 64, s));
    k_clear_stash<<<(unsigned)((words + 255) / 256), 256, 0, s>>>(h->t, words);
    int rc = launch_check();
    if (rc) return rc;
    HIVE_CUDA(cudaMemsetAsync(h->t.stash_bits, 0, (size_t)words * 4, s));
    HIVE_CUDA(cudaMemsetAsync(h->t.locks, 0, (size_t)(nb + 3) / 4 * 4, s));
    HIVE_CUDA(cudaMemsetAsync(h->t.full_bits, 0, (size_t)words * 4, s));
    HIVE_CUDA(cudaMemsetAsync(h->t.counters, 0, kCounterBytes, s));
    HIVE_CUDA(cudaMemsetAsync(h->t.tags, 0, (size_t)nb * 8, s));
    return HIVE_OK;
}

bool valid_table(const hive_table* h) { return h && h->block; }

// Per-slot tags pay while their words stay in L2 (8 bytes per bucket).  Beyond that a tag word
// is one more random DRAM access per op, so larger tables run without them (HIVE_TUNE_TAGS:
// 0 never, 1 while the words fit kTagL2Bytes, 2 always).
constexpr uint64_t kTagL2Bytes = 64ull << 20;
bool use_tags(const hive_table* h) {
    const int64_t m = h->tune[HIVE_TUNE_TAGS];
    return m == 2 || (m == 1 && num_buckets(h) * 8 <= kTagL2Bytes);
}

hive::Table untagged_view(const hive_table* h) {
    hive::Table t = h->t;
    t.flags |= hive::kFlagUntagged;
    return t;
}

// Rebuild the tag words of the buckets in use from their slots.
void retag(hive_table* h, cudaStream_t s) {
    const uint64_t nb = num_buckets(h);
    k_retag<<<grid_for(nb), kBlock, 0, s>>>(h->t, nb);
    h->tags_valid = true;
}

// The Table copy a launch uses: with tags when the table uses them (rebuilding stale words first),
// else marked untagged, which leaves the words stale.
int table_view(hive_table* h, cudaStream_t s, hive::Table* tv) {
    if (use_tags(h)) {
        if (!h->tags_valid) retag(h, s);
        *tv = h->t;
    } else {
        *tv = untagged_view(h);
        h->tags_valid = false;
    }
    return launch_check();
}

// The deferred-op queue for a batch of n ops; grows (synchronously) to the largest batch seen.
// Batches of 2^32 ops or more run without deferral.
// The queue of a batch of n ops: n indices and, for bulk inserts (with_kv), n packed kv words.
// Capacity of the third-pass queue for a batch of n ops: ops reach it only after a first pass
// found both buckets full and then found H0's lock taken or no eviction victim (about 0.5 % of
// the ops of a bulk insert at load factor 0.9); further ones are finished in the second pass.
uint64_t stash_queue_cap(uint64_t n) { return n / 16 + 1024; }

// Batches from this size on hand ops on to a third pass (Defer::sq).  The extra launch costs a
// few microseconds, which a stream of small mixed batches (2^10..2^20 ops) pays thousands of
// times: measured there, it lowered the plain batched workload from 3.0 to 2.6 G ops/s.
constexpr uint64_t kHandOnMinOps = 1ull << 21;

// The queue of a batch of n ops: n indices and, for bulk inserts (with_kv), n packed kv words
// and the third-pass queue (stash_queue_cap(n) indices and kv words), used for n >= kHandOnMinOps.
int prepare_defer(hive_table* h, uint64_t n, cudaStream_t s, Defer* d, bool with_kv = false) {
    *d = Defer{nullptr, h->scratch + 1};
    if (n > 0xFFFFFFFFull) return HIVE_OK;
    const auto layout = [](uint64_t cap, size_t* kv, size_t* sq, size_t* skv, size_t* total) {
        const uint64_t sc = stash_queue_cap(cap);
        *kv = align256((size_t)cap * 4);
        *sq = align256(*kv + (size_t)cap * 8);
        *skv = align256(*sq + (size_t)sc * 4);
        *total = *skv + (size_t)sc * 8;
    };
    size_t okv, osq, oskv, total;
    if (n > h->defer_cap) {
        HIVE_CUDA(cudaDeviceSynchronize());
        if (h->defer_q) cudaFree(h->defer_q);
        h->defer_q = nullptr;
        h->defer_cap = 0;
        layout(n, &okv, &osq, &oskv, &total);
        cudaError_t e = cudaMalloc(&h->defer_q, total);
        if (e != cudaSuccess) return cuda_fail(e);
        h->defer_cap = n;
    }
    HIVE_CUDA(cudaMemsetAsync(h->scratch + 1, 0, 8, s));
    d->q = h->defer_q;
    if (with_kv) {
        layout(h->defer_cap, &okv, &osq, &oskv, &total);
        char* base = (char*)h->defer_q;
        d->kv = (u64*)(base + okv);
        if (n >= kHandOnMinOps) {
            d->sq = (uint32_t*)(base + osq);
            d->skv = (u64*)(base + oskv);
            d->sn = h->scratch + 6;
            d->scap = stash_queue_cap(h->defer_cap);
            HIVE_CUDA(cudaMemsetAsync(d->sn, 0, 8, s));
        }
    }
    return HIVE_OK;
}

unsigned second_pass_grid(const hive_table* h, uint64_t n) {
    return (unsigned)std::min<uint64_t>(grid_for(n), (uint64_t)h->num_sms * h->tune[HIVE_TUNE_SECOND_PASS_BLOCKS]);
}

// Region ordering pays off when the batch touches each bucket about once or more and the table
// is well beyond what stays in L2 anyway.
constexpr uint64_t kRegionMinBuckets = 1ull << 17;  // 8 MiB of slots

struct Regions {
    int rshift = 0, nreg = 0, nsub = 1;
    uint32_t *rkeys = nullptr, *rvals = nullptr, *ridx = nullptr, *counts = nullptr, *cursors = nullptr;
    uint8_t* rst = nullptr;
};

// A bulk insert runs binned (HIVE_TUNE_BINNED: 0 never, 1 (default) for batches of at least 2^20
// ops and one op per bucket into a table whose slots span at least three times the L2, 2 whenever
// allowed) into a table without holes or a split in progress, with the tag words rebuilt after
// the batch (or unused), and at most kMaxBins bins.  Where much of the table stays in L2 the
// unbinned insert's random accesses are served there and the partition passes do not pay:
// binned 0.44 ms against 0.27 ms at 2^22 slots (32 MiB), 1.89 against 1.62 ms at 2^25 (256 MiB,
// twice the L2).
// Measured at 2^26 slots, LF 0.9 (60.4 M ops): 2.89 ms against 3.26 ms unbinned, 124 against 183
// DRAM bytes per op.  The histogram and the two partition passes take 0.91 ms, the H0 and H1
// stages about 1.0 ms where the unbinned first pass takes about 2.6 ms, and the locked passes
// more than the unbinned insert's: with every H0 claim first, 2.9 M ops reach them instead of
// 2.4 M, and they evict from H1 before the stash.
bool use_bins(const hive_table* h, uint64_t n, const hive::Table& tv) {
    const int64_t m = h->tune[HIVE_TUNE_BINNED];
    const uint64_t nb = num_buckets(h);
    if (!m || n > 0xFFFFFFFFull || h->t.split || (tv.flags & hive::kFlagHoles) || !(tv.flags & hive::kFlagUntagged))
        return false;
    if ((nb + kBinBuckets - 1) >> kBinShift > kMaxBins) return false;
    return m == 2 || (n >= kBinMinOps && n >= nb && nb * hive::kSlots * 8 >= 3ull * (uint64_t)h->l2_bytes);
}

// Buffers of a binned insert of n ops; they grow (synchronously) to the largest batch seen.
int prepare_bins(hive_table* h, uint64_t n, cudaStream_t s, Bins* b) {
    b->nbins = (uint32_t)((num_buckets(h) + kBinBuckets - 1) >> kBinShift);
    b->nsupers = (b->nbins + kSuperBins - 1) / kSuperBins;
    const auto layout = [](uint64_t cap, size_t off[7], size_t* total) {
        const uint64_t max_tiles = cap / kPartTile + kMaxSupers + 1;
        off[0] = 0;                                                 // akv (and okv)
        off[1] = align256(off[0] + (size_t)cap * 8);                // rkv
        off[2] = align256(off[1] + (size_t)cap * 8);                // aidx (and oidx)
        off[3] = align256(off[2] + (size_t)cap * 4);                // ridx
        off[4] = align256(off[3] + (size_t)cap * 4);                // tiles
        off[5] = align256(off[4] + (size_t)max_tiles * 16);         // ntiles, counts, starts, cursors, ocnt
        *total = off[5] + 256 + (size_t)(4 * kMaxBins + 1 + kMaxSupers) * 4;
        return (uint32_t)max_tiles;
    };
    size_t off[7], total;
    if (n > h->bcap) {
        HIVE_CUDA(cudaDeviceSynchronize());
        if (h->bbuf) cudaFree(h->bbuf);
        h->bbuf = nullptr;
        h->bcap = 0;
        layout(n, off, &total);
        cudaError_t e = cudaMalloc(&h->bbuf, total);
        if (e != cudaSuccess) return cuda_fail(e);
        h->bcap = n;
    }
    b->max_tiles = layout(h->bcap, off, &total);
    char* p = (char*)h->bbuf;
    b->akv = b->okv = (u64*)(p + off[0]);
    b->rkv = (u64*)(p + off[1]);
    b->aidx = b->oidx = (uint32_t*)(p + off[2]);
    b->ridx = (uint32_t*)(p + off[3]);
    b->tiles = (uint4*)(p + off[4]);
    b->ntiles = (uint32_t*)(p + off[5]);
    b->counts = (uint32_t*)(p + off[5] + 256);
    b->starts = b->counts + kMaxBins;       // kMaxBins + 1 words
    b->bincur = b->starts + kMaxBins + 1;
    b->ocnt = b->bincur + kMaxBins;
    b->supcur = b->ocnt + kMaxBins;
    HIVE_CUDA(cudaMemsetAsync(b->counts, 0, (size_t)b->nbins * 4, s));
    return HIVE_OK;
}

// The binned insert's launches up to the deferred queue (histogram, scan, the two partition
// passes, the H0 stage per bin, the H1 stage per bin); the locked passes and the tag rebuild
// follow as for the unbinned insert.
template <int P>
int bin_passes(hive_table* h, const hive::Table& t, const Bins& b, const Defer& d, const uint32_t* keys,
               const uint32_t* vals, uint64_t n, uint8_t* status, cudaStream_t s) {
    static_assert((size_t)kMaxBins * 4 <= 64 * 1024, "the histogram fits 64 KiB");
    static_assert(kMaxSupers <= 1024 && kMaxPartDigits <= kBinBlock, "one thread per destination");
    static_assert(kPartTile < (1u << 16) && kMaxPartDigits <= 256, "rank and destination pack into an int");
    const unsigned hist_tiles = (unsigned)((n + kHistTile - 1) / kHistTile);
    const unsigned part_tiles = (unsigned)((n + kPartTile - 1) / kPartTile);
    const size_t hist_bytes = (size_t)b.nbins * 4;
    const size_t slab_bytes = (size_t)kBinBuckets * hive::kSlots * 8;
    const size_t part_bytes = sizeof(PartSmem);
    HIVE_CUDA(cudaFuncSetAttribute(k_bin_count<P>, cudaFuncAttributeMaxDynamicSharedMemorySize, 64 * 1024));
    HIVE_CUDA(cudaFuncSetAttribute(k_bin_part_super<P>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)part_bytes));
    HIVE_CUDA(cudaFuncSetAttribute(k_bin_part_bin<P>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)part_bytes));
    HIVE_CUDA(cudaFuncSetAttribute(k_bin_h0<P>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)slab_bytes));
    k_bin_count<P><<<hist_tiles, kBinBlock, hist_bytes, s>>>(t, keys, n, b.nbins, b.counts);
    k_bin_scan<<<1, 1024, 0, s>>>(b);
    k_bin_part_super<P><<<part_tiles, kBinBlock, part_bytes, s>>>(t, keys, vals, n, b, status);
    k_bin_part_bin<P><<<b.max_tiles, kBinBlock, part_bytes, s>>>(t, b);
    k_bin_h0<P><<<b.nbins, kBinBlock, slab_bytes, s>>>(t, b, status, d);
    k_bin_h1<P><<<b.nbins, kBlock, 0, s>>>(t, b, status, d);
    return launch_check();
}

// `knob` = HIVE_TUNE_REGION_INSERT or HIVE_TUNE_REGION_FIND.
bool use_regions(const hive_table* h, uint64_t n, int knob) {
    const uint64_t nb = num_buckets(h);
    return h->tune[knob] && nb >= kRegionMinBuckets && n >= nb && n <= 0xFFFFFFFFull;
}

// Geometry and buffers of the region ordering for a batch of n ops; the buffers grow
// (synchronously) to the largest batch seen.
int prepare_regions(hive_table* h, uint64_t n, int nsub, cudaStream_t s, Regions* r) {
    const uint64_t nb = num_buckets(h);
    int lg = 0;
    while ((2ull << lg) <= nb) ++lg;  // floor(log2(nb))
    int sh = std::min(kMaxRegionShift, std::max(kMinRegionShift, lg - 3));
    while (((nb + (1ull << sh) - 1) >> sh) * (uint64_t)nsub > (uint64_t)kMaxRegions) ++sh;
    r->nsub = nsub;
    r->rshift = sh;
    r->nreg = (int)((nb + (1ull << sh) - 1) >> sh);
    if (n > h->rcap) {
        HIVE_CUDA(cudaDeviceSynchronize());
        if (h->rbuf) cudaFree(h->rbuf);
        h->rbuf = nullptr;
        h->rcap = 0;
        const size_t bytes = align256((size_t)n * 4) * 3 + align256((size_t)n) + 2 * kMaxRegions * 4;
        cudaError_t e = cudaMalloc(&h->rbuf, bytes);
        if (e != cudaSuccess) return cuda_fail(e);
        h->rcap = n;
    }
    char* p = (char*)h->rbuf;
    const size_t w = align256((size_t)h->rcap * 4);
    r->rkeys = (uint32_t*)p;
    r->rvals = (uint32_t*)(p + w);
    r->ridx = (uint32_t*)(p + 2 * w);
    r->rst = (uint8_t*)(p + 3 * w);
    r->counts = (uint32_t*)(p + 3 * w + align256((size_t)h->rcap));
    r->cursors = r->counts + kMaxRegions;
    HIVE_CUDA(cudaMemsetAsync(r->counts, 0, (size_t)r->nreg * r->nsub * 4, s));
    return HIVE_OK;
}

// Sub-batches for a region-ordered insert of n ops: more when the batch adds a larger share of
// the table's capacity (see region_bin).
int insert_subbatches(const hive_table* h, uint64_t n) {
    if (h->tune[HIVE_TUNE_SUBBATCHES]) return (int)h->tune[HIVE_TUNE_SUBBATCHES];
    const double share = (double)n / (double)(num_buckets(h) * hive::kSlots);
    return share <= 0.25 ? 1 : share <= 0.5 ? 2 : share <= 0.75 ? 4 : 8;
}

// Counting sort of (key[, value], index) by region into r's buffers.
int region_sort(hive_table* h, const uint32_t* keys, const uint32_t* vals, uint64_t n, const Regions& r,
                cudaStream_t s) {
    const unsigned g = (unsigned)((n + kRegionTile - 1) / kRegionTile);
    if (h->policy == HIVE_POLICY_MURMURCITYHASH)
        k_region_hist<1><<<g, kBlock, 0, s>>>(h->t, keys, n, r.nreg, r.rshift, r.nsub, r.counts);
    else
        k_region_hist<0><<<g, kBlock, 0, s>>>(h->t, keys, n, r.nreg, r.rshift, r.nsub, r.counts);
    k_region_scan<<<1, kMaxRegions, 0, s>>>(r.counts, r.nreg * r.nsub, r.cursors);
    uint32_t* rv = vals ? r.rvals : nullptr;
    if (h->policy == HIVE_POLICY_MURMURCITYHASH)
        k_region_scatter<1><<<g, kBlock, 0, s>>>(h->t, keys, vals, n, r.nreg, r.rshift, r.nsub, r.cursors, r.rkeys, rv,
                                                 r.ridx);
    else
        k_region_scatter<0><<<g, kBlock, 0, s>>>(h->t, keys, vals, n, r.nreg, r.rshift, r.nsub, r.cursors, r.rkeys, rv,
                                                 r.ridx);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? HIVE_OK : cuda_fail(e);
}

int grow_capacity(hive_table* h, uint64_t need_buckets, cudaStream_t s) {
    if (need_buckets <= h->nb_cap) return HIVE_OK;
    uint64_t nb_cap = std::max<uint64_t>(need_buckets, h->nb_cap * 2);
    if (nb_cap > 0xFFFFFFFFull) nb_cap = 0xFFFFFFFFull;
    if (need_buckets > nb_cap) return HIVE_ERR_CAPACITY;
    Carve c = carve(nb_cap), oc = carve(h->nb_cap);
    void* nblock = nullptr;
    HIVE_CUDA(cudaStreamSynchronize(s));
    cudaError_t e = cudaMalloc(&nblock, c.total);
    if (e != cudaSuccess) return cuda_fail(e);
    char *nbase = (char*)nblock, *obase = (char*)h->block;
    const uint64_t nb = num_buckets(h);
    const size_t owords = (size_t)((h->nb_cap + 31) / 32);
    if ((e = cudaMemsetAsync(nblock, 0, c.total, s)) != cudaSuccess ||
        (e = cudaMemcpyAsync(nbase + c.slots, obase + oc.slots, (size_t)nb * 64, cudaMemcpyDeviceToDevice, s)) !=
            cudaSuccess ||
        (e = cudaMemcpyAsync(nbase + c.stash, obase + oc.stash, (size_t)nb * 64, cudaMemcpyDeviceToDevice, s)) !=
            cudaSuccess ||
        (e = cudaMemcpyAsync(nbase + c.sbits, obase + oc.sbits, owords * 4, cudaMemcpyDeviceToDevice, s)) !=
            cudaSuccess ||
        (e = cudaMemcpyAsync(nbase + c.fbits, obase + oc.fbits, owords * 4, cudaMemcpyDeviceToDevice, s)) !=
            cudaSuccess ||
        (e = cudaMemcpyAsync(nbase + c.ctr, obase + oc.ctr, kCounterBytes, cudaMemcpyDeviceToDevice, s)) !=
            cudaSuccess ||
        (e = cudaMemcpyAsync(nbase + c.tags, obase + oc.tags, (size_t)nb * 8, cudaMemcpyDeviceToDevice, s)) !=
            cudaSuccess ||
        (e = cudaStreamSynchronize(s)) != cudaSuccess) {
        cudaFree(nblock);
        return cuda_fail(e);
    }
    cudaFree(h->block);
    bind_arrays(h, nblock, nb_cap);
    return HIVE_OK;
}

template <int P>
int split_range(hive_table* h, uint32_t cnt, cudaStream_t s) {
    hive::Table told = h->t;
    const uint32_t sp = h->t.split;
    hive::Table tnew = told;
    tnew.split = sp + cnt;
    k_split<P><<<(cnt + 127) / 128, 128, 0, s>>>(told, tnew, sp, cnt);
    int rc = launch_check();
    if (rc) return rc;
    if (sp + cnt == h->t.n_lo) set_geometry(h, h->level + 1, 0);
    else set_geometry(h, h->level, sp + cnt);
    return HIVE_OK;
}

// Buckets folded per merge step: bounds the overflow buffer (16 entries per folded bucket: its 8
// slots and 8 stash entries) at 128 MiB, allocated once and kept by the table.
constexpr uint32_t kMergeStep = 1u << 20;

template <int P>
int merge_range(hive_table* h, uint32_t cnt, cudaStream_t s) {
    // Fold buckets [split - cnt, split) + n_lo back into [split - cnt, split).
    hive::Table told = h->t;
    const uint32_t lo = h->t.split - cnt;
    hive::Table tnew = told;
    tnew.split = lo;
    const size_t ovf_cap = (size_t)cnt * 16 + 1;
    if (ovf_cap > h->ovf_cap) {
        HIVE_CUDA(cudaStreamSynchronize(s));
        if (h->ovf) cudaFree(h->ovf);
        h->ovf = nullptr;
        h->ovf_cap = 0;
        cudaError_t e = cudaMalloc(&h->ovf, ovf_cap * 8 + 16);
        if (e != cudaSuccess) return cuda_fail(e);
        h->ovf_cap = ovf_cap;
    }
    u64* ovf = (u64*)h->ovf;
    u64* novf = ovf + ovf_cap;
    uint8_t* fail = (uint8_t*)(novf + 1);
    HIVE_CUDA(cudaMemsetAsync(novf, 0, 16, s));
    k_merge<P><<<(cnt + 127) / 128, 128, 0, s>>>(told, tnew, lo, cnt, ovf, novf);
    int rc = launch_check();
    if (rc) return rc;
    h->t.split = lo;
    tnew.flags |= hive::kFlagHoles;
    if (!h->tags_valid) tnew.flags |= hive::kFlagUntagged;  // stale words are neither read nor kept
    k_reinsert<P><<<(unsigned)((ovf_cap + 255) / 256), 256, 0, s>>>(tnew, ovf, novf, fail);
    if ((rc = launch_check())) return rc;
    uint8_t hfail = 0;
    HIVE_CUDA(cudaMemcpyAsync(&hfail, fail, 1, cudaMemcpyDeviceToHost, s));
    HIVE_CUDA(cudaStreamSynchronize(s));
    return hfail ? HIVE_ERR_CAPACITY : HIVE_OK;
}

template <int P>
int resize_impl(hive_table* h, uint64_t target_buckets, cudaStream_t s) {
    h->t.flags |= hive::kFlagHoles;
    int rc = HIVE_OK;
    while (num_buckets(h) < target_buckets) {
        const uint64_t need = target_buckets - num_buckets(h);
        const uint32_t cnt = (uint32_t)std::min<uint64_t>(need, h->t.n_lo - h->t.split);
        if ((rc = split_range<P>(h, cnt, s))) return rc;
    }
    while (num_buckets(h) > target_buckets) {
        if (h->t.split == 0) {
            if (h->level == 0) break;
            set_geometry(h, h->level - 1, h->t.n_lo >> 1);
        }
        const uint64_t extra = num_buckets(h) - target_buckets;
        const uint32_t cnt = (uint32_t)std::min<uint64_t>(std::min<uint64_t>(extra, h->t.split), kMergeStep);
        if ((rc = merge_range<P>(h, cnt, s))) return rc;
    }
    return HIVE_OK;
}

}  // namespace

// =============================================================================================
// C ABI
// =============================================================================================

extern "C" {

const char* hive_strerror(int status) {
    switch (status) {
        case HIVE_OK: return "ok";
        case HIVE_ERR_INVALID_ARG: return "invalid argument";
        case HIVE_ERR_CUDA: return "CUDA runtime error";
        case HIVE_ERR_OOM: return "device out of memory";
        case HIVE_ERR_LOCK_TIMEOUT: return "bucket lock wait expired inside a kernel";
        case HIVE_ERR_RETRY_LIMIT: return "CAS retry budget ran out inside a kernel";
        case HIVE_ERR_CAPACITY: return "capacity exceeded";
        case HIVE_ERR_NO_DEVICE: return "no usable CUDA device";
        case HIVE_ERR_TOO_LARGE: return "batch larger than HIVE_NOALLOC_MAX_OPS";
        default: return "unknown status";
    }
}

int hive_last_cuda_error(void) { return g_last_cuda_error; }

int hive_create(const hive_config* cfg, hive_table** out) {
    if (!cfg || !out) return HIVE_ERR_INVALID_ARG;
    *out = nullptr;
    if (cfg->policy != HIVE_POLICY_DEFAULT2HASH && cfg->policy != HIVE_POLICY_MURMURCITYHASH)
        return HIVE_ERR_INVALID_ARG;
    if (cfg->max_evictions < 0 || cfg->max_evictions > hive::kSlots || cfg->reserved != 0)
        return HIVE_ERR_INVALID_ARG;
    if (cfg->capacity_slots == 0) return HIVE_ERR_INVALID_ARG;
    const uint64_t nb = (cfg->capacity_slots + hive::kSlots - 1) / hive::kSlots;
    uint64_t nb_cap = std::max<uint64_t>(nb, (cfg->max_capacity_slots + hive::kSlots - 1) / hive::kSlots);
    if (nb > 0x7FFFFFFFull || nb_cap > 0xFFFFFFFFull) return HIVE_ERR_INVALID_ARG;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return HIVE_ERR_NO_DEVICE;
    int dev = cfg->device;
    if (dev < 0) HIVE_CUDA(cudaGetDevice(&dev));
    if (dev >= ndev) return HIVE_ERR_INVALID_ARG;
    DeviceGuard g(dev);
    if (!g.ok) return HIVE_ERR_CUDA;
    hive_table* h = new (std::nothrow) hive_table();
    if (!h) return HIVE_ERR_OOM;
    h->device = dev;
    h->policy = cfg->policy;
    h->n0 = (uint32_t)nb;
    if (cudaDeviceGetAttribute(&h->num_sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || h->num_sms < 1)
        h->num_sms = 148;
    if (cudaDeviceGetAttribute(&h->l2_bytes, cudaDevAttrL2CacheSize, dev) != cudaSuccess || h->l2_bytes < 1)
        h->l2_bytes = 126 << 20;
    Carve c = carve(nb_cap);
    void* block = nullptr;
    cudaError_t e = cudaMalloc(&block, c.total);
    if (e != cudaSuccess) {
        delete h;
        return cuda_fail(e);
    }
    e = cudaMemset(block, 0, c.total);
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e != cudaSuccess) {
        cudaFree(block);
        delete h;
        return cuda_fail(e);
    }
    bind_arrays(h, block, nb_cap);
    h->t.max_evictions = (uint32_t)cfg->max_evictions;
    h->t.stash_depth = (uint32_t)h->tune[HIVE_TUNE_STASH_DEPTH];
    h->t.flags = 0;
    set_geometry(h, 0, 0);
    *out = h;
    return HIVE_OK;
}

int hive_destroy(hive_table* h) {
    if (!h) return HIVE_ERR_INVALID_ARG;
    int rc = HIVE_OK;
    if (h->block) {
        DeviceGuard g(h->device);
        cudaError_t e = cudaFree(h->block);
        if (e != cudaSuccess) rc = cuda_fail(e);
        if (h->defer_q && (e = cudaFree(h->defer_q)) != cudaSuccess) rc = cuda_fail(e);
        if (h->rbuf && (e = cudaFree(h->rbuf)) != cudaSuccess) rc = cuda_fail(e);
        if (h->bbuf && (e = cudaFree(h->bbuf)) != cudaSuccess) rc = cuda_fail(e);
        if (h->hbuf && (e = cudaFree(h->hbuf)) != cudaSuccess) rc = cuda_fail(e);
        if (h->ovf && (e = cudaFree(h->ovf)) != cudaSuccess) rc = cuda_fail(e);
        for (cudaEvent_t ev : {h->ev_in, h->ev_out, h->ev_ins_free, h->ev_find_free})
            if (ev) cudaEventDestroy(ev);
        for (cudaStream_t st : {h->pipe_h2d, h->pipe_d2h})
            if (st) cudaStreamDestroy(st);
    }
    delete h;
    return rc;
}

int hive_clear(hive_table* h, void* stream) {
    if (!valid_table(h)) return HIVE_ERR_INVALID_ARG;
    DeviceGuard g(h->device);
    cudaStream_t s = (cudaStream_t)stream;
    int rc = reset(h, s);
    if (rc) return rc;
    set_geometry(h, 0, 0);
    h->t.flags = 0;
    h->tags_valid = true;  // zeroed words describe the empty table
    return HIVE_OK;
}

// Calls the host-side launcher fn<P>(...) for the table's policy.
#define HIVE_DISPATCH_FN(fn, ...)                                                          \
    do {                                                                                   \
        if (h->policy == HIVE_POLICY_MURMURCITYHASH) fn<1>(__VA_ARGS__);                    \
        else fn<0>(__VA_ARGS__);                                                           \
    } while (0)

#define HIVE_DISPATCH(kern, grid, block, stream, ...)                                      \
    do {                                                                                   \
        if (h->policy == HIVE_POLICY_MURMURCITYHASH) kern<1><<<grid, block, 0, stream>>>(__VA_ARGS__); \
        else kern<0><<<grid, block, 0, stream>>>(__VA_ARGS__);                             \
    } while (0)

// Launch a two-pass kernel: the first pass with deferral when the queue exists, else one pass.
// HIVE_DISPATCH_DX adds the mode bits `extra` to the holes and run-time modes (kModeUnique).
#define HIVE_DISPATCH_D(kern, d, grid, block, stream, ...) HIVE_DISPATCH_DX(kern, 0, d, grid, block, stream, __VA_ARGS__)
#define HIVE_DISPATCH_DX(kern, extra, d, grid, block, stream, ...)                          \
    do {                                                                                   \
        const bool p1_ = h->policy == HIVE_POLICY_MURMURCITYHASH;                          \
        const bool holes_ = h->t.flags & hive::kFlagHoles;                                 \
        if (d.q && !holes_) {                                                              \
            if (p1_) kern<1, true, hive::kModeMono><<<grid, block, 0, stream>>>(__VA_ARGS__);  \
            else kern<0, true, hive::kModeMono><<<grid, block, 0, stream>>>(__VA_ARGS__);      \
        } else if (d.q) {                                                                  \
            if (p1_) kern<1, true, hive::kModeHoles | (extra)><<<grid, block, 0, stream>>>(__VA_ARGS__); \
            else kern<0, true, hive::kModeHoles | (extra)><<<grid, block, 0, stream>>>(__VA_ARGS__);     \
        } else {                                                                           \
            if (p1_) kern<1, false, hive::kModeRuntime | (extra)><<<grid, block, 0, stream>>>(__VA_ARGS__); \
            else kern<0, false, hive::kModeRuntime | (extra)><<<grid, block, 0, stream>>>(__VA_ARGS__);     \
        }                                                                                  \
    } while (0)

}  // extern "C"

namespace {

// Tag upkeep of a bulk insert of n ops: per op, or none during its launches and one rebuild of
// the tag words after them (HIVE_TUNE_BULK_RETAG: 0 never, 1 when the batch holds at least one
// op per eight buckets, 2 always).  Per-op upkeep is a random L2 atomic on the tag words, which
// the insert's own dirty slot sectors push out of L2; a rebuild streams the slots once.
bool bulk_untagged(const hive_table* h, uint64_t n) {
    const int64_t m = h->tune[HIVE_TUNE_BULK_RETAG];
    return m == 2 || (m == 1 && n * 8 >= num_buckets(h));
}

// The Table copy an insert of n ops launches with, and whether the tag words must be rebuilt
// after it (*retag_after).  Without tags (use_tags false) nothing reads or keeps them.
int insert_view(hive_table* h, uint64_t n, cudaStream_t s, hive::Table* tv, bool* retag_after) {
    *retag_after = false;
    if (!use_tags(h)) {
        *tv = untagged_view(h);
        h->tags_valid = false;
        return HIVE_OK;
    }
    if (bulk_untagged(h, n)) {
        *tv = untagged_view(h);
        *retag_after = true;
        return HIVE_OK;
    }
    return table_view(h, s, tv);
}

// First pass of an insert (k_insert) over ops [lo, hi): deferring when the queue exists, with
// the mode bits kExtra on top of the table's base mode.
template <int kExtra>
void first_pass(const hive_table* h, const hive::Table& t, const Defer& d, unsigned grid, cudaStream_t s,
                const uint32_t* keys, const uint32_t* vals, uint64_t lo, uint64_t hi, uint8_t* status) {
    const bool p1 = h->policy == HIVE_POLICY_MURMURCITYHASH;
    const bool holes = t.flags & hive::kFlagHoles;
    if (d.q && !holes) {
        if (p1) k_insert<1, true, hive::kModeMono | kExtra><<<grid, kBlock, 0, s>>>(t, keys, vals, lo, hi, status, d);
        else k_insert<0, true, hive::kModeMono | kExtra><<<grid, kBlock, 0, s>>>(t, keys, vals, lo, hi, status, d);
    } else if (d.q) {
        if (p1) k_insert<1, true, hive::kModeHoles | kExtra><<<grid, kBlock, 0, s>>>(t, keys, vals, lo, hi, status, d);
        else k_insert<0, true, hive::kModeHoles | kExtra><<<grid, kBlock, 0, s>>>(t, keys, vals, lo, hi, status, d);
    } else {
        if (p1) k_insert<1, false, hive::kModeRuntime | kExtra><<<grid, kBlock, 0, s>>>(t, keys, vals, lo, hi, status, d);
        else k_insert<0, false, hive::kModeRuntime | kExtra><<<grid, kBlock, 0, s>>>(t, keys, vals, lo, hi, status, d);
    }
}

// primary: claim in H0 only in the first pass (region-ordered batches).
void launch_first_pass(const hive_table* h, const hive::Table& t, const Defer& d, uint64_t lo, uint64_t hi,
                       cudaStream_t s, const uint32_t* keys, const uint32_t* vals, uint8_t* status, bool primary) {
    const unsigned grid = grid_for(hi - lo);
    if (t.flags & hive::kFlagUntagged) {
        if (primary) first_pass<hive::kModeUntagged | hive::kModePrimary>(h, t, d, grid, s, keys, vals, lo, hi, status);
        else first_pass<hive::kModeUntagged>(h, t, d, grid, s, keys, vals, lo, hi, status);
    } else {
        if (primary) first_pass<hive::kModePrimary>(h, t, d, grid, s, keys, vals, lo, hi, status);
        else first_pass<0>(h, t, d, grid, s, keys, vals, lo, hi, status);
    }
}


}  // namespace

extern "C" {

int hive_insert(hive_table* h, const uint32_t* keys, const uint32_t* values, uint64_t n, uint8_t* status,
                void* stream) {
    if (!valid_table(h)) return HIVE_ERR_INVALID_ARG;
    if (n == 0) return HIVE_OK;
    if (!keys || !values) return HIVE_ERR_INVALID_ARG;
    DeviceGuard g(h->device);
    cudaStream_t s = (cudaStream_t)stream;
    L2Window l2w(h, s);
    Defer d;
    int rc = prepare_defer(h, n, s, &d, true);
    if (rc) return rc;
    hive::Table tt;
    bool untag;
    if ((rc = insert_view(h, n, s, &tt, &untag))) return rc;
    if (use_regions(h, n, HIVE_TUNE_REGION_INSERT)) {
        // region-ordered: sort, both passes over the sorted arrays, statuses back to caller order.
        // Knob 1: sub-batches with an H0-only first pass; knob 2: one pass claiming in H0 then H1,
        // the locked path evicting from H1 before it uses the stash.
        Regions r;
        const bool single = h->tune[HIVE_TUNE_REGION_INSERT] == 2;
        const int nsub = single ? 1 : insert_subbatches(h, n);
        hive::Table tr = tt;
        tr.flags |= single ? hive::kFlagEvictH1 : hive::kFlagPrimaryFirst;
        if ((rc = prepare_regions(h, n, nsub, s, &r)) || (rc = region_sort(h, keys, values, n, r, s))) return rc;
        for (int k = 0; k < nsub; ++k) {
            // sub-batch k holds ops i with i * nsub / n == k, i.e. [ceil(k n / nsub), ceil((k+1) n / nsub))
            const uint64_t lo = ((uint64_t)k * n + nsub - 1) / nsub, hi = ((uint64_t)(k + 1) * n + nsub - 1) / nsub;
            const uint64_t m = hi - lo;
            if (!m) continue;
            if (k && (rc = prepare_defer(h, m, s, &d, true))) return rc;
            d.permute = 1;  // the queue is in bucket order
            uint8_t* rst = status ? r.rst + lo : nullptr;
            launch_first_pass(h, tr, d, 0, m, s, r.rkeys + lo, r.rvals + lo, rst, !single);
            if (d.q)
                HIVE_DISPATCH_FN(launch_second_pass, second_pass_grid(h, m), s, tr, r.rkeys + lo, r.rvals + lo,
                                 rst, d);
        }
        if (untag) retag(h, s);
        if (status) k_unpermute_u8<<<grid_for(n), kBlock, 0, s>>>(r.ridx, r.rst, n, status);
        return launch_check();
    }
    if (d.q && use_bins(h, n, tt)) {
        Bins b;
        if ((rc = prepare_bins(h, n, s, &b))) return rc;
        if (h->policy == HIVE_POLICY_MURMURCITYHASH) rc = bin_passes<1>(h, tt, b, d, keys, values, n, status, s);
        else rc = bin_passes<0>(h, tt, b, d, keys, values, n, status, s);
        if (rc) return rc;
        // Every H1 claim came after every H0 claim, so the locked passes meet buckets that hold
        // all their primaries: they try H1's own keys as victims before the stash, which keeps
        // the stashes from overflowing (a sequential model of this placement leaves 0 of 2^24 keys
        // unplaced at LF 1.0 this way, 33 with the stash first; with the stash first, one key of
        // 2^24 slots at LF 0.9 was left unplaced on the GPU).
        tt.flags |= hive::kFlagEvictH1;
        // the deferred queue is in bin order (the H1 stage reads its queue in the order the bins
        // filled it): visited in that order, the locked passes' warps would crowd onto the locks
        // of neighbouring buckets
        d.permute = 1;
    } else {
        launch_first_pass(h, tt, d, 0, n, s, keys, values, status, false);
    }
    if (d.q) HIVE_DISPATCH_FN(launch_second_pass, second_pass_grid(h, n), s, tt, keys, values, status, d);
    if (untag) retag(h, s);
    return launch_check();
}

}  // extern "C"

// ---- hive_insert_noalloc: the second-pass queue in static device memory -------------------------
// Layout: bytes [0, 8) the queue count, [256, 256 + 4 * HIVE_NOALLOC_MAX_OPS) the op indices.
// Every device that loads this library holds the array until the process exits.  In host code
// the name g_noalloc_queue is a host-side stand-in, not a device address: a kernel given it
// would fault (or, where the GPU can reach host memory, silently use the wrong memory), so the
// device address is looked up per device with cudaGetSymbolAddress and cached.
namespace {
constexpr size_t kNoAllocHeaderWords = 64;  // 256 bytes
static __device__ __align__(256) uint32_t g_noalloc_queue[kNoAllocHeaderWords + HIVE_NOALLOC_MAX_OPS];

constexpr int kMaxDevices = 64;
void* g_noalloc_addr[kMaxDevices] = {};
std::mutex g_noalloc_mutex;

// Device address of g_noalloc_queue on the current device (dev), looked up once per device.
int noalloc_queue(int dev, uint32_t** out) {
    if (dev < 0 || dev >= kMaxDevices) return HIVE_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (!g_noalloc_addr[dev]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_queue);
        if (e != cudaSuccess) return cuda_fail(e);
        g_noalloc_addr[dev] = p;
    }
    *out = (uint32_t*)g_noalloc_addr[dev];
    return HIVE_OK;
}
}  // namespace

extern "C" {

int hive_insert_noalloc(hive_table* h, const uint32_t* keys, const uint32_t* values, uint64_t n, uint8_t* status,
                        void* stream) {
    if (!valid_table(h)) return HIVE_ERR_INVALID_ARG;
    if (n > HIVE_NOALLOC_MAX_OPS) return HIVE_ERR_TOO_LARGE;
    if (n == 0) return HIVE_OK;
    if (!keys || !values) return HIVE_ERR_INVALID_ARG;
    DeviceGuard g(h->device);
    if (!g.ok) return HIVE_ERR_CUDA;
    uint32_t* base = nullptr;
    int rc = noalloc_queue(h->device, &base);
    if (rc) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    Defer d{base + kNoAllocHeaderWords, (u64*)base};
    HIVE_CUDA(cudaMemsetAsync(d.n, 0, sizeof(u64), s));  // the queue count must start at zero
    hive::Table tt;
    bool untag;
    if ((rc = insert_view(h, n, s, &tt, &untag))) return rc;
    launch_first_pass(h, tt, d, 0, n, s, keys, values, status, false);
    HIVE_DISPATCH_FN(launch_second_pass, second_pass_grid(h, n), s, tt, keys, values, status, d);
    if (untag) retag(h, s);
    return launch_check();
}

int hive_find(hive_table* h, const uint32_t* keys, uint64_t n, uint32_t* values, uint8_t* found, void* stream) {
    if (!valid_table(h)) return HIVE_ERR_INVALID_ARG;
    if (n == 0) return HIVE_OK;
    if (!keys) return HIVE_ERR_INVALID_ARG;
    DeviceGuard g(h->device);
    cudaStream_t s = (cudaStream_t)stream;
    L2Window l2w(h, s);
    hive::Table tv;
    if (int vrc = table_view(h, s, &tv)) return vrc;
    if (use_regions(h, n, HIVE_TUNE_REGION_FIND)) {
        Regions r;
        int rc;
        if ((rc = prepare_regions(h, n, 1, s, &r)) || (rc = region_sort(h, keys, nullptr, n, r, s))) return rc;
        HIVE_DISPATCH(k_find, grid_for(n), kBlock, s, tv, r.rkeys, n, r.rvals, r.rst);
        k_unpermute_find<<<grid_for(n), kBlock, 0, s>>>(r.ridx, r.rvals, r.rst, n, values, found);
        return launch_check();
    }
    HIVE_DISPATCH(k_find, grid_for(n), kBlock, s, tv, keys, n, values, found);
    return launch_check();
}

}  // extern "C"

// ---- host-buffer pipeline ------------------------------------------------------------------------
// A batch in host memory is copied in chunks on a copy stream and each chunk is processed on the
// caller's stream as soon as it has landed, so PCIe transfers overlap the table work; results go
// back on a second copy stream (PCIe is full duplex).  The caller's stream waits for the last
// copy, so synchronising it covers the whole call.  The device staging arrays of a kind (insert
// or find) are reused by the next call of that kind only after this call has finished with them
// (ev_ins_free / ev_find_free), which lets a find's key upload run while an insert is computing.
namespace {
constexpr uint64_t kPipeChunk = 1ull << 22;  // ops per chunk: 16 MiB of keys

struct Staging {
    uint32_t *ik, *iv, *fk, *fv;
    uint8_t *ist, *ff;
};

int prepare_pipe(hive_table* h, uint64_t n, Staging* st) {
    if (!h->pipe_h2d) {
        HIVE_CUDA(cudaStreamCreateWithFlags(&h->pipe_h2d, cudaStreamNonBlocking));
        HIVE_CUDA(cudaStreamCreateWithFlags(&h->pipe_d2h, cudaStreamNonBlocking));
        for (cudaEvent_t* ev : {&h->ev_in, &h->ev_out, &h->ev_ins_free, &h->ev_find_free})
            HIVE_CUDA(cudaEventCreateWithFlags(ev, cudaEventDisableTiming));
    }
    if (n > h->hcap) {
        HIVE_CUDA(cudaDeviceSynchronize());
        if (h->hbuf) cudaFree(h->hbuf);
        h->hbuf = nullptr;
        h->hcap = 0;
        cudaError_t e = cudaMalloc(&h->hbuf, align256((size_t)n * 4) * 4 + align256((size_t)n) * 2);
        if (e != cudaSuccess) return cuda_fail(e);
        h->hcap = n;
    }
    const size_t w = align256((size_t)h->hcap * 4), b = align256((size_t)h->hcap);
    char* p = (char*)h->hbuf;
    st->ik = (uint32_t*)p;
    st->iv = (uint32_t*)(p + w);
    st->fk = (uint32_t*)(p + 2 * w);
    st->fv = (uint32_t*)(p + 3 * w);
    st->ist = (uint8_t*)(p + 4 * w);
    st->ff = (uint8_t*)(p + 4 * w + b);
    return HIVE_OK;
}

// `after` waits for everything issued so far on `before`.
cudaError_t order(cudaEvent_t ev, cudaStream_t before, cudaStream_t after) {
    cudaError_t e = cudaEventRecord(ev, before);
    return e == cudaSuccess ? cudaStreamWaitEvent(after, ev, 0) : e;
}
}  // namespace

extern "C" {

int hive_insert_host(hive_table* h, const uint32_t* keys, const uint32_t* values, uint64_t n, uint8_t* status,
                     void* stream) {
    if (!valid_table(h)) return HIVE_ERR_INVALID_ARG;
    if (n == 0) return HIVE_OK;
    if (!keys || !values) return HIVE_ERR_INVALID_ARG;
    DeviceGuard g(h->device);
    if (!g.ok) return HIVE_ERR_CUDA;
    cudaStream_t s = (cudaStream_t)stream;
    L2Window l2w(h, s);
    Staging st;
    Defer d;
    int rc;
    if ((rc = prepare_pipe(h, n, &st)) || (rc = prepare_defer(h, n, s, &d, true))) return rc;
    HIVE_CUDA(cudaStreamWaitEvent(h->pipe_h2d, h->ev_ins_free, 0));
    uint8_t* dst = status ? st.ist : nullptr;
    hive::Table tt;
    bool untag;
    if ((rc = insert_view(h, n, s, &tt, &untag))) return rc;
    for (uint64_t lo = 0; lo < n; lo += kPipeChunk) {
        const uint64_t m = std::min(kPipeChunk, n - lo);
        HIVE_CUDA(cudaMemcpyAsync(st.ik + lo, keys + lo, m * 4, cudaMemcpyHostToDevice, h->pipe_h2d));
        HIVE_CUDA(cudaMemcpyAsync(st.iv + lo, values + lo, m * 4, cudaMemcpyHostToDevice, h->pipe_h2d));
        HIVE_CUDA(order(h->ev_in, h->pipe_h2d, s));
        // first pass of this chunk; its deferred ops join the batch's one queue
        launch_first_pass(h, tt, d, lo, lo + m, s, st.ik, st.iv, dst, false);
    }
    if (d.q) HIVE_DISPATCH_FN(launch_second_pass, second_pass_grid(h, n), s, tt, st.ik, st.iv, dst, d);
    if (untag) retag(h, s);
    if (status) {
        HIVE_CUDA(order(h->ev_out, s, h->pipe_d2h));
        HIVE_CUDA(cudaMemcpyAsync(status, st.ist, n, cudaMemcpyDeviceToHost, h->pipe_d2h));
        HIVE_CUDA(order(h->ev_out, h->pipe_d2h, s));
    }
    HIVE_CUDA(cudaEventRecord(h->ev_ins_free, s));
    return launch_check();
}

int hive_find_host(hive_table* h, const uint32_t* keys, uint64_t n, uint32_t* values, uint8_t* found, void* stream) {
    if (!valid_table(h)) return HIVE_ERR_INVALID_ARG;
    if (n == 0) return HIVE_OK;
    if (!keys) return HIVE_ERR_INVALID_ARG;
    DeviceGuard g(h->device);
    if (!g.ok) return HIVE_ERR_CUDA;
    cudaStream_t s = (cudaStream_t)stream;
    L2Window l2w(h, s);
    Staging st;
    int rc = prepare_pipe(h, n, &st);
    if (rc) return rc;
    hive::Table tv;
    if (int vrc = table_view(h, s, &tv)) return vrc;
    HIVE_CUDA(cudaStreamWaitEvent(h->pipe_h2d, h->ev_find_free, 0));
    for (uint64_t lo = 0; lo < n; lo += kPipeChunk) {
        const uint64_t m = std::min(kPipeChunk, n - lo);
        HIVE_CUDA(cudaMemcpyAsync(st.fk + lo, keys + lo, m * 4, cudaMemcpyHostToDevice, h->pipe_h2d));
        HIVE_CUDA(order(h->ev_in, h->pipe_h2d, s));
        HIVE_DISPATCH(k_find, grid_for(m), kBlock, s, tv, st.fk + lo, m, st.fv + lo, st.ff + lo);
        if (values || found) HIVE_CUDA(order(h->ev_out, s, h->pipe_d2h));
        if (values) HIVE_CUDA(cudaMemcpyAsync(values + lo, st.fv + lo, m * 4, cudaMemcpyDeviceToHost, h->pipe_d2h));
        if (found) HIVE_CUDA(cudaMemcpyAsync(found + lo, st.ff + lo, m, cudaMemcpyDeviceToHost, h->pipe_d2h));
    }
    HIVE_CUDA(order(h->ev_out, h->pipe_d2h, s));
    HIVE_CUDA(cudaEventRecord(h->ev_find_free, s));
    return launch_check();
}

int hive_erase(hive_table* h, const uint32_t* keys, uint64_t n, uint8_t* status, void* stream) {
    if (!valid_table(h)) return HIVE_ERR_INVALID_ARG;
    if (n == 0) return HIVE_OK;
    if (!keys) return HIVE_ERR_INVALID_ARG;
    DeviceGuard g(h->device);
    h->t.flags |= hive::kFlagHoles;
    cudaStream_t s = (cudaStream_t)stream;
    L2Window l2w(h, s);
    hive::Table tv;
    if (int vrc = table_view(h, s, &tv)) return vrc;
    HIVE_DISPATCH(k_erase, grid_for(n), kBlock, s, tv, keys, n, status);
    return launch_check();
}

int hive_apply_ops(hive_table* h, const uint8_t* types, const uint32_t* keys, const uint32_t* values, uint64_t n,
                   uint8_t* status, uint32_t* out_values, uint32_t hints, void* stream) {
    if (!valid_table(h)) return HIVE_ERR_INVALID_ARG;
    if (n == 0) return HIVE_OK;
    if (!types || !keys) return HIVE_ERR_INVALID_ARG;
    DeviceGuard g(h->device);
    cudaStream_t s = (cudaStream_t)stream;
    L2Window l2w(h, s);
    if (!(hints & HIVE_HINT_NO_DELETES)) h->t.flags |= hive::kFlagHoles;
    Defer d;
    int rc = prepare_defer(h, n, s, &d, true);
    if (rc) return rc;
    hive::Table tv;
    if (int vrc = table_view(h, s, &tv)) return vrc;
    if (hints & HIVE_HINT_UNIQUE_KEYS)
        HIVE_DISPATCH_DX(k_apply, hive::kModeUnique, d, grid_for(n), kBlock, s, tv, types, keys, values, n, status,
                         out_values, d);
    else
        HIVE_DISPATCH_D(k_apply, d, grid_for(n), kBlock, s, tv, types, keys, values, n, status, out_values, d);
    // the deferred inserts: the bulk insert's second pass and the third pass over what it hands on
    if (d.q) HIVE_DISPATCH_FN(launch_second_pass, second_pass_grid(h, n), s, tv, keys, values, status, d);
    return launch_check();
}

int hive_apply_batches(hive_table* h, const uint8_t* types, const uint32_t* keys, const uint32_t* values,
                       const uint64_t* offsets, uint32_t n_batches, uint64_t max_batch_ops, uint8_t* status,
                       uint32_t* out_values, uint32_t hints, int threads_per_block, int blocks_per_sm, void* stream) {
    if (!valid_table(h)) return HIVE_ERR_INVALID_ARG;
    if (n_batches == 0) return HIVE_OK;
    if (!types || !keys || !offsets || max_batch_ops == 0 || max_batch_ops > 0xFFFFFFFFull) return HIVE_ERR_INVALID_ARG;
    if (threads_per_block <= 0) threads_per_block = kBlock;
    if (threads_per_block % 32 || threads_per_block > 1024 || blocks_per_sm < 0) return HIVE_ERR_INVALID_ARG;
    DeviceGuard g(h->device);
    cudaStream_t s = (cudaStream_t)stream;
    L2Window l2w(h, s);
    if (!(hints & HIVE_HINT_NO_DELETES)) h->t.flags |= hive::kFlagHoles;
    Defer d;
    int rc = prepare_defer(h, max_batch_ops, s, &d);
    if (rc) return rc;
    if (!d.q) return HIVE_ERR_INVALID_ARG;
    hive::Table tv;
    if (int vrc = table_view(h, s, &tv)) return vrc;
    HIVE_CUDA(cudaMemsetAsync(h->scratch, 0, 16, s));  // both alternating queue counts
    const bool holes = h->t.flags & hive::kFlagHoles;
    const bool p1 = h->policy == HIVE_POLICY_MURMURCITYHASH;
    const bool uniq = hints & HIVE_HINT_UNIQUE_KEYS;
    constexpr int kHU = hive::kModeHoles | hive::kModeUnique;
    const void* fn = p1 ? (holes ? (uniq ? (const void*)k_apply_batches<1, kHU> : (const void*)k_apply_batches<1, hive::kModeHoles>)
                                 : (const void*)k_apply_batches<1, hive::kModeMono>)
                        : (holes ? (uniq ? (const void*)k_apply_batches<0, kHU> : (const void*)k_apply_batches<0, hive::kModeHoles>)
                                 : (const void*)k_apply_batches<0, hive::kModeMono>);
    int fit = 0;
    HIVE_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&fit, fn, threads_per_block, 0));
    if (fit < 1) return HIVE_ERR_INVALID_ARG;
    const int per_sm = blocks_per_sm > 0 ? std::min(blocks_per_sm, fit) : fit;
    dim3 grid((unsigned)(per_sm * h->num_sms)), block((unsigned)threads_per_block);
    u64* qn = h->scratch;  // two counts: scratch[0], scratch[1]
    void* args[] = {(void*)&tv, (void*)&types, (void*)&keys, (void*)&values, (void*)&offsets, (void*)&n_batches,
                    (void*)&status, (void*)&out_values, (void*)&d.q, (void*)&qn};
    HIVE_CUDA(cudaLaunchCooperativeKernel(fn, grid, block, args, 0, s));
    return HIVE_OK;
}

int hive_apply_ops_split(hive_table* h, const uint8_t* types, const uint32_t* keys, const uint32_t* values,
                         uint64_t n, uint8_t* status, uint32_t* out_values, uint32_t hints, uint64_t split_buckets,
                         void* stream) {
    if (!valid_table(h)) return HIVE_ERR_INVALID_ARG;
    if (n && (!types || !keys)) return HIVE_ERR_INVALID_ARG;
    if (n > 0xFFFFFFFFull) return HIVE_ERR_INVALID_ARG;
    DeviceGuard g(h->device);
    if (!g.ok) return HIVE_ERR_CUDA;
    cudaStream_t s = (cudaStream_t)stream;
    L2Window l2w(h, s);
    const uint32_t sp = h->t.split, nlo = h->t.n_lo;
    const uint32_t w = (uint32_t)std::min<uint64_t>(split_buckets, (uint64_t)(nlo - sp));
    if (w == 0) return n ? hive_apply_ops(h, types, keys, values, n, status, out_values, hints, stream) : HIVE_OK;
    int rc = grow_capacity(h, (uint64_t)nlo + sp + w, s);
    if (rc) return rc;
    h->t.flags |= hive::kFlagHoles;  // entries leave their buckets
    Defer d;
    if ((rc = prepare_defer(h, std::max<uint64_t>(n, 1), s, &d))) return rc;
    hive::Table tv;
    if ((rc = table_view(h, s, &tv))) return rc;
    hive::Table tmig = tv, tnew = tv;
    tmig.flags |= hive::kFlagMigrating;
    tmig.win_end = sp + w;
    tnew.split = sp + w;  // split == n_lo addresses exactly as the next level with split 0
    HIVE_CUDA(cudaMemsetAsync(d.n, 0, 8, s));
    const bool p1 = h->policy == HIVE_POLICY_MURMURCITYHASH;
    const bool uniq = hints & HIVE_HINT_UNIQUE_KEYS;
    constexpr int kHU = hive::kModeHoles | hive::kModeUnique;
    const void* fn = p1 ? (uniq ? (const void*)k_apply_split<1, kHU> : (const void*)k_apply_split<1, hive::kModeHoles>)
                        : (uniq ? (const void*)k_apply_split<0, kHU> : (const void*)k_apply_split<0, hive::kModeHoles>);
    int fit = 0;
    HIVE_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&fit, fn, kBlock, 0));
    if (fit < 1) return HIVE_ERR_INVALID_ARG;
    dim3 grid((unsigned)(fit * h->num_sms)), block((unsigned)kBlock);
    void* args[] = {(void*)&tmig, (void*)&tnew, (void*)&types, (void*)&keys, (void*)&values, (void*)&n,
                    (void*)&status, (void*)&out_values, (void*)&d.q, (void*)&d.n};
    HIVE_CUDA(cudaLaunchCooperativeKernel(fn, grid, block, args, 0, s));
    if (sp + w == nlo) set_geometry(h, h->level + 1, 0);
    else set_geometry(h, h->level, sp + w);
    return HIVE_OK;
}

int hive_apply_reference_ops(hive_table* h, const void* ops, uint64_t n, uint64_t* results, uint32_t hints,
                             void* stream) {
    if (!valid_table(h)) return HIVE_ERR_INVALID_ARG;
    if (n == 0) return HIVE_OK;
    if (!ops || ((uintptr_t)ops & 15)) return HIVE_ERR_INVALID_ARG;
    DeviceGuard g(h->device);
    cudaStream_t s = (cudaStream_t)stream;
    L2Window l2w(h, s);
    // the holes flag first: the launch's view carries the flags
    if (!(hints & (HIVE_HINT_LOOKUPS_ONLY | HIVE_HINT_NO_DELETES))) h->t.flags |= hive::kFlagHoles;
    hive::Table tv;
    if (int vrc = table_view(h, s, &tv)) return vrc;
    if (hints & HIVE_HINT_LOOKUPS_ONLY) {
        HIVE_DISPATCH(k_apply_ref_ro, grid_for(n), kBlock, s, tv, (const ulonglong2*)ops, n,
                      (unsigned long long*)results);
        return launch_check();
    }
    Defer d;
    int rc = prepare_defer(h, n, s, &d);
    if (rc) return rc;
    if (hints & HIVE_HINT_UNIQUE_KEYS)
        HIVE_DISPATCH_DX(k_apply_ref, hive::kModeUnique, d, grid_for(n), kBlock, s, tv, (const ulonglong2*)ops, n,
                         (unsigned long long*)results, d);
    else
        HIVE_DISPATCH_D(k_apply_ref, d, grid_for(n), kBlock, s, tv, (const ulonglong2*)ops, n,
                        (unsigned long long*)results, d);
    if (d.q)
        HIVE_DISPATCH(k_apply_ref_deferred, second_pass_grid(h, n), kBlock, s, tv, (const ulonglong2*)ops,
                      (unsigned long long*)results, d);
    return launch_check();
}

int hive_size(hive_table* h, uint64_t* n_out, void* stream) {
    if (!valid_table(h) || !n_out) return HIVE_ERR_INVALID_ARG;
    DeviceGuard g(h->device);
    cudaStream_t s = (cudaStream_t)stream;
    const uint64_t nb = num_buckets(h);
    HIVE_CUDA(cudaMemsetAsync(h->scratch, 0, 8, s));
    k_count<<<grid_for(nb), kBlock, 0, s>>>(h->t, nb, h->scratch);
    int rc = launch_check();
    if (rc) return rc;
    u64 v = 0;
    HIVE_CUDA(cudaMemcpyAsync(&v, h->scratch, 8, cudaMemcpyDeviceToHost, s));
    HIVE_CUDA(cudaStreamSynchronize(s));
    *n_out = v;
    return HIVE_OK;
}

int hive_dump(hive_table* h, uint64_t* kv, uint64_t cap, uint64_t* n_out, void* stream) {
    if (!valid_table(h) || !n_out || (cap && !kv)) return HIVE_ERR_INVALID_ARG;
    DeviceGuard g(h->device);
    cudaStream_t s = (cudaStream_t)stream;
    const uint64_t nb = num_buckets(h);
    HIVE_CUDA(cudaMemsetAsync(h->scratch, 0, 8, s));
    k_dump<<<grid_for(nb), kBlock, 0, s>>>(h->t, nb, (u64*)kv, cap, h->scratch);
    int rc = launch_check();
    if (rc) return rc;
    u64 v = 0;
    HIVE_CUDA(cudaMemcpyAsync(&v, h->scratch, 8, cudaMemcpyDeviceToHost, s));
    HIVE_CUDA(cudaStreamSynchronize(s));
    *n_out = v;
    return HIVE_OK;
}

int hive_load(hive_table* h, const uint64_t* kv, uint64_t n, uint64_t* n_unplaced, void* stream) {
    if (!valid_table(h) || (n && !kv)) return HIVE_ERR_INVALID_ARG;
    DeviceGuard g(h->device);
    cudaStream_t s = (cudaStream_t)stream;
    if (n_unplaced) *n_unplaced = 0;
    // empty the table at its current geometry (hive_clear would also return it to level 0)
    int rc = reset(h, s);
    if (rc) return rc;
    // Mid-level, a bucket not yet split takes keys of 1/n_lo of the hash space, twice a split
    // bucket's share, so the load that bounds placement is n / (8 n_lo).  Grow (the table is
    // empty, so the split kernels move nothing) to the first full level that keeps it at
    // kMaxShrinkLoad.
    uint64_t lvl = h->t.n_lo;
    while ((double)n > kMaxShrinkLoad * (double)(lvl * hive::kSlots)) lvl *= 2;
    if (lvl > h->t.n_lo && (rc = hive_resize(h, lvl * hive::kSlots, stream))) return rc;
    h->t.flags = 0;  // an empty table has no holes, whatever resized it
    h->tags_valid = true;
    if (!n) return HIVE_OK;
    // chunks through one temporary staging area: keys, values, statuses, the unplaced count
    const uint64_t chunk = std::min<uint64_t>(n, kLoadChunk);
    const size_t w = align256((size_t)chunk * 4);
    char* tmp = nullptr;
    cudaError_t e = cudaMalloc(&tmp, 2 * w + align256((size_t)chunk) + 256);
    if (e != cudaSuccess) return e == cudaErrorMemoryAllocation ? HIVE_ERR_OOM : cuda_fail(e);
    uint32_t* keys = (uint32_t*)tmp;
    uint32_t* vals = (uint32_t*)(tmp + w);
    uint8_t* st = (uint8_t*)(tmp + 2 * w);
    u64* cnt = (u64*)(tmp + 2 * w + align256((size_t)chunk));
    u64 unplaced = 0;
    if ((e = cudaMemsetAsync(cnt, 0, 8, s)) != cudaSuccess) rc = cuda_fail(e);
    for (uint64_t off = 0; !rc && off < n; off += chunk) {
        const uint64_t m = std::min(chunk, n - off);
        k_unpack<<<grid_for(m), kBlock, 0, s>>>((const u64*)kv + off, m, keys, vals);
        if ((rc = launch_check()) || (rc = hive_insert(h, keys, vals, m, st, stream))) break;
        k_count_unplaced<<<grid_for(m), kBlock, 0, s>>>(st, m, cnt);
        rc = launch_check();
    }
    if (!rc && (e = cudaMemcpyAsync(&unplaced, cnt, 8, cudaMemcpyDeviceToHost, s)) != cudaSuccess) rc = cuda_fail(e);
    if (!rc && (e = cudaStreamSynchronize(s)) != cudaSuccess) rc = cuda_fail(e);
    // the staging area is only freed once the stream has finished with it
    if (rc) cudaStreamSynchronize(s);
    cudaFree(tmp);
    if (rc) return rc;
    if (n_unplaced) *n_unplaced = unplaced;
    if ((rc = hive_check(h, stream))) return rc;
    return unplaced ? HIVE_ERR_CAPACITY : HIVE_OK;
}

int hive_resize(hive_table* h, uint64_t target_slots, void* stream) {
    if (!valid_table(h) || target_slots == 0) return HIVE_ERR_INVALID_ARG;
    DeviceGuard g(h->device);
    cudaStream_t s = (cudaStream_t)stream;
    uint64_t target = (target_slots + hive::kSlots - 1) / hive::kSlots;
    if (target > 0xFFFFFFFFull) return HIVE_ERR_CAPACITY;
    if (target < h->n0) target = h->n0;  // never below the creation size (level 0)
    if (target < num_buckets(h)) {
        // A shrink is refused (table unchanged) unless the live entries fit the smaller table at
        // load factor <= kMaxShrinkLoad, so the merge's re-inserts cannot run out of room.  The
        // load counted is that of the target's unsplit level: mid-level, a bucket not yet split
        // takes keys of 1/n_lo of the hash space, twice a split bucket's share.
        uint64_t live = 0;
        int rc = hive_size(h, &live, stream);
        if (rc) return rc;
        uint64_t lvl = h->n0;
        while (lvl * 2 <= target) lvl *= 2;
        if ((double)live > kMaxShrinkLoad * (double)(lvl * hive::kSlots)) return HIVE_ERR_CAPACITY;
    }
    int rc = grow_capacity(h, target, s);
    if (rc) return rc;
    if (h->policy == HIVE_POLICY_MURMURCITYHASH) return resize_impl<1>(h, target, s);
    return resize_impl<0>(h, target, s);
}

int hive_bucket_of(hive_table* h, const uint32_t* keys, uint64_t n, uint32_t* b0, uint32_t* b1, void* stream) {
    if (!valid_table(h)) return HIVE_ERR_INVALID_ARG;
    if (n == 0) return HIVE_OK;
    if (!keys) return HIVE_ERR_INVALID_ARG;
    DeviceGuard g(h->device);
    HIVE_DISPATCH(k_bucket_of, grid_for(n), kBlock, (cudaStream_t)stream, h->t, keys, n, b0, b1);
    return launch_check();
}

int hive_get_info(const hive_table* h, hive_info* out) {
    if (!valid_table(h) || !out) return HIVE_ERR_INVALID_ARG;
    std::memset(out, 0, sizeof(*out));
    out->num_buckets = num_buckets(h);
    out->capacity_slots = out->num_buckets * hive::kSlots;
    out->max_buckets = h->nb_cap;
    out->base_buckets = h->n0;
    out->level = h->level;
    out->split = h->t.split;
    out->policy = h->policy;
    out->max_evictions = (int32_t)h->t.max_evictions;
    out->flags = h->t.flags;
    out->device = h->device;
    return HIVE_OK;
}

int hive_counters(hive_table* h, uint64_t* out, void* stream) {
    if (!valid_table(h) || !out) return HIVE_ERR_INVALID_ARG;
    DeviceGuard g(h->device);
    cudaStream_t s = (cudaStream_t)stream;
    uint64_t stripes[hive::kCounterStripes * hive::kCounterStride];
    HIVE_CUDA(cudaMemcpyAsync(stripes, h->t.counters, kCounterBytes, cudaMemcpyDeviceToHost, s));
    HIVE_CUDA(cudaStreamSynchronize(s));
    for (int c = 0; c < HIVE_NUM_COUNTERS; ++c) {
        uint64_t v = 0;
        for (int k = 0; k < hive::kCounterStripes; ++k)
            v = c == HIVE_CTR_ERROR ? v | stripes[k * hive::kCounterStride + c] : v + stripes[k * hive::kCounterStride + c];
        out[c] = v;
    }
    return HIVE_OK;
}

int hive_verify(hive_table* h, uint64_t* out, void* stream) {
    if (!valid_table(h) || !out) return HIVE_ERR_INVALID_ARG;
    DeviceGuard g(h->device);
    if (!g.ok) return HIVE_ERR_CUDA;
    cudaStream_t s = (cudaStream_t)stream;
    hive::Table tv;
    if (int vrc = table_view(h, s, &tv)) return vrc;
    u64* d = h->scratch + 2;  // scratch words 2..5
    HIVE_CUDA(cudaMemsetAsync(d, 0, HIVE_VERIFY_COUNT * 8, s));
    const uint64_t nb = num_buckets(h);
    HIVE_DISPATCH(k_verify, grid_for(nb), kBlock, s, tv, nb, !(h->t.flags & hive::kFlagHoles), d);
    int rc = launch_check();
    if (rc) return rc;
    HIVE_CUDA(cudaMemcpyAsync(out, d, HIVE_VERIFY_COUNT * 8, cudaMemcpyDeviceToHost, s));
    HIVE_CUDA(cudaStreamSynchronize(s));
    return HIVE_OK;
}

int hive_debug_hold_lock(hive_table* h, uint64_t bucket, int held, void* stream) {
    if (!valid_table(h) || bucket >= num_buckets(h) || (held != 0 && held != 1)) return HIVE_ERR_INVALID_ARG;
    DeviceGuard g(h->device);
    if (!g.ok) return HIVE_ERR_CUDA;
    // the lock byte of `bucket` (byte b & 3 of word b >> 2; little-endian)
    HIVE_CUDA(cudaMemsetAsync((char*)h->t.locks + bucket, held, 1, (cudaStream_t)stream));
    return HIVE_OK;
}

int hive_set_tuning(hive_table* h, int32_t key, int64_t value) {
    if (!valid_table(h) || key < 0 || key >= HIVE_NUM_TUNES) return HIVE_ERR_INVALID_ARG;
    static const int64_t lo[HIVE_NUM_TUNES] = {0, 0, 0, 1, 0, 0, 0, 1, 0},
                         hi[HIVE_NUM_TUNES] = {2, 1, 8, 8, 2, 2, 2, 8, 2};
    if (value < lo[key] || value > hi[key]) return HIVE_ERR_INVALID_ARG;
    h->tune[key] = value;
    if (key == HIVE_TUNE_STASH_DEPTH) h->t.stash_depth = (uint32_t)value;
    return HIVE_OK;
}

int hive_get_tuning(const hive_table* h, int32_t key, int64_t* value) {
    if (!valid_table(h) || !value || key < 0 || key >= HIVE_NUM_TUNES) return HIVE_ERR_INVALID_ARG;
    *value = h->tune[key];
    return HIVE_OK;
}

int hive_check(hive_table* h, void* stream) {
    uint64_t c[HIVE_NUM_COUNTERS];
    int rc = hive_counters(h, c, stream);
    if (rc) return rc;
    if (c[HIVE_CTR_ERROR] & hive::kErrLockTimeout) return HIVE_ERR_LOCK_TIMEOUT;
    if (c[HIVE_CTR_ERROR] & hive::kErrRetryOut) return HIVE_ERR_RETRY_LIMIT;
    return HIVE_OK;
}

}  // extern "C"
