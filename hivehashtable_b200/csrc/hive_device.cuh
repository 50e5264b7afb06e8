// hive_device.cuh -- device-side data layout, hash policies and per-operation protocols of the
// B200 Hive hash table.  Included only by hive_table.cu.
//
// Layout in HBM (one table):
//   slots      u64[nb_cap * 8]   8-slot buckets, 64 B each, 64 B aligned (the reference pads a
//                                bucket to 128 B, include/hive_hash_table_struct.cuh:56-59; here
//                                a bucket is exactly two 32 B sectors and one 256-bit load pair)
//   stash      u64[nb_cap * 8]   per-canonical-bucket overflow stash, 8 slots
//                                (include/hive_stash_table.cuh:20-27)
//   stash_bits u32[nb_cap / 32]  bit b set = stash of bucket b may hold entries (the reference
//                                keeps this as bit 31 of a per-bucket freeMask word,
//                                include/hive_hash_insert.cuh:512-514); 1 bit per bucket keeps
//                                it L2-resident (1 MiB at 2^23 buckets)
//   locks      u8[nb_cap]        eviction locks, one byte per bucket (the reference keeps a word
//                                per bucket, include/hive_hash_table_struct.cuh:101-117): 8 MiB
//                                at 2^23 buckets, so the locked path's lock updates stay in L2;
//                                a byte is set with a CAS on its 32-bit word
//   full_bits  u32[nb_cap / 32]  bit b set = bucket b was seen full (set by the claim that took
//                                its last free slot, cleared by deletes).  A hint only: the
//                                evictor reads it for all 8 victims' alternate buckets at once
//                                (L2 hits) and then reads just one bucket that has room, where
//                                the reference probes victims' buckets one by one
//   counters   u64[64 * 16]      slow-path event counters in 64 stripes of 16 words (summed by
//                                the host) and the sticky error word (stripe 0, word 15)
//   tags       u64[nb_cap]       byte j of tags[b] = an 8-bit fingerprint of the key in slot j of
//                                bucket b (1..255), 0 when the slot is free.  64 MiB at 2^23
//                                buckets against 512 MiB of slots: a lookup reads the tag words
//                                and then only the 32 B sector whose fingerprint matches, and an
//                                absent key usually reads no slot at all.  Random 32 B sector
//                                reads run at about 1.7x the rate of 64 B bucket reads on B200.
//                                Invariant: an occupied slot's byte holds its key's fingerprint.
//                                Small batches keep it per op (the claimer publishes the byte
//                                after its claim CAS); a bulk insert skips the upkeep and
//                                rebuilds every tag word from the slots afterwards (k_retag).  A
//                                free slot's byte is 0 as long as no delete or resize ran since
//                                the last clear; afterwards it may hold a stale fingerprint,
//                                which costs a read but never hides a key.
//
// A slot holds (value << 32) | key (include/hive_hash_table_struct.cuh:297-311); key 0 is the
// empty sentinel, so an all-zero slot is free (include/utils.h:39-47).  There is no freeMask
// array: a slot is free iff it reads 0, and a free slot is claimed with one 64-bit CAS.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace hive {

typedef unsigned long long u64;

constexpr int kSlots = 8;

// Per-op status codes (uint8 outputs).  Success is any non-zero code except kStError.
enum : uint8_t {
    kStFail = 0,      // insert: not placed (stash full) or key 0; find/erase: not found
    kStInserted = 1,  // insert placed a new key in a bucket; find/erase/increment: success
    kStUpdated = 2,   // insert overwrote the value of an existing key (upsert)
    kStStashed = 3,   // insert placed a new key in the overflow stash
    kStDefer = 0xFE,  // internal: the op needs the locked path and was queued for the second pass
    kStError = 0xFF,  // a bounded wait expired (lock timeout or retry budget spent)
};

// Counter slots.
enum {
    kCtrSlowPath = 0,     // inserts that found their canonical bucket full
    kCtrEvictions = 1,    // victims moved H0 -> H1
    kCtrStashPush = 2,    // keys written to the stash
    kCtrFailed = 3,       // inserts that could not be placed
    kCtrLockTimeout = 4,  // lock waits that expired
    kCtrRetryOut = 5,     // CAS retry budgets that ran out
    kCtrDupFixed = 6,     // unused: claims of one key are serialised, so no copy is ever removed
    kCtrLockWaits = 7,    // lock attempts that found the bucket locked (contention)
    kCtrError = 15,       // sticky error bits (kErr*)
};
enum : unsigned long long { kErrLockTimeout = 1ull, kErrRetryOut = 2ull };

constexpr uint32_t kFlagHoles = 1u;     // deletes or a resize ran since the last clear
constexpr uint32_t kFlagEvictH1 = 4u;   // set on the launch's copy only: the locked path tries
                                        // H1's own keys as victims before the stash (region-
                                        // ordered batches), not only once the stash is full
constexpr uint32_t kFlagPrimaryFirst = 8u;  // set on the launch's copy only: its first pass
                                            // claimed in H0 only (region order, sub-batches)
constexpr uint32_t kFlagUntagged = 2u;  // set on the launch's copy only: the launch neither reads
                                        // nor keeps the tag words (a bulk insert that rebuilds them
                                        // after it, or a table too large for them to stay in L2)
constexpr uint32_t kFlagHandOn = 16u;  // set on the launch's copy only: a locked-path insert
                                      // whose H0 lock is taken at its first attempt, or whose
                                      // eviction found no victim, returns kStDefer (holding no
                                      // lock) instead of waiting or using the stash, for a later
                                      // pass that finishes such ops together
constexpr uint32_t kFlagResumed = 32u;     // set on the launch's copy only: the ops were counted
                                           // on the slow path by the pass that handed them on
constexpr uint32_t kFlagMigrating = 64u;   // set on the launch's copy only: the same launch splits
                                           // buckets [split, win_end) of the level while its ops
                                           // run (see in_window)

// The device view of a table, passed to every kernel by value.
//
// Addressing is linear hashing over the policy's 32-bit hash h (level L, base N0):
//   n_lo = N0 << L;  b = h mod n_lo;  if b < split: b = h mod 2*n_lo.
// With L = 0 and split = 0 this is exactly the reference's get_bucket = hash % num_buckets
// (include/HashPolicies.cuh:13-16).  Splitting bucket b moves its keys to b or b + n_lo.
struct Table {
    u64* slots;
    u64* stash;
    uint32_t* stash_bits;
    uint32_t* locks;  // lock bytes, 4 per word
    uint32_t* full_bits;
    u64* counters;
    u64* tags;
    u64 m_lo;  // fastmod magic for n_lo
    u64 m_hi;  // fastmod magic for 2 * n_lo
    uint32_t n_lo;
    uint32_t split;
    uint32_t max_evictions;
    uint32_t flags;
    uint32_t win_end;      // with kFlagMigrating: the window being split is [split, win_end)
    uint32_t stash_depth;  // slots of a canonical stash that inserts may use (1..8)
};

// ---------------------------------------------------------------------------------------------
// Hashes (restated from include/hash.hpp of the reference; published integer hashes)
// ---------------------------------------------------------------------------------------------

// Thomas Wang's integer hash, the reference's hash1 (include/hash.hpp:29-37).
__host__ __device__ __forceinline__ uint32_t wang_hash(uint32_t k) {
    k = ~k + (k << 15);
    k ^= k >> 12;
    k += k << 2;
    k ^= k >> 4;
    k *= 2057u;
    k ^= k >> 16;
    return k;
}

// Bob Jenkins' 32-bit integer hash, the reference's hash2 (include/hash.hpp:49-62; its two PTX
// lop3 0x96 steps are 3-input XORs).
__host__ __device__ __forceinline__ uint32_t jenkins_hash(uint32_t k) {
    k = (k + 0x7ed55d16u) + (k << 12);
    k = (k ^ 0xc761c23cu) ^ (k >> 19);
    k = (k + 0x165667b1u) + (k << 5);
    k = (k + 0xd3a2646cu) ^ (k << 9);
    k = (k + 0xfd7046c5u) + (k << 3);
    k = (k ^ 0xb55a4f09u) ^ (k >> 16);
    return k;
}

__host__ __device__ __forceinline__ uint32_t fmix32(uint32_t h) {
    h ^= h >> 16;
    h *= 0x85ebca6bu;
    h ^= h >> 13;
    h *= 0xc2b2ae35u;
    h ^= h >> 16;
    return h;
}

// One-block MurmurHash3_x86_32, seed 0, length 4: the reference's murmurhash
// (include/hash.hpp:110-138).
__host__ __device__ __forceinline__ uint32_t murmur_hash(uint32_t key) {
    uint32_t k = key * 0xcc9e2d51u;
    k = (k << 15) | (k >> 17);
    k *= 0x1b873593u;
    uint32_t h = (k << 13) | (k >> 19);
    h = h * 5u + 0xe6546b64u;
    return fmix32(h ^ 4u);
}

// The reference's cityhash mixer (include/hash.hpp:80-108).
__host__ __device__ __forceinline__ uint32_t city_hash(uint32_t key) {
    uint32_t k = key ^ 0x9ae16a3bu;
    k *= 0xc2b2ae35u;
    k ^= 0x1b873593u;
    k *= 0x85ebca6bu;
    uint32_t h = k * 0xc2b2ae35u;
    h ^= 0x1b873593u;
    h *= 0x85ebca6bu;
    return fmix32(h ^ 4u);
}

// Hash policies: NumHashes = 2 and the two raw hashes of a key
// (include/HashPolicies.cuh:10-17 Default2HashPolicy, :29-36 MurmurCityHashPolicy).
template <int P>
struct Policy;
template <>
struct Policy<0> {
    __device__ __forceinline__ static uint32_t h0(uint32_t k) { return wang_hash(k); }
    __device__ __forceinline__ static uint32_t h1(uint32_t k) { return jenkins_hash(k); }
};
template <>
struct Policy<1> {
    __device__ __forceinline__ static uint32_t h0(uint32_t k) { return murmur_hash(k); }
    __device__ __forceinline__ static uint32_t h1(uint32_t k) { return city_hash(k); }
};

// a mod d for 32-bit a and d >= 1 with m = floor((2^64 - 1) / d) + 1 (Lemire, Kaser, Kurz,
// "Faster Remainder by Direct Computation", 2019): exact for every 32-bit a and d.
__device__ __forceinline__ uint32_t fastmod(uint32_t a, u64 m, uint32_t d) {
    return (uint32_t)__umul64hi(m * (u64)a, (u64)d);
}

__device__ __forceinline__ uint32_t bucket_addr(const Table& t, uint32_t h) {
    uint32_t b = fastmod(h, t.m_lo, t.n_lo);
    if (b < t.split) b = fastmod(h, t.m_hi, t.n_lo << 1);
    return b;
}

// Whether hash h addresses a bucket of the window that the running launch is splitting: such a
// key may sit in its old home b = h mod n_lo or its new one, h mod 2 n_lo (b or b + n_lo).
__device__ __forceinline__ bool in_window(const Table& t, uint32_t h) {
    if (!(t.flags & kFlagMigrating)) return false;
    const uint32_t b = fastmod(h, t.m_lo, t.n_lo);
    return b >= t.split && b < t.win_end;
}
__device__ __forceinline__ uint32_t new_home(const Table& t, uint32_t h) { return fastmod(h, t.m_hi, t.n_lo << 1); }

// ---------------------------------------------------------------------------------------------
// Bucket access
// ---------------------------------------------------------------------------------------------

struct Bucket {
    u64 s[kSlots];
};

// Read-only kernels: the table does not change during the launch, so the non-coherent path is
// valid; L1 allocation is skipped because bucket reads are random.
__device__ __forceinline__ void load_bucket_ro(const u64* p, Bucket& b) {
    asm volatile("ld.global.nc.L1::no_allocate.v4.u64 {%0,%1,%2,%3}, [%4];"
                 : "=l"(b.s[0]), "=l"(b.s[1]), "=l"(b.s[2]), "=l"(b.s[3])
                 : "l"(p));
    asm volatile("ld.global.nc.L1::no_allocate.v4.u64 {%0,%1,%2,%3}, [%4];"
                 : "=l"(b.s[4]), "=l"(b.s[5]), "=l"(b.s[6]), "=l"(b.s[7])
                 : "l"(p + 4));
}

// Kernels that modify the table: relaxed gpu-scope loads are served by L2 (the coherence point),
// never by a stale L1 line, so a retry after a lost CAS always sees the current bucket.
__device__ __forceinline__ void load_bucket(const u64* p, Bucket& b) {
    asm volatile("ld.relaxed.gpu.global.v4.u64 {%0,%1,%2,%3}, [%4];"
                 : "=l"(b.s[0]), "=l"(b.s[1]), "=l"(b.s[2]), "=l"(b.s[3])
                 : "l"(p)
                 : "memory");
    asm volatile("ld.relaxed.gpu.global.v4.u64 {%0,%1,%2,%3}, [%4];"
                 : "=l"(b.s[4]), "=l"(b.s[5]), "=l"(b.s[6]), "=l"(b.s[7])
                 : "l"(p + 4)
                 : "memory");
}

__device__ __forceinline__ uint32_t ld_relaxed_u32(const uint32_t* p) {
    uint32_t v;
    asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ u64 pack(uint32_t k, uint32_t v) { return ((u64)v << 32) | k; }
__device__ __forceinline__ uint32_t key_of(u64 kv) { return (uint32_t)kv; }
__device__ __forceinline__ uint32_t val_of(u64 kv) { return (uint32_t)(kv >> 32); }

// Bit j set: slot j holds key k (k != 0, so a match is never an empty slot).
__device__ __forceinline__ uint32_t match_mask(const Bucket& b, uint32_t k) {
    uint32_t m = 0;
#pragma unroll
    for (int j = 0; j < kSlots; ++j) m |= (uint32_t)(key_of(b.s[j]) == k) << j;
    return m;
}
__device__ __forceinline__ uint32_t empty_mask(const Bucket& b) {
    uint32_t m = 0;
#pragma unroll
    for (int j = 0; j < kSlots; ++j) m |= (uint32_t)(b.s[j] == 0ull) << j;
    return m;
}
__device__ __forceinline__ u64 slot_at(const Bucket& b, int j) {
    u64 r = b.s[0];
#pragma unroll
    for (int q = 1; q < kSlots; ++q)
        if (q == j) r = b.s[q];
    return r;
}

__device__ __forceinline__ u64 cas64(u64* p, u64 expect, u64 desired) {
    return atomicCAS(p, expect, desired);
}

__device__ __forceinline__ bool stash_flag(const Table& t, uint32_t b) {
    return (ld_relaxed_u32(t.stash_bits + (b >> 5)) >> (b & 31)) & 1u;
}
__device__ __forceinline__ bool stash_flag_ro(const Table& t, uint32_t b) {
    return (__ldg(t.stash_bits + (b >> 5)) >> (b & 31)) & 1u;
}

// Event counters are striped: stripe s (s = SM id mod kCounterStripes) holds its own 16 words,
// 128 B apart, and the host sums the stripes.  One shared word would serialise every slow-path
// op of a launch on one L2 slice (millions of same-address atomics at about one per clock).
// Within a warp, the lanes counting the same event add their count with one atomic.
constexpr int kCounterStripes = 64;
constexpr int kCounterStride = 16;  // u64 words per stripe

__device__ __forceinline__ unsigned sm_id() {
    unsigned id;
    asm volatile("mov.u32 %0, %%smid;" : "=r"(id));
    return id;
}
__device__ __forceinline__ unsigned lane_id() {
    unsigned id;
    asm volatile("mov.u32 %0, %%laneid;" : "=r"(id));
    return id;
}

__device__ __forceinline__ void count(const Table& t, int ctr) {
    const unsigned peers = __match_any_sync(__activemask(), ctr);
    if (lane_id() == (unsigned)(__ffs(peers) - 1))
        atomicAdd(t.counters + (sm_id() % kCounterStripes) * kCounterStride + ctr, (u64)__popc(peers));
}
// The sticky error word lives in stripe 0 only.
__device__ __forceinline__ void raise_error(const Table& t, u64 bits) { atomicOr(t.counters + kCtrError, bits); }

// Full-bucket hints.  mark_full is called by the claim that took a bucket's last free slot.
__device__ __forceinline__ void mark_full(const Table& t, uint32_t b) {
    asm volatile("red.relaxed.gpu.global.or.b32 [%0], %1;" ::"l"(t.full_bits + (b >> 5)), "r"(1u << (b & 31))
                 : "memory");
}
__device__ __forceinline__ void mark_not_full(const Table& t, uint32_t b) {
    asm volatile("red.relaxed.gpu.global.and.b32 [%0], %1;" ::"l"(t.full_bits + (b >> 5)), "r"(~(1u << (b & 31)))
                 : "memory");
}
__device__ __forceinline__ bool full_flag(const Table& t, uint32_t b) {
    return (ld_relaxed_u32(t.full_bits + (b >> 5)) >> (b & 31)) & 1u;
}

// Release/acquire-ordered fence for the publication steps below (cheaper than __threadfence,
// which is sequentially consistent).
__device__ __forceinline__ void fence_acq_rel() { asm volatile("fence.acq_rel.gpu;" ::: "memory"); }

constexpr int kRetryLimit = 64;       // CAS retries of one op on one bucket
constexpr int kLockSpinLimit = 1 << 16;  // lock attempts before the wait is declared expired

// Set bucket b's lock byte if it is clear: a CAS on the word holding it, retried while only the
// other bytes (other buckets' locks) change.  Returns true when taken, false when the byte is set.
__device__ __forceinline__ bool lock_byte_try(const Table& t, uint32_t b) {
    uint32_t* w = t.locks + (b >> 2);
    const uint32_t bit = 1u << (8 * (b & 3));
    uint32_t old = ld_relaxed_u32(w);
    for (int r = 0; r < kRetryLimit; ++r) {
        if (old & bit) return false;
        const uint32_t obs = atomicCAS(w, old, old | bit);
        if (obs == old) return true;
        old = obs;
    }
    return false;
}

// Bounded test-and-set on the bucket's lock byte.  Returns false when the wait expired.
//
// The lock only excludes other evictors of the same bucket; every table access made while it is
// held is itself a gpu-scope CAS or a strong (ld.relaxed.gpu) load, each completed (its result
// consumed) before the next is issued, and all of them are performed at L2, the point of
// coherence.  The only fire-and-forget writes are the full-bucket hints and the stash flag, and
// the stash flag is published before its entry (see insert_locked).  So relaxed lock operations
// suffice and no fence is paid per eviction.
__device__ __forceinline__ bool lock_bucket(const Table& t, uint32_t b) {
    unsigned ns = 32;
    for (int i = 0; i < kLockSpinLimit; ++i) {
        if (lock_byte_try(t, b)) return true;
        count(t, kCtrLockWaits);
        __nanosleep(ns);
        if (ns < 1024) ns <<= 1;
    }
    count(t, kCtrLockTimeout);
    raise_error(t, kErrLockTimeout);
    return false;
}
__device__ __forceinline__ void unlock_bucket(const Table& t, uint32_t b) {
    atomicAnd(t.locks + (b >> 2), ~(1u << (8 * (b & 3))));
}

// A few attempts at the lock of a second bucket while the first one is held: never waits long,
// so two evictors that each hold one of the pair and want the other cannot block each other.
__device__ __forceinline__ bool try_lock_bucket(const Table& t, uint32_t b) {
    for (int i = 0; i < 4; ++i) {
        if (lock_byte_try(t, b)) return true;
        __nanosleep(64);
    }
    return false;
}

// ---------------------------------------------------------------------------------------------
// Slot tags (see the layout above)
// ---------------------------------------------------------------------------------------------

// The key's 8-bit fingerprint, never 0; a mixer of its own, unrelated to the bucket hashes.
__host__ __device__ __forceinline__ uint32_t tag_of(uint32_t k) {
    const uint32_t f = fmix32(k ^ 0x2545F491u) >> 24;
    return f ? f : 1u;
}

// 0xFF/0x00 per byte -> one bit per byte (the four multiplied bits land on distinct positions).
__device__ __forceinline__ uint32_t byte_bits(uint32_t m) { return ((m & 0x01010101u) * 0x01020408u) >> 24; }

// Bit j set: byte j of the tag word equals f (f = 0: the free slots).
__device__ __forceinline__ uint32_t tag_match(u64 T, uint32_t f) {
    const uint32_t rep = f * 0x01010101u;
    return byte_bits(__vcmpeq4((uint32_t)T, rep)) | (byte_bits(__vcmpeq4((uint32_t)(T >> 32), rep)) << 4);
}

__device__ __forceinline__ u64 ld_relaxed_u64(const u64* p) {
    u64 v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ u64 load_tags(const Table& t, uint32_t b) { return ld_relaxed_u64(t.tags + b); }
// L2 cache policies of the read-only lookup path: the tag words (reused by every lookup) are
// kept in L2 ahead of the slot sectors, each of which a lookup batch touches about once.
__device__ __forceinline__ u64 l2_evict_last() {
    u64 p;
    asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
    return p;
}
__device__ __forceinline__ u64 l2_evict_first() {
    u64 p;
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
    return p;
}
__device__ __forceinline__ u64 load_tags_ro(const Table& t, uint32_t b) {
    u64 v;
    asm volatile("ld.global.nc.L1::no_allocate.L2::cache_hint.u64 %0, [%1], %2;"
                 : "=l"(v)
                 : "l"(t.tags + b), "l"(l2_evict_last()));
    return v;
}

// The claim of a free slot on a table without holes: the byte is 0 and only the winner of the
// slot's claim CAS writes it, so an OR is exact; fire-and-forget.
__device__ __forceinline__ void tag_publish(const Table& t, uint32_t b, int j, uint32_t f) {
    asm volatile("red.relaxed.gpu.global.or.b64 [%0], %1;" ::"l"(t.tags + b), "l"((u64)f << (8 * j)) : "memory");
}

// Byte j := f, other bytes unchanged (a claim on a table with holes, or an eviction's overwrite).
// The word CAS completes before the caller's next access, so a reader that finds the slot's new
// contents through a later step also finds its fingerprint.  tag_set and tag_clear do nothing in
// a launch without tag upkeep (kFlagUntagged).
__device__ __forceinline__ void tag_set(const Table& t, uint32_t b, int j, uint32_t f) {
    if (t.flags & kFlagUntagged) return;
    u64* w = t.tags + b;
    const u64 mask = 0xFFull << (8 * j), val = (u64)f << (8 * j);
    u64 old = ld_relaxed_u64(w);
    for (int r = 0; r < kRetryLimit; ++r) {
        const u64 nw = (old & ~mask) | val;
        if (nw == old) return;
        const u64 obs = atomicCAS(w, old, nw);
        if (obs == old) return;
        old = obs;
    }
    count(t, kCtrRetryOut);
    raise_error(t, kErrRetryOut);
}

// Byte j := 0 after slot j was freed, unless the slot has been claimed again meanwhile (then its
// claimer writes the byte).  A claimer's tag_set that lands between this check and the CAS
// changes the word, so the CAS fails and the check runs again.
__device__ __forceinline__ void tag_clear(const Table& t, uint32_t b, int j) {
    if (t.flags & kFlagUntagged) return;
    u64* w = t.tags + b;
    const u64 mask = 0xFFull << (8 * j);
    const u64* slot = t.slots + (size_t)b * kSlots + j;
    u64 old = ld_relaxed_u64(w);
    for (int r = 0; r < kRetryLimit; ++r) {
        if (!(old & mask)) return;
        if (ld_relaxed_u64(slot) != 0ull) return;
        const u64 obs = atomicCAS(w, old, old & ~mask);
        if (obs == old) return;
        old = obs;
    }
    count(t, kCtrRetryOut);
    raise_error(t, kErrRetryOut);
}

// The tag word of a bucket's contents (the rebuild and the resize kernels, which own the buckets
// they rewrite).
__device__ __forceinline__ u64 tag_word(const u64 (&s)[kSlots]) {
    u64 w = 0;
#pragma unroll
    for (int j = 0; j < kSlots; ++j)
        if (s[j]) w |= (u64)tag_of(key_of(s[j])) << (8 * j);
    return w;
}

// One 32 B sector (slots 4s .. 4s + 3) of bucket p.
struct Sector {
    u64 s[4];
};
__device__ __forceinline__ void load_sector_ro(const u64* p, Sector& S) {
    asm volatile("ld.global.nc.L1::no_allocate.L2::cache_hint.v4.u64 {%0,%1,%2,%3}, [%4], %5;"
                 : "=l"(S.s[0]), "=l"(S.s[1]), "=l"(S.s[2]), "=l"(S.s[3])
                 : "l"(p), "l"(l2_evict_first()));
}
__device__ __forceinline__ void load_sector(const u64* p, Sector& S) {
    asm volatile("ld.relaxed.gpu.global.v4.u64 {%0,%1,%2,%3}, [%4];"
                 : "=l"(S.s[0]), "=l"(S.s[1]), "=l"(S.s[2]), "=l"(S.s[3])
                 : "l"(p)
                 : "memory");
}
__device__ __forceinline__ uint32_t sector_match(const Sector& S, uint32_t k) {
    uint32_t m = 0;
#pragma unroll
    for (int j = 0; j < 4; ++j) m |= (uint32_t)(key_of(S.s[j]) == k) << j;
    return m;
}
__device__ __forceinline__ u64 sector_at(const Sector& S, int j) {
    u64 r = S.s[0];
#pragma unroll
    for (int q = 1; q < 4; ++q)
        if (q == j) r = S.s[q];
    return r;
}

// ---------------------------------------------------------------------------------------------
// Warp-cooperative bucket reads.  On B200 random reads are bounded by the number of L2 requests,
// not by bytes: a random 32 B read and a random 64 B read each move one 128 B DRAM line, but one
// thread's 64 B read is two 32 B load instructions, i.e. two requests.  Two lanes that load the
// two halves of the same bucket in one instruction make a single two-sector request.  Measured
// over a 512 MiB buffer: 59.5 G random buckets/s this way against 34.3 G/s one bucket per thread,
// and 25.8 G/s against 22.9 G/s with a CAS into the bucket after the read (a CAS alone: 26.1).
// ---------------------------------------------------------------------------------------------

// Position of the (n + 1)-th lowest set bit of m (n >= 0), or -1 when m has n bits or fewer.
__device__ __forceinline__ int nth_bit(uint32_t m, int n) {
    if (__popc(m) <= n) return -1;
    int pos = 0;  // the largest pos with at most n set bits below it
#pragma unroll
    for (int w = 16; w; w >>= 1)
        if (__popc(m & ((1u << (pos + w)) - 1u)) <= n) pos += w;
    return pos;
}

// Slot masks of one half-bucket S for key k, placed for half h: bits 4h..4h+3 the free slots,
// bits 8+4h..11+4h the slots holding k.
__device__ __forceinline__ uint32_t half_masks(const Sector& S, uint32_t k, unsigned h) {
    uint32_t m = 0;
#pragma unroll
    for (int q = 0; q < 4; ++q) m |= ((uint32_t)(S.s[q] == 0ull) << q) | ((uint32_t)(key_of(S.s[q]) == k) << (8 + q));
    return m << (4 * h);
}

// Every lane of a converged warp calls it.  A lane with `need` gets bucket b's slot masks: bits
// 0-7 the free slots, bits 8-15 the slots holding k (k != 0, so a free slot never matches); other
// lanes get 0.  In each round lane l loads half (l & 1) of the bucket of the (l >> 1)-th needing
// lane not yet served, so up to 16 buckets take one load instruction.  (Issuing both rounds'
// loads before using either was measured no faster and needs 8 more registers.)
__device__ __forceinline__ uint32_t warp_bucket_masks(const u64* __restrict__ slots, bool need, uint32_t b,
                                                      uint32_t k) {
    const unsigned lane = lane_id();
    const unsigned all = __ballot_sync(0xffffffffu, need);
    const unsigned rank = __popc(all & ((1u << lane) - 1u));
    const int rounds = (__popc(all) + 15) >> 4;
    uint32_t out = 0;
    for (int r = 0; r < rounds; ++r) {
        const int owner = nth_bit(all, 16 * r + (int)(lane >> 1));
        const int src = owner < 0 ? 0 : owner;
        const uint32_t ob = __shfl_sync(0xffffffffu, b, src);
        const uint32_t ok = __shfl_sync(0xffffffffu, k, src);
        uint32_t m = 0;
        if (owner >= 0) {
            Sector S;
            load_sector(slots + (size_t)ob * kSlots + 4 * (lane & 1), S);
            m = half_masks(S, ok, lane & 1u);
        }
        m |= __shfl_xor_sync(0xffffffffu, m, 1);
        const uint32_t got = __shfl_sync(0xffffffffu, m, (int)((2 * rank) & 31u));
        if (need && (int)(rank >> 4) == r) out = got;
    }
    return out;
}

// warp_bucket_masks over two buckets per needing lane at once (both halves of both in the same
// rounds): *ma and *mb receive the masks of buckets a and b, and keys_a the eight keys of a.
__device__ __forceinline__ void warp_two_buckets(const u64* __restrict__ slots, bool need, uint32_t a, uint32_t b,
                                                 uint32_t k, uint32_t (&keys_a)[kSlots], uint32_t* ma,
                                                 uint32_t* mb) {
    const unsigned lane = lane_id();
    const unsigned h = lane & 1u;
    const unsigned all = __ballot_sync(0xffffffffu, need);
    const unsigned rank = __popc(all & ((1u << lane) - 1u));
    const int rounds = (__popc(all) + 15) >> 4;
    const int from = (int)((2 * rank) & 31u);
    *ma = *mb = 0;
    for (int r = 0; r < rounds; ++r) {
        const int owner = nth_bit(all, 16 * r + (int)(lane >> 1));
        const int src = owner < 0 ? 0 : owner;
        const uint32_t oa = __shfl_sync(0xffffffffu, a, src);
        const uint32_t ob = __shfl_sync(0xffffffffu, b, src);
        const uint32_t ok = __shfl_sync(0xffffffffu, k, src);
        uint32_t xa = 0, xb = 0, kk[4] = {0, 0, 0, 0};
        if (owner >= 0) {
            Sector SA, SB;
            load_sector(slots + (size_t)oa * kSlots + 4 * h, SA);
            load_sector(slots + (size_t)ob * kSlots + 4 * h, SB);
            xa = half_masks(SA, ok, h);
            xb = half_masks(SB, ok, h);
#pragma unroll
            for (int q = 0; q < 4; ++q) kk[q] = key_of(SA.s[q]);
        }
        xa |= __shfl_xor_sync(0xffffffffu, xa, 1);
        xb |= __shfl_xor_sync(0xffffffffu, xb, 1);
        const uint32_t ga = __shfl_sync(0xffffffffu, xa, from);
        const uint32_t gb = __shfl_sync(0xffffffffu, xb, from);
        const bool mine = need && (int)(rank >> 4) == r;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const uint32_t lo = __shfl_sync(0xffffffffu, kk[q], from);
            const uint32_t hi = __shfl_sync(0xffffffffu, kk[q], from + 1);
            if (mine) {
                keys_a[q] = lo;
                keys_a[4 + q] = hi;
            }
        }
        if (mine) {
            *ma = ga;
            *mb = gb;
        }
    }
}

// Find k in bucket b using its tag word T: reads only the sectors holding a matching fingerprint.
template <bool kReadOnly>
__device__ __forceinline__ bool find_tagged(const Table& t, uint32_t b, u64 T, uint32_t k, uint32_t f, uint32_t* v) {
    uint32_t m = tag_match(T, f);
    while (m) {
        const int sec = (__ffs(m) - 1) >> 2;
        m &= ~(0xFu << (4 * sec));
        Sector S;
        if (kReadOnly) load_sector_ro(t.slots + (size_t)b * kSlots + 4 * sec, S);
        else load_sector(t.slots + (size_t)b * kSlots + 4 * sec, S);
        const uint32_t hit = sector_match(S, k);
        if (hit) {
            *v = val_of(sector_at(S, __ffs(hit) - 1));
            return true;
        }
    }
    return false;
}

// ---------------------------------------------------------------------------------------------
// Lookup: H0, H1, then the canonical stash gated by its flag
// (include/hive_hash_lookup.cuh:126-155)
// ---------------------------------------------------------------------------------------------

// The slots are read only where a fingerprint matches; the stash has no tags and is read whole
// when its flag is set.  Read-only kernels (nothing changes during the launch) read both tag
// words up front, two independent L2 reads (reading H1's only after H0 missed saves tag-word
// accesses but was measured slower, even at 2^23 buckets where the words outgrow what L2 keeps).
// Otherwise H1's tags are read only after H0 missed:
// an eviction writes the victim (and its fingerprint) to H1 before removing it from H0, so
// reading H0 then H1 in that order always finds it.
template <int P, bool kReadOnly>
__device__ __forceinline__ bool find_one_buckets(const Table& t, uint32_t k, uint32_t* v);

template <int P>
__device__ __noinline__ bool find_one_migrating(const Table& t, uint32_t k, uint32_t* v);

template <int P, bool kReadOnly>
__device__ __forceinline__ bool find_one(const Table& t, uint32_t k, uint32_t* v) {
    if (!kReadOnly && (t.flags & kFlagMigrating) &&
        (in_window(t, Policy<P>::h0(k)) || in_window(t, Policy<P>::h1(k))))
        return find_one_migrating<P>(t, k, v);
    if (t.flags & kFlagUntagged) return find_one_buckets<P, kReadOnly>(t, k, v);
    if (k == 0) return false;
    const uint32_t f = tag_of(k);
    const uint32_t b0 = bucket_addr(t, Policy<P>::h0(k));
    const uint32_t b1 = bucket_addr(t, Policy<P>::h1(k));
    const u64 T0 = kReadOnly ? load_tags_ro(t, b0) : load_tags(t, b0);
    u64 T1 = kReadOnly ? load_tags_ro(t, b1) : 0ull;
    if (find_tagged<kReadOnly>(t, b0, T0, k, f, v)) return true;
    if (!kReadOnly) T1 = load_tags(t, b1);
    if (b1 != b0 && find_tagged<kReadOnly>(t, b1, T1, k, f, v)) return true;
    if (kReadOnly ? stash_flag_ro(t, b0) : stash_flag(t, b0)) {
        Bucket B;
        if (kReadOnly) load_bucket_ro(t.stash + (size_t)b0 * kSlots, B);
        else load_bucket(t.stash + (size_t)b0 * kSlots, B);
        const uint32_t m = match_mask(B, k);
        if (m) {
            *v = val_of(slot_at(B, __ffs(m) - 1));
            return true;
        }
    }
    return false;
}

// Lookup without tags (a table whose tag words are not kept): H0 whole, then H1, then the stash.
template <int P, bool kReadOnly>
__device__ __forceinline__ bool find_one_buckets(const Table& t, uint32_t k, uint32_t* v) {
    if (k == 0) return false;
    const uint32_t b0 = bucket_addr(t, Policy<P>::h0(k));
    Bucket B;
    if (kReadOnly) load_bucket_ro(t.slots + (size_t)b0 * kSlots, B);
    else load_bucket(t.slots + (size_t)b0 * kSlots, B);
    uint32_t m = match_mask(B, k);
    if (!m) {
        const uint32_t b1 = bucket_addr(t, Policy<P>::h1(k));
        if (b1 != b0) {
            if (kReadOnly) load_bucket_ro(t.slots + (size_t)b1 * kSlots, B);
            else load_bucket(t.slots + (size_t)b1 * kSlots, B);
            m = match_mask(B, k);
        }
        if (!m && (kReadOnly ? stash_flag_ro(t, b0) : stash_flag(t, b0))) {
            if (kReadOnly) load_bucket_ro(t.stash + (size_t)b0 * kSlots, B);
            else load_bucket(t.stash + (size_t)b0 * kSlots, B);
            m = match_mask(B, k);
        }
        if (!m) return false;
    }
    *v = val_of(slot_at(B, __ffs(m) - 1));
    return true;
}

// Lookup of a key with a candidate bucket in the window being split by the running launch.  The
// splitter writes a bucket's new home (and the new home's stash) before it clears what moved
// out of the old one, so reading each old home before its new home, and the old stash before the
// new, always finds a key that is present (whole buckets: the tag words of the window are
// rewritten by the splitter).  Keys of the window are not evicted during such a launch and no
// key is evicted into it, so the H0-then-H1 order needs nothing more.
template <int P>
__device__ __noinline__ bool find_one_migrating(const Table& t, uint32_t k, uint32_t* v) {
    if (k == 0) return false;
    uint32_t homes[5];
    int nh = 0;
    const uint32_t hs[2] = {Policy<P>::h0(k), Policy<P>::h1(k)};
#pragma unroll
    for (int x = 0; x < 2; ++x) {
        if (in_window(t, hs[x])) {
            const uint32_t b = fastmod(hs[x], t.m_lo, t.n_lo), b2 = new_home(t, hs[x]);
            homes[nh++] = b;
            if (b2 != b) homes[nh++] = b2;
        } else {
            homes[nh++] = bucket_addr(t, hs[x]);
        }
    }
    Bucket B;
    for (int x = 0; x < nh; ++x) {
        load_bucket(t.slots + (size_t)homes[x] * kSlots, B);
        const uint32_t m = match_mask(B, k);
        if (m) {
            *v = val_of(slot_at(B, __ffs(m) - 1));
            return true;
        }
    }
    // the canonical stash: old, then new
    uint32_t c[2];
    int nc = 0;
    if (in_window(t, hs[0])) {
        c[nc++] = fastmod(hs[0], t.m_lo, t.n_lo);
        if (new_home(t, hs[0]) != c[0]) c[nc++] = new_home(t, hs[0]);
    } else {
        c[nc++] = bucket_addr(t, hs[0]);
    }
    for (int x = 0; x < nc; ++x) {
        if (!stash_flag(t, c[x])) continue;
        load_bucket(t.stash + (size_t)c[x] * kSlots, B);
        const uint32_t m = match_mask(B, k);
        if (m) {
            *v = val_of(slot_at(B, __ffs(m) - 1));
            return true;
        }
    }
    return false;
}

// Whether an op on key k would write into the window being split (its candidate buckets, or its
// canonical stash): such writes wait until the window is done.
template <int P>
__device__ __forceinline__ bool touches_window(const Table& t, uint32_t k) {
    return in_window(t, Policy<P>::h0(k)) || in_window(t, Policy<P>::h1(k));
}

// ---------------------------------------------------------------------------------------------
// Update in place: CAS the first copy of k in bucket p to kv.
// Returns 1 updated, 0 key absent, -1 lost a race (caller reloads).
// ---------------------------------------------------------------------------------------------
__device__ __forceinline__ int update_in(u64* p, uint32_t k, u64 kv) {
    Bucket B;
    load_bucket(p, B);
    uint32_t m = match_mask(B, k);
    if (!m) return 0;
    int j = __ffs(m) - 1;
    u64 old = slot_at(B, j);
    return cas64(p + j, old, kv) == old ? 1 : -1;
}

// Increment the value of the first copy of k in bucket p.  Returns 1 done (new value in *nv),
// 0 absent, -1 lost a race.
__device__ __forceinline__ int increment_in(u64* p, uint32_t k, uint32_t* nv) {
    Bucket B;
    load_bucket(p, B);
    uint32_t m = match_mask(B, k);
    if (!m) return 0;
    int j = __ffs(m) - 1;
    u64 old = slot_at(B, j);
    uint32_t v = val_of(old) + 1u;
    if (cas64(p + j, old, pack(k, v)) != old) return -1;
    *nv = v;
    return 1;
}

// ---------------------------------------------------------------------------------------------
// Insert = upsert (S2).  Four stages as in include/hive_hash_insert.cuh:898-1042:
//   A  try-replace in the candidate buckets and the canonical stash,
//   B  claim a free slot with a 64-bit CAS: in the canonical bucket H0, and when H0 is full in
//      the key's other bucket H1 (the reference claims in H0 only and goes straight to C),
//   C  bounded depth-1 cuckoo eviction from H0 under H0's lock (and of H1's own keys under H1's
//      lock: before the stash for region-ordered batches, else once the stash is full),
//   D  the canonical bucket's overflow stash.
//
// Invariants that keep every key in exactly one place and visible at all times:
//   * a new key is placed in H0, in H1 only when H0 is full, else in H0's stash;
//   * a victim is moved only from its own H0 to its H1, and is written to H1 before its H0 slot
//     is overwritten, so a reader scanning H0 then H1 always sees it;
//   * an evictor holds the lock of the victim's own bucket (its H0), so one victim has one mover;
//   * every slot change is a CAS from an observed value, so a concurrent update or delete of
//     the victim is detected and either propagated to the copy or undone.
// Without kFlagHoles (no delete or resize since the last clear) slots only ever go from free to
// occupied and every claimer (new keys and moved victims alike) takes the lowest free slot, so:
//   * a key lives in H1 only if H0 is full, and in the stash only if H0 and H1 are both full;
//   * stage B needs no lock: two inserts of one key race for the same lowest free slot of the
//     same bucket, one CAS wins and the other re-reads the bucket and finds the key.
// Ops that reach stages C/D (both buckets full) can be deferred by the first pass to a queue that
// a second, compact pass finishes, so a warp of one-op threads does not wait on its slowest lane.
// ---------------------------------------------------------------------------------------------

enum { kEvPlaced = 1, kEvRetry = 2, kEvNone = 0 };

// Victims are considered in groups of kEvictGroup slots: a group's candidates (slots j < limit,
// the reference's kick % 8 order, whose key lives in its own H0 = b0 and whose H1 is another
// bucket) are hashed and their H1 full bits read in one round of independent L2 reads, then the
// open ones are tried in slot order; the next group is hashed only if none of them took a victim.
// The order of attempts is that of all open candidates in slot order, but a first group that
// places the victim (the common case) spares the other group's hashing, most of this path's
// instructions.
constexpr int kEvictGroup = 4;

template <int P>
__device__ __forceinline__ int try_evict(const Table& t, u64* B0p, const Bucket& B0, uint32_t b0, u64 kv) {
    const int limit = t.max_evictions < (uint32_t)kSlots ? (int)t.max_evictions : kSlots;
#pragma unroll 1
    for (int g = 0; g < limit; g += kEvictGroup) {
        uint32_t alts[kEvictGroup];
        uint32_t cand = 0;
#pragma unroll
        for (int q = 0; q < kEvictGroup; ++q) {
            const int j = g + q;
            alts[q] = b0;
            if (j >= limit) continue;
            const u64 vkv = slot_at(B0, j);
            if (vkv == 0ull) {  // a slot that freed up is taken directly
                if (cas64(B0p + j, 0ull, kv) != 0ull) return kEvRetry;
                tag_set(t, b0, j, tag_of(key_of(kv)));
                return kEvPlaced;
            }
            const uint32_t vk = key_of(vkv);
            if (bucket_addr(t, Policy<P>::h0(vk)) != b0) continue;  // victim lives in its H1
            const uint32_t h1 = Policy<P>::h1(vk);
            const uint32_t alt = bucket_addr(t, h1);
            if (alt == b0 || in_window(t, h1)) continue;  // no victim moves into a window being split
            alts[q] = alt;
            cand |= 1u << q;
        }
        uint32_t open = 0;
#pragma unroll
        for (int q = 0; q < kEvictGroup; ++q)
            if ((cand >> q) & 1u)
                if (!((__ldcg(t.full_bits + (alts[q] >> 5)) >> (alts[q] & 31)) & 1u)) open |= 1u << q;
        while (open) {
            const int q0 = __ffs(open) - 1;
            open &= open - 1;
            const int j = g + q0;
            u64 vkv = slot_at(B0, j);
            const uint32_t vk = key_of(vkv);
            uint32_t alt = alts[0];
#pragma unroll
            for (int q = 1; q < kEvictGroup; ++q)
                if (q == q0) alt = alts[q];
            u64* Ap = t.slots + (size_t)alt * kSlots;
            Bucket A;
            load_bucket(Ap, A);
            const uint32_t e = empty_mask(A);
            if (!e) {
                mark_full(t, alt);
                continue;
            }
            const int d = __ffs(e) - 1;
            if (cas64(Ap + d, 0ull, vkv) != 0ull) continue;  // lost the free slot; next victim
            if (__popc(e) == 1) mark_full(t, alt);
            // The copy's fingerprint is in place before H0's slot changes (tag_set completes).
            tag_set(t, alt, d, tag_of(vk));
            // The victim is now visible in both H0 slot j and H1 slot d.
            const uint32_t f = tag_of(key_of(kv));
            for (int r = 0; r < kRetryLimit; ++r) {
                u64 obs = cas64(B0p + j, vkv, kv);
                if (obs == vkv) {
                    tag_set(t, b0, j, f);
                    count(t, kCtrEvictions);
                    return kEvPlaced;
                }
                if (obs == 0ull) {
                    // Victim deleted meanwhile: drop the copy unless it changed, take the free slot.
                    if (cas64(Ap + d, vkv, 0ull) == vkv) {
                        tag_clear(t, alt, d);
                        mark_not_full(t, alt);
                    }
                    if (cas64(B0p + j, 0ull, kv) != 0ull) return kEvRetry;
                    tag_set(t, b0, j, f);
                    return kEvPlaced;
                }
                if (key_of(obs) == vk) {
                    // Victim updated meanwhile: carry the new value to the copy, then retry.
                    if (cas64(Ap + d, vkv, obs) != vkv) return kEvRetry;
                    vkv = obs;
                    continue;
                }
                if (cas64(Ap + d, vkv, 0ull) == vkv) {
                    tag_clear(t, alt, d);
                    mark_not_full(t, alt);
                }
                return kEvRetry;
            }
            count(t, kCtrRetryOut);
            raise_error(t, kErrRetryOut);
            return kEvRetry;
        }
    }
    return kEvNone;
}

// Eviction from the key's H1 (victims are H1's own keys, whose H0 is H1) under H1's lock, taken
// with a few attempts only: the caller already holds H0's lock.
template <int P>
__device__ __forceinline__ int try_evict_h1(const Table& t, u64* B1p, const Bucket& B1, uint32_t b1, u64 kv) {
    if (!try_lock_bucket(t, b1)) return kEvNone;
    const int ev = try_evict<P>(t, B1p, B1, b1, kv);
    unlock_bucket(t, b1);
    return ev;
}

// Stage C/D under H0's lock.  The caller holds the lock on b0.
template <int P>
__device__ __noinline__ uint8_t insert_locked(const Table& t, uint32_t k, u64 kv, uint32_t b0, uint32_t b1) {
    u64* B0p = t.slots + (size_t)b0 * kSlots;
    u64* B1p = t.slots + (size_t)b1 * kSlots;
    u64* Sp = t.stash + (size_t)b0 * kSlots;
    for (int r = 0; r < kRetryLimit; ++r) {
        Bucket B0, B1;
        load_bucket(B0p, B0);
        load_bucket(B1p, B1);
        uint32_t m = match_mask(B0, k);
        if (m) {
            int j = __ffs(m) - 1;
            u64 old = slot_at(B0, j);
            if (cas64(B0p + j, old, kv) == old) return kStUpdated;
            continue;
        }
        m = match_mask(B1, k);
        if (m) {
            int j = __ffs(m) - 1;
            u64 old = slot_at(B1, j);
            if (cas64(B1p + j, old, kv) == old) return kStUpdated;
            continue;
        }
        if (stash_flag(t, b0)) {
            int u = update_in(Sp, k, kv);
            if (u == 1) return kStUpdated;
            if (u < 0) continue;
        }
        uint32_t e = empty_mask(B0);
        if (e) {
            int j = __ffs(e) - 1;
            if (cas64(B0p + j, 0ull, kv) == 0ull) {
                tag_set(t, b0, j, tag_of(k));
                if (__popc(e) == 1) mark_full(t, b0);
                return kStInserted;
            }
            continue;
        }
        e = b1 != b0 ? empty_mask(B1) : 0u;
        if (e) {
            int j = __ffs(e) - 1;
            if (cas64(B1p + j, 0ull, kv) == 0ull) {
                tag_set(t, b1, j, tag_of(k));
                if (__popc(e) == 1) mark_full(t, b1);
                return kStInserted;
            }
            continue;
        }
        int ev = try_evict<P>(t, B0p, B0, b0, kv);
        if (ev == kEvPlaced) return kStInserted;
        if (ev == kEvRetry) continue;
        // No victim of H0 can move: the same with H1's own keys (keys whose H0 is H1), under H1's
        // lock, and the key takes the freed slot in its H1.  Every invariant above still holds: a
        // victim moves from its H0 to its H1, and the key lands in H1 while its H0 is full.  Tried
        // before the stash for region-ordered batches (kFlagEvictH1), whose placement it keeps
        // from overflowing stashes; otherwise only once the stash is full.
        const bool h1_first = t.flags & kFlagEvictH1;
        if (h1_first && b1 != b0) {
            ev = try_evict_h1<P>(t, B1p, B1, b1, kv);
            if (ev == kEvPlaced) return kStInserted;
            if (ev == kEvRetry) continue;
        }
        // Handed on (the caller releases the lock): ops bound for the stash take several more
        // dependent steps than an eviction, so finishing them in a later pass of their own keeps
        // them from holding up the warps of the eviction pass.
        if (t.flags & kFlagHandOn) return kStDefer;
        // Stage D: the canonical bucket's stash.  Its flag is raised before the entry is
        // written, so a reader that finds the entry also finds the flag set.
        if (!(atomicOr(t.stash_bits + (b0 >> 5), 1u << (b0 & 31)) & (1u << (b0 & 31)))) fence_acq_rel();
        bool again = false;  // a last-resort eviction raced: rescan from the top
        for (int q = 0; q < kRetryLimit; ++q) {
            Bucket S;
            load_bucket(Sp, S);
            uint32_t se = empty_mask(S) & ((1u << t.stash_depth) - 1u);
            if (!se) {
                if (!h1_first && b1 != b0) {
                    ev = try_evict_h1<P>(t, B1p, B1, b1, kv);
                    if (ev == kEvPlaced) return kStInserted;
                    again = ev == kEvRetry;
                    if (again) break;
                }
                count(t, kCtrFailed);
                return kStFail;
            }
            int j = __ffs(se) - 1;
            if (cas64(Sp + j, 0ull, kv) == 0ull) {
                count(t, kCtrStashPush);
                return kStStashed;
            }
        }
        if (again) continue;
        break;
    }
    count(t, kCtrRetryOut);
    raise_error(t, kErrRetryOut);
    return kStError;
}

// Update the value of k in slot j of bucket p, whose current contents are `cur` (key k).
// Returns kStUpdated, or 0 if the retry budget ran out (the locked path finishes the op).
__device__ __forceinline__ uint8_t update_slot(u64* p, int j, u64 cur, u64 kv) {
    for (int r = 0; r < kRetryLimit; ++r) {
        const u64 obs = cas64(p + j, cur, kv);
        if (obs == cur) return kStUpdated;
        cur = obs;  // a racing update of the same key; slots never change keys without holes
    }
    return 0;
}

// Without holes and without tag upkeep (a bulk insert whose tag words are rebuilt after it):
// update k in bucket b or claim b's lowest free slot from one 64 B read of the bucket.  Without
// holes a slot never becomes free again, so after a lost CAS the next free slot of the same
// snapshot is the next candidate: the bucket is read once however many claimers race for it (a
// slot passed over was observed by its failed CAS, so a racing insert of k is always seen).
// Returns kStUpdated / kStInserted, or 0 when b is full or a budget ran out.
__device__ __forceinline__ uint8_t claim_or_update_untagged(const Table& t, uint32_t b, uint32_t k, u64 kv) {
    u64* p = t.slots + (size_t)b * kSlots;
    Bucket B;
    load_bucket(p, B);
    const uint32_t m = match_mask(B, k);
    if (m) {
        const int j = __ffs(m) - 1;
        return update_slot(p, j, slot_at(B, j), kv);
    }
    uint32_t e = empty_mask(B);
    while (e) {
        const int j = __ffs(e) - 1;
        e &= e - 1;
        const u64 obs = cas64(p + j, 0ull, kv);
        if (obs == 0ull) {
            if (!e) mark_full(t, b);
            return kStInserted;
        }
        if (key_of(obs) == k) return update_slot(p, j, obs, kv);
    }
    return 0;
}

// claim_or_update_untagged from masks a warp_bucket_masks read produced, for the first pass of a
// bulk insert without holes: no other launch runs and the pass itself never moves a key, so a slot
// that holds k keeps holding k and an update is one exchange.  Returns as
// claim_or_update_untagged.
__device__ __forceinline__ uint8_t claim_from_masks(const Table& t, uint32_t b, uint32_t k, u64 kv, uint32_t masks) {
    u64* p = t.slots + (size_t)b * kSlots;
    const uint32_t m = masks >> 8;
    if (m) {
        atomicExch(p + (__ffs(m) - 1), kv);
        return kStUpdated;
    }
    uint32_t e = masks & 0xFFu;
    while (e) {
        const int j = __ffs(e) - 1;
        e &= e - 1;
        const u64 obs = cas64(p + j, 0ull, kv);
        if (obs == 0ull) {
            if (!e) mark_full(t, b);
            return kStInserted;
        }
        if (key_of(obs) == k) {
            atomicExch(p + j, kv);
            return kStUpdated;
        }
    }
    return 0;
}

// Without holes, with tag upkeep: update k in bucket b or claim b's lowest free slot, guided by
// b's tag word.  Without holes the free slots by the tag word are a superset of the truly free
// ones (a claim publishes its fingerprint after its CAS), so trying them in ascending order
// reaches the lowest free slot, and two inserts of one key race for the same slot: one CAS wins
// and the other sees the key and updates it.  A key already in b has its fingerprint published
// unless its claim races with this op, which the sector snapshot or the CAS then shows.  Only the
// sector holding a candidate slot is read, before its CAS: a CAS that misses L2 runs far slower
// than a 32 B read followed by a CAS that hits.  Returns as claim_or_update_untagged.
template <bool kTagged = true>
__device__ __forceinline__ uint8_t claim_or_update(const Table& t, uint32_t b, uint32_t k, u64 kv) {
    if (!kTagged || (t.flags & kFlagUntagged)) return claim_or_update_untagged(t, b, k, kv);
    u64* p = t.slots + (size_t)b * kSlots;
    const uint32_t f = tag_of(k);
    const u64 T = load_tags(t, b);
    uint32_t m = tag_match(T, f);
    while (m) {
        const int j = __ffs(m) - 1;
        m &= m - 1;
        const u64 cur = ld_relaxed_u64(p + j);
        if (key_of(cur) == k) return update_slot(p, j, cur, kv);
    }
    uint32_t e = tag_match(T, 0u);
    while (e) {
        const int sec = (__ffs(e) - 1) >> 2;
        uint32_t es = (e >> (4 * sec)) & 0xFu;
        e &= ~(0xFu << (4 * sec));
        u64* sp = p + 4 * sec;
        Sector S;
        load_sector(sp, S);
        const uint32_t hit = sector_match(S, k);
        if (hit) {
            const int q = __ffs(hit) - 1;
            return update_slot(sp, q, sector_at(S, q), kv);
        }
        while (es) {
            const int q = __ffs(es) - 1;
            es &= es - 1;
            if (sector_at(S, q) != 0ull) continue;  // taken by a claim still publishing its tag
            const u64 obs = cas64(sp + q, 0ull, kv);
            if (obs == 0ull) {
                tag_publish(t, b, 4 * sec + q, f);
                if (!e && !es) mark_full(t, b);  // every other slot carries a fingerprint
                return kStInserted;
            }
            if (key_of(obs) == k) return update_slot(sp, q, obs, kv);
        }
    }
    return 0;
}

// With holes and per-slot tags, update k in bucket b if a copy is there.  Only the sectors with
// a matching fingerprint are read.  A copy that changes key between the read and the CAS was
// moved by an eviction (its copy is already in H1) and is looked for there.  Returns 1 updated,
// 0 not in b.
__device__ __forceinline__ int update_tagged(const Table& t, uint32_t b, uint32_t k, uint32_t f, u64 kv) {
    u64* p = t.slots + (size_t)b * kSlots;
    uint32_t m = tag_match(load_tags(t, b), f);
    while (m) {
        const int sec = (__ffs(m) - 1) >> 2;
        m &= ~(0xFu << (4 * sec));
        Sector S;
        load_sector(p + 4 * sec, S);
        const uint32_t hit = sector_match(S, k);
        if (!hit) continue;
        u64* sp = p + 4 * sec + (__ffs(hit) - 1);
        u64 cur = sector_at(S, __ffs(hit) - 1);
        for (int r = 0; r < kRetryLimit; ++r) {
            const u64 obs = cas64(sp, cur, kv);
            if (obs == cur) return 1;
            if (key_of(obs) != k) break;
            cur = obs;
        }
    }
    return 0;
}

// With holes and per-slot tags, claim a free slot of bucket b for kv: the slots whose tag byte is
// 0, one sector at a time, each sector read before its CAS (a CAS that misses L2 is far slower).
// Returns kStInserted, or 0 when b has no free slot by its tag word.
__device__ __forceinline__ uint8_t claim_tagged(const Table& t, uint32_t b, uint32_t f, u64 kv) {
    u64* p = t.slots + (size_t)b * kSlots;
    uint32_t e = tag_match(load_tags(t, b), 0u);
    while (e) {
        const int sec = (__ffs(e) - 1) >> 2;
        uint32_t es = (e >> (4 * sec)) & 0xFu;
        e &= ~(0xFu << (4 * sec));
        Sector S;
        load_sector(p + 4 * sec, S);
        while (es) {
            const int q = __ffs(es) - 1;
            es &= es - 1;
            if (sector_at(S, q) != 0ull) continue;
            if (cas64(p + 4 * sec + q, 0ull, kv) == 0ull) {
                tag_set(t, b, 4 * sec + q, f);
                if (!e && !es) mark_full(t, b);
                return kStInserted;
            }
        }
    }
    return 0;
}

// Lock-free stages A and B with holes, per-slot tags and at most one op per key in the batch: an
// existing copy is looked for in H0, then H1 (whose tags are read after H0, as in find_one), then
// the stash; with none, the key claims a free slot of H0, else of H1.  No other insert of the key
// runs in the batch, so no second copy can appear and there is no duplicate check.  Returns the
// op's status, or 0 for the locked path.
template <bool kPrimaryOnly>
__device__ __noinline__ uint8_t insert_holes_unique(const Table& t, uint32_t k, u64 kv, uint32_t b0, uint32_t b1) {
    const uint32_t f = tag_of(k);
    if (update_tagged(t, b0, k, f, kv)) return kStUpdated;
    if (b1 != b0 && update_tagged(t, b1, k, f, kv)) return kStUpdated;
    if (stash_flag(t, b0)) {
        u64* Sp = t.stash + (size_t)b0 * kSlots;
        for (int r = 0; r < kRetryLimit; ++r) {
            const int u = update_in(Sp, k, kv);
            if (u == 1) return kStUpdated;
            if (u == 0) break;
        }
    }
    const uint8_t st = claim_tagged(t, b0, f, kv);
    if (st || b1 == b0 || kPrimaryOnly) return st;
    return claim_tagged(t, b1, f, kv);
}

// Which insert protocol a kernel compiles: chosen from the table's flags at run time, or fixed
// by the host (which knows the flags) so the kernel carries only the code it needs.  The base
// (low two bits) says whether the table may have holes; two flag bits refine it:
//   kModePrimary   a deferring first pass claims in H0 only (region-ordered batches, see
//                  insert_lockfree)
//   kModeUntagged  no tag upkeep: a bulk insert whose tag words are rebuilt after it; the
//                  launch's Table copy carries kFlagUntagged for the code chosen at run time
//   kModeUnique    the caller guarantees each key at most once in the batch: with holes, an
//                  insert cannot race another insert of its key, so it finds an existing copy and
//                  a free slot through the tag words and skips the duplicate check
enum Mode { kModeRuntime = 0, kModeMono = 1, kModeHoles = 2, kModePrimary = 4, kModeUntagged = 8, kModeUnique = 16 };
__host__ __device__ constexpr int mode_base(int m) { return m & 3; }
__device__ __forceinline__ bool tagged(const Table& t) { return !(t.flags & kFlagUntagged); }

// Lock-free stages A and B.  Returns the op's final status, or 0 when the op must go on: to the
// locked path (stages C/D) when H0 and H1 are both full, or -- with kPrimaryOnly, the first pass
// of a region-ordered insert -- as soon as H0 is full.  A region-ordered batch reaches the
// buckets in address order, so a first pass that claimed in H1 would let the early regions'
// overflow take the H1 slots that later regions' own keys need; claiming only in H0 there and
// leaving every H1 claim to the second pass keeps the placement independent of the region order.
// In submission order (the default) the first pass claims in H0, then in H1: overflow then meets
// a table that is still filling, and fewer ops reach eviction and the stash.
template <int P, int kMode = kModeRuntime, bool kPrimaryOnly = false>
__device__ __forceinline__ uint8_t insert_lockfree(const Table& t, uint32_t k, u64 kv, uint32_t b0, uint32_t b1) {
    u64* B0p = t.slots + (size_t)b0 * kSlots;
    u64* B1p = t.slots + (size_t)b1 * kSlots;
    constexpr bool kTagged = !(kMode & kModeUntagged);
    const bool holes = mode_base(kMode) == kModeHoles || (mode_base(kMode) == kModeRuntime && (t.flags & kFlagHoles));
    if (!holes) {
        uint8_t st = claim_or_update<kTagged>(t, b0, k, kv);
        if (st || b1 == b0 || kPrimaryOnly) return st;
        return claim_or_update<kTagged>(t, b1, k, kv);
    }
    if (kTagged && (kMode & kModeUnique) && tagged(t)) return insert_holes_unique<kPrimaryOnly>(t, k, kv, b0, b1);
    // With holes a key may sit in H1 or the stash while H0 has room: look in all three and update
    // a copy in place.  A new key is claimed only on the locked path, under H0's lock: two inserts
    // of one key that both find it absent are serialised there, and the second one's rescan under
    // the lock finds the first one's copy, so no key ever gets two copies.  (A claim made without
    // the lock could land in H0 while a racing insert of the same key, which found H0 full before
    // a delete freed a slot, lands in H1 or the stash.  The reference guards the same race with a
    // duplicate check under the canonical bucket's lock, include/hive_hash_insert.cuh:522-541.)
    u64* Sp = t.stash + (size_t)b0 * kSlots;
    for (int r = 0; r < kRetryLimit; ++r) {
        Bucket B0, B1;
        load_bucket(B0p, B0);
        load_bucket(B1p, B1);
        uint32_t m = match_mask(B0, k);
        if (m) {
            int j = __ffs(m) - 1;
            u64 old = slot_at(B0, j);
            if (cas64(B0p + j, old, kv) == old) return kStUpdated;
            continue;
        }
        m = match_mask(B1, k);
        if (m) {
            int j = __ffs(m) - 1;
            u64 old = slot_at(B1, j);
            if (cas64(B1p + j, old, kv) == old) return kStUpdated;
            continue;
        }
        if (stash_flag(t, b0)) {
            int u = update_in(Sp, k, kv);
            if (u == 1) return kStUpdated;
            if (u < 0) continue;
        }
        return 0;
    }
    return 0;
}

// Stages C/D: H0's lock, a rescan, eviction, the stash.
template <int P>
__device__ __noinline__ uint8_t insert_locked_path(const Table& t, uint32_t k, u64 kv, uint32_t b0, uint32_t b1) {
    if (!(t.flags & kFlagResumed)) count(t, kCtrSlowPath);
    if (t.flags & kFlagHandOn) {
        // one attempt: an op that would wait for the lock is handed on instead of stalling its warp
        if (!lock_byte_try(t, b0)) {
            count(t, kCtrLockWaits);
            return kStDefer;
        }
    } else if (!lock_bucket(t, b0)) {
        return kStError;
    }
    uint8_t st = insert_locked<P>(t, k, kv, b0, b1);
    unlock_bucket(t, b0);
    return st;
}

// One upsert.  With kDefer, an op that needs the locked path returns kStDefer untouched (and the
// locked path is not compiled into the caller).
template <int P, bool kDefer = false, int kMode = kModeRuntime>
__device__ __forceinline__ uint8_t insert_one(const Table& t, uint32_t k, uint32_t v) {
    if (k == 0) return kStFail;
    const u64 kv = pack(k, v);
    const uint32_t b0 = bucket_addr(t, Policy<P>::h0(k));
    const uint32_t b1 = bucket_addr(t, Policy<P>::h1(k));
    uint8_t st = insert_lockfree<P, kMode, kDefer && (kMode & kModePrimary) != 0>(t, k, kv, b0, b1);
    if (st) return st;
    if (kDefer) return kStDefer;
    return insert_locked_path<P>(t, k, kv, b0, b1);
}

// A deferred op in the second pass.  Without holes the buckets the first pass found full stay
// full; with holes the whole protocol runs again (a slot may have freed up since).
template <int P>
__device__ __forceinline__ uint8_t insert_deferred_one(const Table& t, uint32_t k, uint32_t v) {
    if (t.flags & kFlagHoles) return insert_one<P>(t, k, v);
    const u64 kv = pack(k, v);
    const uint32_t b0 = bucket_addr(t, Policy<P>::h0(k));
    const uint32_t b1 = bucket_addr(t, Policy<P>::h1(k));
    // A first pass that also claimed in H1 deferred the op because both buckets were full, and
    // without holes they stay full: the locked path follows directly (it rescans both buckets
    // under the lock, which also finds a racing insert of k).  After an H0-only first pass the
    // op claims in H1 first.
    if (b1 != b0 && (t.flags & kFlagPrimaryFirst)) {
        const uint8_t st = tagged(t) ? claim_or_update<true>(t, b1, k, kv) : claim_or_update<false>(t, b1, k, kv);
        if (st) return st;
    }
    return insert_locked_path<P>(t, k, kv, b0, b1);
}

// The locked path of a second-pass insert into a table without holes, with every lane of the
// warp in step: each lane (with `on`) takes its op through one fixed sequence -- one attempt at
// H0's lock; H0 and H1 read together, one request per bucket shared by a lane pair
// (warp_two_buckets), and H0's stash flag; an update if the key is already there (placed by an
// earlier op of the same key, whose insert holds the same lock); else the H1 and full hint of
// four slots of H0 at a time; the masks of the first open victim's bucket (one shared request)
// and the victim's slot; the copy of the victim there, then the key over the victim -- so the
// lanes' dependent memory accesses overlap instead of running one divergent path after another.
// (Per-lane whole-bucket reads, two requests per bucket, measured slower here.)  Returns kStInserted / kStUpdated, or kStDefer for an op that meets anything else
// (lock taken, H0's stash flagged, no open victim, a victim bucket found full, a lost CAS, a slot
// free against expectation): such an op holds no lock and has changed nothing, and is handed on
// to a pass that runs the general locked path.  Only for launches without tag upkeep
// (kFlagUntagged).
//
// Without holes a bucket the first pass found full stays full, and every change to a key's
// entries is made under that key's H0 lock, so under H0's lock the victim's slot cannot change
// between the copy and the overwrite, and an existing copy of k is updated by an exchange.
template <int P>
__device__ __forceinline__ uint8_t insert_locked_converged(const Table& t, bool on, uint32_t k, uint32_t v) {
    const u64 kv = pack(k, v);
    const uint32_t b0 = on ? bucket_addr(t, Policy<P>::h0(k)) : 0u;
    const uint32_t b1 = on ? bucket_addr(t, Policy<P>::h1(k)) : 0u;
    if (on) count(t, kCtrSlowPath);
    const bool locked = on && lock_byte_try(t, b0);
    if (on && !locked) count(t, kCtrLockWaits);
    u64* B0p = t.slots + (size_t)b0 * kSlots;
    // H0 (its keys and masks) and H1 (masks) in shared requests, and the stash flag; the victim's
    // whole slot is read again, an L2 hit, once it is chosen
    const bool stashed = locked && stash_flag(t, b0);
    uint32_t keys[kSlots], m0, m1;
    warp_two_buckets(t.slots, locked, b0, b1, k, keys, &m0, &m1);
    if (b1 == b0) m1 = 0u;  // no second bucket: neither room nor a copy there
    uint8_t st = kStDefer;
    bool evict = false;
    if (locked) {
        if (m0 >> 8) {
            atomicExch(B0p + (__ffs(m0 >> 8) - 1), kv);
            st = kStUpdated;
        } else if ((m1 >> 8) && b1 != b0) {
            atomicExch(t.slots + (size_t)b1 * kSlots + (__ffs(m1 >> 8) - 1), kv);
            st = kStUpdated;
        } else {
            // a flagged stash may hold k (its entries change only under H0's lock): general path
            evict = !(m0 & 0xFFu) && !(m1 & 0xFFu) && !stashed;
        }
    }
    // the first open victim: H1 and full hint of four slots at a time, the next four only when
    // none of the first is open
    const int limit = t.max_evictions < (uint32_t)kSlots ? (int)t.max_evictions : kSlots;
    uint32_t alt = 0;
    int jv = -1;
#pragma unroll 1
    for (int g = 0; evict && jv < 0 && g < limit; g += kEvictGroup) {
        uint32_t open = 0;
#pragma unroll
        for (int q = 0; q < kEvictGroup; ++q) {
            uint32_t kq = keys[0];
#pragma unroll
            for (int j = 1; j < kSlots; ++j)
                if (j == g + q) kq = keys[j];
            const uint32_t a = bucket_addr(t, Policy<P>::h1(kq));
            if (g + q < limit && a != b0 && !((__ldcg(t.full_bits + (a >> 5)) >> (a & 31)) & 1u)) open |= 1u << q;
        }
        if (open) {
            jv = g + __ffs(open) - 1;
            uint32_t kj = keys[0];
#pragma unroll
            for (int j = 1; j < kSlots; ++j)
                if (j == jv) kj = keys[j];
            alt = bucket_addr(t, Policy<P>::h1(kj));
        }
    }
    const bool try_alt = evict && jv >= 0;
    const u64 vkv = try_alt ? ld_relaxed_u64(B0p + jv) : 0ull;
    const uint32_t ma = warp_bucket_masks(t.slots, try_alt, alt, 0xFFFFFFFFu);
    if (try_alt) {
        const uint32_t e = ma & 0xFFu;
        if (!e) {
            mark_full(t, alt);
        } else {
            u64* Ap = t.slots + (size_t)alt * kSlots;
            const int d = __ffs(e) - 1;
            if (cas64(Ap + d, 0ull, vkv) == 0ull) {
                if (__popc(e) == 1) mark_full(t, alt);
                // the victim is now in both places; the key takes its H0 slot
                if (cas64(B0p + jv, vkv, kv) == vkv) {
                    count(t, kCtrEvictions);
                    st = kStInserted;
                } else if (cas64(Ap + d, vkv, 0ull) == vkv) {
                    mark_not_full(t, alt);
                }
            }
        }
    }
    if (locked) unlock_bucket(t, b0);
    return st;
}

// ---------------------------------------------------------------------------------------------
// Delete: remove every copy in H0, H1 and the canonical stash, no early exit
// (include/hive_hash_delete.cuh:168-194).  Returns true if any copy was removed.
// ---------------------------------------------------------------------------------------------
// Removes every copy of k from bucket p.  is_slots: p is table bucket b (not a stash), whose
// full hint is cleared after a removal.
// A table bucket whose tag word holds no matching fingerprint is not read.
__device__ __forceinline__ bool erase_in(const Table& t, u64* p, uint32_t k, bool is_slots, uint32_t b) {
    if (is_slots && tagged(t) && !tag_match(load_tags(t, b), tag_of(k))) return false;
    bool removed = false;
    for (int r = 0; r < kRetryLimit; ++r) {
        Bucket B;
        load_bucket(p, B);
        uint32_t m = match_mask(B, k);
        if (!m) {
            if (removed && is_slots) mark_not_full(t, b);
            return removed;
        }
        int j = __ffs(m) - 1;
        u64 old = slot_at(B, j);
        if (cas64(p + j, old, 0ull) == old) {
            removed = true;
            if (is_slots) tag_clear(t, b, j);
        }
    }
    if (removed && is_slots) mark_not_full(t, b);
    count(t, kCtrRetryOut);
    raise_error(t, kErrRetryOut);
    return removed;
}

template <int P>
__device__ __forceinline__ bool erase_one(const Table& t, uint32_t k) {
    if (k == 0) return false;
    const uint32_t b0 = bucket_addr(t, Policy<P>::h0(k));
    const uint32_t b1 = bucket_addr(t, Policy<P>::h1(k));
    bool removed = erase_in(t, t.slots + (size_t)b0 * kSlots, k, true, b0);
    if (b1 != b0) removed |= erase_in(t, t.slots + (size_t)b1 * kSlots, k, true, b1);
    if (stash_flag(t, b0)) removed |= erase_in(t, t.stash + (size_t)b0 * kSlots, k, false, b0);
    return removed;
}

// ---------------------------------------------------------------------------------------------
// Increment (the reference's OperationType::ATOMIC_INC, include/utils.h:14, which its mixed
// kernel leaves unhandled): value += 1 on the first copy found in H0, H1, stash order.
// ---------------------------------------------------------------------------------------------
template <int P>
__device__ __forceinline__ bool increment_one(const Table& t, uint32_t k, uint32_t* nv) {
    if (k == 0) return false;
    const uint32_t b0 = bucket_addr(t, Policy<P>::h0(k));
    const uint32_t b1 = bucket_addr(t, Policy<P>::h1(k));
    for (int r = 0; r < kRetryLimit; ++r) {
        int u = increment_in(t.slots + (size_t)b0 * kSlots, k, nv);
        if (u == 1) return true;
        if (u < 0) continue;
        if (b1 != b0) {
            u = increment_in(t.slots + (size_t)b1 * kSlots, k, nv);
            if (u == 1) return true;
            if (u < 0) continue;
        }
        if (stash_flag(t, b0)) {
            u = increment_in(t.stash + (size_t)b0 * kSlots, k, nv);
            if (u == 1) return true;
            if (u < 0) continue;
        }
        return false;
    }
    count(t, kCtrRetryOut);
    raise_error(t, kErrRetryOut);
    return false;
}

}  // namespace hive
