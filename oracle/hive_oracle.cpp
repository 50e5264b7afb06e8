// hive_oracle.cpp -- TEST INFRASTRUCTURE ONLY (the oracle), never part of the product path.
//
// A CPU restatement of the Hive hash table's semantics and of its bucketed cuckoo algorithm,
// used by tests/ as the parity checker and by bench.py's cpu_baseline / `--impl reference`
// leg as the CPU baseline.  Nothing in hivehashtable_b200/ links, loads or calls this file.
//
// Contents
//   1. Hash functions and the bucket-selection policies (restated from the reference's
//      include/hash.hpp and include/HashPolicies.cuh).
//   2. The seeded workload generators (splitmix64 step of include/zipf_distribution.h:10-16).
//   3. A std::unordered_map replay: the semantic oracle for every op result and for the final
//      key->value set (reference semantics S1-S6 of include/hive_hash_insert.cuh,
//      include/hive_hash_lookup.cuh, include/hive_hash_delete.cuh).
//   3b. The per-key serialisation check of concurrent launches: every op result and final state
//      must come from some order of each key's ops that keeps launch order.
//   4. A multithreaded CPU bucketed cuckoo table (8-slot buckets, two hashes, CAS slot claims,
//      depth-1 eviction under bucket locks, per-bucket overflow stash) driven by std::thread:
//      the reported CPU baseline for the same policy.
//
// Parity pin: the hash functions are checked against the reference's own hash.hpp compiled in
// this container (oracle/ref/hash_kat.cpp -> oracle/_ref/hash_kat) and, on the GPU, against its
// device-only hash2 (oracle/ref/hash_dev_kat.cu).  The generators and the replay have no
// counterpart in the reference (it has no tests and seeds from std::random_device), so they are
// pinned by the golden fixtures under tests/golden/ made by tests/golden/make_golden.py.
//
// Exported with C linkage for ctypes.

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <thread>
#include <unordered_map>
#include <unordered_set>
#include <vector>

namespace {

// ---------------------------------------------------------------------------------------------
// 1. Hash functions
// ---------------------------------------------------------------------------------------------

// Thomas Wang's 32-bit integer hash as used by the reference's hash1
// (include/hash.hpp:29-37 device form with modulus, :39-47 host form without).
inline uint32_t ref_hash1(uint32_t key) {
    key = ~key + (key << 15);
    key = key ^ (key >> 12);
    key = key + (key << 2);
    key = key ^ (key >> 4);
    key = key * 2057u;
    key = key ^ (key >> 16);
    return key;
}

// Bob Jenkins' 6-shift 32-bit integer hash as used by the reference's hash2
// (include/hash.hpp:49-62).  The reference writes two of the six steps as inline PTX
// `shr.u32` + `lop3.b32 ..., 0x96`; truth table 0x96 is the 3-input XOR, so each of those
// steps is (key ^ C) ^ (key >> s).  Plain-C form of the same: UniformHashFunction/src/
// hash_function.cu:181-189.
inline uint32_t ref_hash2(uint32_t key) {
    key = (key + 0x7ed55d16u) + (key << 12);
    key = (key ^ 0xc761c23cu) ^ (key >> 19);
    key = (key + 0x165667b1u) + (key << 5);
    key = (key + 0xd3a2646cu) ^ (key << 9);
    key = (key + 0xfd7046c5u) + (key << 3);
    key = (key ^ 0xb55a4f09u) ^ (key >> 16);
    return key;
}

inline uint32_t rotl32(uint32_t x, int r) { return (x << r) | (x >> (32 - r)); }

// MurmurHash3 32-bit finaliser (published, Austin Appleby).
inline uint32_t fmix32(uint32_t h) {
    h ^= h >> 16;
    h *= 0x85ebca6bu;
    h ^= h >> 13;
    h *= 0xc2b2ae35u;
    h ^= h >> 16;
    return h;
}

// The reference's "murmurhash": one MurmurHash3_x86_32 block with seed 0 and length 4
// (include/hash.hpp:110-138).
inline uint32_t ref_murmur(uint32_t key) {
    uint32_t k = key * 0xcc9e2d51u;
    k = rotl32(k, 15);
    k *= 0x1b873593u;
    uint32_t h = k;  // seed 0 ^ k
    h = rotl32(h, 13);
    h = h * 5u + 0xe6546b64u;
    h ^= 4u;
    return fmix32(h);
}

// The reference's "cityhash" 32-bit mixer (include/hash.hpp:80-108).
inline uint32_t ref_city(uint32_t key) {
    uint32_t k = key ^ 0x9ae16a3bu;
    k *= 0xc2b2ae35u;
    k ^= 0x1b873593u;
    k *= 0x85ebca6bu;
    uint32_t h = k;  // 0 ^ k
    h *= 0xc2b2ae35u;
    h ^= 0x1b873593u;
    h *= 0x85ebca6bu;
    h ^= 4u;
    return fmix32(h);
}

// Policy 0 = Default2Hash {hash1, hash2} (include/HashPolicies.cuh:10-17);
// policy 1 = MurmurCityHash {murmurhash, cityhash} (include/HashPolicies.cuh:29-36).
inline uint32_t raw_hash(int policy, int idx, uint32_t key) {
    if (policy == 1) return idx == 0 ? ref_murmur(key) : ref_city(key);
    return idx == 0 ? ref_hash1(key) : ref_hash2(key);
}

// get_bucket(idx, key, num_buckets) = hash_idx(key) % num_buckets
// (include/HashPolicies.cuh:13-16, :32-35).
inline uint32_t bucket_of(int policy, int idx, uint32_t key, uint32_t num_buckets) {
    return raw_hash(policy, idx, key) % num_buckets;
}

// ---------------------------------------------------------------------------------------------
// 2. Generators
// ---------------------------------------------------------------------------------------------

// One SplitMix64 step (include/zipf_distribution.h:10-16).
inline uint64_t sm64(uint64_t& x) {
    uint64_t z = (x += 0x9e3779b97f4a7c15ULL);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}

// Keys are drawn uniformly in [1, 2^32 - 3]: 0 is the empty sentinel and the top two values
// are kept out of every workload.
constexpr uint64_t kKeySpan = 4294967293ULL;  // 2^32 - 3
inline uint32_t draw_key(uint64_t& state) { return 1u + (uint32_t)(sm64(state) % kKeySpan); }

inline uint32_t value_of(uint32_t key) {
    uint64_t s = key;
    return (uint32_t)sm64(s);
}

// ---------------------------------------------------------------------------------------------
// 4. Multithreaded CPU bucketed cuckoo table (the reported CPU baseline)
// ---------------------------------------------------------------------------------------------

constexpr int kSlots = 8;

struct CpuTable {
    int policy;
    uint32_t nb;
    int max_evictions;
    std::vector<std::atomic<uint64_t>> slots;
    std::vector<std::atomic<uint64_t>> stash;
    std::vector<std::atomic<uint32_t>> stash_bits;
    std::vector<std::atomic<uint32_t>> lock_bits;
    std::atomic<uint64_t> failed{0};

    CpuTable(int p, uint32_t nbk, int me)
        : policy(p), nb(nbk), max_evictions(me), slots((size_t)nbk * kSlots),
          stash((size_t)nbk * kSlots), stash_bits((nbk + 31) / 32), lock_bits((nbk + 31) / 32) {
        for (auto& s : slots) s.store(0, std::memory_order_relaxed);
        for (auto& s : stash) s.store(0, std::memory_order_relaxed);
        for (auto& s : stash_bits) s.store(0, std::memory_order_relaxed);
        for (auto& s : lock_bits) s.store(0, std::memory_order_relaxed);
    }

    static uint64_t pack(uint32_t k, uint32_t v) { return ((uint64_t)v << 32) | k; }
    static uint32_t key_of(uint64_t kv) { return (uint32_t)kv; }

    uint32_t b0_of(uint32_t k) const { return bucket_of(policy, 0, k, nb); }
    uint32_t b1_of(uint32_t k) const { return bucket_of(policy, 1, k, nb); }

    bool stash_flag(uint32_t b) const {
        return (stash_bits[b >> 5].load(std::memory_order_acquire) >> (b & 31)) & 1u;
    }
    void lock(uint32_t b) {
        uint32_t bit = 1u << (b & 31);
        while (lock_bits[b >> 5].fetch_or(bit, std::memory_order_acquire) & bit) std::this_thread::yield();
    }
    void unlock(uint32_t b) { lock_bits[b >> 5].fetch_and(~(1u << (b & 31)), std::memory_order_release); }

    // Returns 1 updated, 0 absent, -1 lost a race (reload).
    int try_update(std::atomic<uint64_t>* B, uint32_t k, uint64_t kv) {
        for (int j = 0; j < kSlots; ++j) {
            uint64_t s = B[j].load(std::memory_order_acquire);
            if (s != 0 && key_of(s) == k) return B[j].compare_exchange_strong(s, kv) ? 1 : -1;
        }
        return 0;
    }

    // Bulk insert protocol of include/hive_hash_insert.cuh:969-1042 (try-replace over the
    // candidates, claim in the canonical bucket H0, bounded cuckoo eviction from H0, stash),
    // with the eviction restricted to victims that sit in their own H0 so that a key only
    // ever moves H0 -> H1.  Returns 1 inserted, 2 updated, 3 stashed, 0 failed.
    int insert(uint32_t k, uint32_t v) {
        if (k == 0) return 0;
        const uint64_t kv = pack(k, v);
        const uint32_t b0 = b0_of(k), b1 = b1_of(k);
        std::atomic<uint64_t>* B0 = &slots[(size_t)b0 * kSlots];
        std::atomic<uint64_t>* B1 = &slots[(size_t)b1 * kSlots];
        std::atomic<uint64_t>* S = &stash[(size_t)b0 * kSlots];
        // Fast path: no deletes ever ran, so a key can live in H1 or the stash only if H0 is full.
        for (;;) {
            int u = try_update(B0, k, kv);
            if (u == 1) return 2;
            if (u == -1) continue;
            int e = -1;
            for (int j = 0; j < kSlots; ++j)
                if (B0[j].load(std::memory_order_acquire) == 0) { e = j; break; }
            if (e < 0) break;
            uint64_t exp = 0;
            if (B0[e].compare_exchange_strong(exp, kv)) return 1;
        }
        for (;;) {
            int u = try_update(B1, k, kv);
            if (u == 1) return 2;
            if (u == -1) continue;
            break;
        }
        lock(b0);
        int result = 0;
        for (;;) {
            int u = try_update(B0, k, kv);
            if (u == -1) continue;
            if (u == 1) { result = 2; break; }
            u = try_update(B1, k, kv);
            if (u == -1) continue;
            if (u == 1) { result = 2; break; }
            if (stash_flag(b0)) {
                u = try_update(S, k, kv);
                if (u == -1) continue;
                if (u == 1) { result = 2; break; }
            }
            // Depth-1 eviction: victim slot j = kick % 8 (include/hive_hash_insert.cuh:764-833).
            bool placed = false, raced = false;
            for (int j = 0; j < kSlots && j < max_evictions; ++j) {
                uint64_t vkv = B0[j].load(std::memory_order_acquire);
                if (vkv == 0) {
                    uint64_t exp = 0;
                    if (B0[j].compare_exchange_strong(exp, kv)) { placed = true; break; }
                    raced = true;
                    break;
                }
                uint32_t vk = key_of(vkv);
                if (b0_of(vk) != b0) continue;
                uint32_t alt = b1_of(vk);
                if (alt == b0) continue;
                std::atomic<uint64_t>* A = &slots[(size_t)alt * kSlots];
                int d = -1;
                for (int q = 0; q < kSlots; ++q)
                    if (A[q].load(std::memory_order_acquire) == 0) { d = q; break; }
                if (d < 0) continue;
                uint64_t exp = 0;
                if (!A[d].compare_exchange_strong(exp, vkv)) continue;
                uint64_t src = vkv;
                if (B0[j].compare_exchange_strong(src, kv)) { placed = true; break; }
                uint64_t undo = vkv;
                A[d].compare_exchange_strong(undo, 0);
                raced = true;
                break;
            }
            if (placed) { result = 1; break; }
            if (raced) continue;
            // Overflow stash of the canonical bucket (include/hive_hash_insert.cuh:489-517).
            stash_bits[b0 >> 5].fetch_or(1u << (b0 & 31), std::memory_order_acq_rel);
            result = 0;
            for (int j = 0; j < kSlots; ++j) {
                uint64_t exp = 0;
                if (S[j].compare_exchange_strong(exp, kv)) { result = 3; break; }
            }
            break;
        }
        unlock(b0);
        if (result == 0) failed.fetch_add(1, std::memory_order_relaxed);
        return result;
    }

    // Lookup of include/hive_hash_lookup.cuh:126-155: H0, H1, then the canonical stash.
    bool find(uint32_t k, uint32_t* v) const {
        if (k == 0) return false;
        const uint32_t b0 = b0_of(k);
        const std::atomic<uint64_t>* B = &slots[(size_t)b0 * kSlots];
        for (int j = 0; j < kSlots; ++j) {
            uint64_t s = B[j].load(std::memory_order_relaxed);
            if (s != 0 && key_of(s) == k) { *v = (uint32_t)(s >> 32); return true; }
        }
        const uint32_t b1 = b1_of(k);
        B = &slots[(size_t)b1 * kSlots];
        for (int j = 0; j < kSlots; ++j) {
            uint64_t s = B[j].load(std::memory_order_relaxed);
            if (s != 0 && key_of(s) == k) { *v = (uint32_t)(s >> 32); return true; }
        }
        if (stash_flag(b0)) {
            B = &stash[(size_t)b0 * kSlots];
            for (int j = 0; j < kSlots; ++j) {
                uint64_t s = B[j].load(std::memory_order_relaxed);
                if (s != 0 && key_of(s) == k) { *v = (uint32_t)(s >> 32); return true; }
            }
        }
        return false;
    }
};

template <typename F>
double run_threads(int threads, uint64_t n, F&& body) {
    if (threads < 1) threads = 1;
    auto t0 = std::chrono::steady_clock::now();
    std::vector<std::thread> pool;
    pool.reserve(threads);
    for (int t = 0; t < threads; ++t) {
        uint64_t lo = n * t / threads, hi = n * (t + 1) / threads;
        pool.emplace_back([lo, hi, &body] {
            for (uint64_t i = lo; i < hi; ++i) body(i);
        });
    }
    for (auto& th : pool) th.join();
    auto t1 = std::chrono::steady_clock::now();
    return std::chrono::duration<double>(t1 - t0).count();
}

struct ReplayMap {
    std::unordered_map<uint32_t, uint32_t> m;
};

// ---------------------------------------------------------------------------------------------
// 3b. Concurrent batches: the per-key serialisation check
// ---------------------------------------------------------------------------------------------
// The ops of one launch are unordered (the reference's mixed kernel runs one op per thread with
// no order among them, include/hive_kernels.cuh:119-192); launches are ordered by the stream.
// A run is correct when, for every key, some order of that key's ops that keeps launch order
// (any order inside a launch) reproduces every observed result of those ops and the key's final
// state.  Ops on different keys commute, so keys are checked one at a time.

struct SerialOp {
    uint8_t type;   // 0 insert, 1 lookup, 2 delete, 3 increment, other: no-op
    uint32_t val;   // insert value
    uint8_t st;     // observed status
    uint32_t ov;    // observed out value
};

// Applies op o to the key's state (present, value) as the replay does; false when the observed
// result cannot come from that state.  Insert statuses: 1 or 3 new key, 2 updated, 0 not placed
// (possible only while the key is absent; no effect).
inline bool serial_step(const SerialOp& o, bool& present, uint32_t& value) {
    switch (o.type) {
        case 0:
            if (o.ov != 0) return false;
            if (o.st == 0) return !present;
            if (present) {
                if (o.st != 2) return false;
            } else if (o.st != 1 && o.st != 3) {
                return false;
            }
            present = true;
            value = o.val;
            return true;
        case 1:
            return present ? (o.st == 1 && o.ov == value) : (o.st == 0 && o.ov == 0);
        case 2:
            if (o.ov != 0 || o.st != (present ? 1 : 0)) return false;
            present = false;
            return true;
        case 3:
            if (!present) return o.st == 0 && o.ov == 0;
            if (o.st != 1 || o.ov != value + 1u) return false;
            value += 1u;
            return true;
        default:
            return o.st == 0 && o.ov == 0;
    }
}

struct SerialState {
    uint64_t used, rest;  // rest = launch << 33 | present << 32 | value
    bool operator==(const SerialState& o) const { return used == o.used && rest == o.rest; }
};
struct SerialStateHash {
    size_t operator()(const SerialState& s) const { return (size_t)(s.used * 0x9E3779B97F4A7C15ull ^ s.rest); }
};

struct SerialSearch {
    const std::vector<std::vector<SerialOp>>* groups;  // the key's ops per launch, launches in order
    bool fin_present;
    uint32_t fin_value;
    int64_t budget;  // search steps left
    std::unordered_set<SerialState, SerialStateHash> dead;  // states known to lead nowhere

    // Ops of launch g not in `used` in some order, then the later launches.  Among identical
    // unused ops only the first is tried (they lead to the same states); a state already shown
    // to fail is not searched again.
    bool run(size_t g, uint64_t used, bool present, uint32_t value) {
        const auto& gs = *groups;
        if (g == gs.size()) return present == fin_present && (!present || value == fin_value);
        const auto& G = gs[g];
        if (used == (G.size() == 64 ? ~0ull : (1ull << G.size()) - 1ull)) return run(g + 1, 0, present, value);
        const SerialState key{used, ((uint64_t)g << 33) | ((uint64_t)present << 32) | value};
        if (dead.count(key)) return false;
        if (search(g, used, present, value)) return true;
        dead.insert(key);
        return false;
    }

    bool search(size_t g, uint64_t used, bool present, uint32_t value) {
        const auto& G = (*groups)[g];
        for (size_t j = 0; j < G.size(); ++j) {
            if ((used >> j) & 1ull) continue;
            bool twin = false;
            for (size_t q = 0; q < j && !twin; ++q)
                twin = !((used >> q) & 1ull) && G[q].type == G[j].type && G[q].val == G[j].val &&
                       G[q].st == G[j].st && G[q].ov == G[j].ov;
            if (twin) continue;
            bool p = present;
            uint32_t v = value;
            if (!serial_step(G[j], p, v)) continue;
            if (--budget < 0) return false;
            if (run(g, used | (1ull << j), p, v)) return true;
        }
        return false;
    }
};

// One launch's ops on a key, none of them an increment, from a known state: decided without a
// search.  Without increments the state after a write depends on that write alone: a new-key
// insert (N) needs the key absent and leaves (present, its value); an update (U) needs it present
// and leaves (present, its value); a delete that removed (D) needs it present and leaves it
// absent.  Observers leave the state alone: a lookup that found value v needs (present, v); a
// lookup that missed, a delete that found nothing and an insert that was not placed need the key
// absent.  An observer can always go right after a write that produced its state (or first, for
// the state before the launch), so an order exists iff the writes can be ordered: N and D
// alternate starting from the state before, U only while present, every observed value is
// written by some N or U (or was there before), and the last write leaves the final state.
// Returns 1 when some order exists, 0 when none does.
inline int serial_closed_form(const std::vector<SerialOp>& G, bool present, uint32_t value, bool fin_present,
                              uint32_t fin_value) {
    int64_t nN = 0, nU = 0, nD = 0;
    bool absent_seen = false;
    bool fin_by_u = false, fin_by_n = false;
    std::vector<uint32_t> written, looked;
    for (const SerialOp& o : G) {
        switch (o.type) {
            case 0:
                if (o.ov != 0) return 0;
                if (o.st == 0) {
                    absent_seen = true;
                } else if (o.st == 1 || o.st == 3) {
                    ++nN;
                    written.push_back(o.val);
                    fin_by_n |= o.val == fin_value;
                } else if (o.st == 2) {
                    ++nU;
                    written.push_back(o.val);
                    fin_by_u |= o.val == fin_value;
                } else {
                    return 0;
                }
                break;
            case 1:
                if (o.st == 1) looked.push_back(o.ov);
                else if (o.st == 0 && o.ov == 0) absent_seen = true;
                else return 0;
                break;
            case 2:
                if (o.ov != 0) return 0;
                if (o.st == 1) ++nD;
                else if (o.st == 0) absent_seen = true;
                else return 0;
                break;
            case 3:
                return 0;  // not decided by this form
            default:
                if (o.st != 0 || o.ov != 0) return 0;
                break;
        }
    }
    bool end_present;
    if (!present) {
        if (nN != nD && nN != nD + 1) return 0;
        if (nU > 0 && nN == 0) return 0;
        end_present = nN == nD + 1;
    } else {
        if (nD != nN && nD != nN + 1) return 0;
        end_present = nD == nN;
    }
    if (end_present != fin_present) return 0;
    if (absent_seen && present && nD == 0) return 0;
    std::sort(written.begin(), written.end());
    for (uint32_t v : looked)
        if (!std::binary_search(written.begin(), written.end(), v) && !(present && value == v)) return 0;
    if (fin_present) {
        if (nN + nU == 0) return value == fin_value ? 1 : 0;
        // the last write is a U carrying the final value, or the last N carrying it with every U
        // in an earlier present stretch (the one before the launch, or one after another N)
        if (!fin_by_u && !(fin_by_n && (nU == 0 || present || nN >= 2))) return 0;
    }
    return 1;
}

inline bool has_increment(const std::vector<SerialOp>& G) {
    for (const SerialOp& o : G)
        if (o.type == 3) return true;
    return false;
}

}  // namespace

extern "C" {

// ---- 1. hashes ------------------------------------------------------------------------------
uint32_t hive_oracle_raw_hash(int policy, int idx, uint32_t key) { return raw_hash(policy, idx, key); }

void hive_oracle_buckets(int policy, const uint32_t* keys, uint64_t n, uint32_t num_buckets,
                         uint32_t* b0, uint32_t* b1) {
    for (uint64_t i = 0; i < n; ++i) {
        b0[i] = bucket_of(policy, 0, keys[i], num_buckets);
        b1[i] = bucket_of(policy, 1, keys[i], num_buckets);
    }
}

// ---- 2. generators --------------------------------------------------------------------------
uint64_t hive_oracle_sm64(uint64_t* state) { return sm64(*state); }

// Draws n_present unique keys, then n_absent further unique keys that are not among them, from
// one splitmix64 stream seeded with `seed`.  Returns the stream state after the last draw.
uint64_t hive_oracle_gen_keys(uint64_t seed, uint64_t n_present, uint64_t n_absent,
                              uint32_t* present, uint32_t* absent) {
    uint64_t state = seed;
    // keys drawn so far: an open-addressing set (keys are never 0, so 0 marks a free cell) at
    // most half full
    uint64_t cells = 2;
    while (cells < 2 * (n_present + n_absent)) cells <<= 1;
    std::vector<uint32_t> seen(cells, 0u);
    auto fresh = [&](uint32_t k) {
        for (uint64_t c = (k * 0x9E3779B97F4A7C15ull) >> 20;; ++c) {
            uint32_t& cell = seen[c & (cells - 1)];
            if (cell == k) return false;
            if (cell == 0u) {
                cell = k;
                return true;
            }
        }
    };
    uint64_t i = 0;
    while (i < n_present) {
        uint32_t k = draw_key(state);
        if (fresh(k)) present[i++] = k;
    }
    i = 0;
    while (i < n_absent) {
        uint32_t k = draw_key(state);
        if (fresh(k)) absent[i++] = k;
    }
    return state;
}

void hive_oracle_values(const uint32_t* keys, uint64_t n, uint32_t* vals) {
    for (uint64_t i = 0; i < n; ++i) vals[i] = value_of(keys[i]);
}

// Fisher-Yates driven by the splitmix64 stream in *state.
void hive_oracle_shuffle_u32(uint32_t* a, uint64_t n, uint64_t* state) {
    if (n < 2) return;
    for (uint64_t i = n - 1; i > 0; --i) {
        uint64_t j = sm64(*state) % (i + 1);
        std::swap(a[i], a[j]);
    }
}

// Lookup set: n_present keys sampled without replacement from inserted[0, n) by a partial
// Fisher-Yates (i = 0 .. n_present-1, j = i + sm64 % (n - i)), then absent[0, n_absent), then a
// full Fisher-Yates shuffle of the concatenation.
void hive_oracle_lookup_set(const uint32_t* inserted, uint64_t n, const uint32_t* absent, uint64_t n_present,
                            uint64_t n_absent, uint64_t* state, uint32_t* out) {
    std::vector<uint32_t> pick(inserted, inserted + n);
    for (uint64_t i = 0; i < n_present && i < n; ++i) {
        uint64_t j = i + sm64(*state) % (n - i);
        std::swap(pick[i], pick[j]);
    }
    for (uint64_t i = 0; i < n_present; ++i) out[i] = pick[i];
    for (uint64_t i = 0; i < n_absent; ++i) out[n_present + i] = absent[i];
    hive_oracle_shuffle_u32(out, n_present + n_absent, state);
}

// ---- 3. unordered_map replay ----------------------------------------------------------------
void* hive_oracle_map_new() { return new ReplayMap(); }
void hive_oracle_map_free(void* h) { delete (ReplayMap*)h; }
void hive_oracle_map_clear(void* h) { ((ReplayMap*)h)->m.clear(); }
uint64_t hive_oracle_map_size(void* h) { return ((ReplayMap*)h)->m.size(); }

// Upsert (S2).  status: 1 inserted, 2 updated, 0 rejected (key 0, S1).  Entries whose
// apply_mask byte is 0 are skipped with status 0 (inserts the table under test reported as
// failed are not replayed).
void hive_oracle_map_insert(void* h, const uint32_t* keys, const uint32_t* vals, uint64_t n,
                            const uint8_t* apply_mask, uint8_t* status) {
    auto& m = ((ReplayMap*)h)->m;
    m.reserve(m.size() + n);
    for (uint64_t i = 0; i < n; ++i) {
        uint8_t st = 0;
        if (keys[i] != 0 && (!apply_mask || apply_mask[i])) {
            auto r = m.insert_or_assign(keys[i], vals[i]);
            st = r.second ? 1 : 2;
        }
        if (status) status[i] = st;
    }
}

void hive_oracle_map_find(void* h, const uint32_t* keys, uint64_t n, uint32_t* vals, uint8_t* found) {
    auto& m = ((ReplayMap*)h)->m;
    for (uint64_t i = 0; i < n; ++i) {
        auto it = keys[i] == 0 ? m.end() : m.find(keys[i]);
        bool f = it != m.end();
        found[i] = f;
        vals[i] = f ? it->second : 0;
    }
}

void hive_oracle_map_erase(void* h, const uint32_t* keys, uint64_t n, uint8_t* status) {
    auto& m = ((ReplayMap*)h)->m;
    for (uint64_t i = 0; i < n; ++i) status[i] = keys[i] != 0 && m.erase(keys[i]) ? 1 : 0;
}

// Mixed ops in array order.  types: 0 insert, 1 lookup, 2 delete, 3 increment, 4 none
// (the numbering of OperationType, include/utils.h:10-16).  Outputs per op: status
// (insert 1/2, lookup 0/1, delete 0/1, increment 0/1) and value (lookup: value found;
// increment: value after the increment; else 0).  Inserts whose apply_mask byte is 0 are
// skipped (status 0).
void hive_oracle_map_apply(void* h, const uint8_t* types, const uint32_t* keys, const uint32_t* vals,
                           uint64_t n, const uint8_t* apply_mask, uint8_t* status, uint32_t* out_vals) {
    auto& m = ((ReplayMap*)h)->m;
    for (uint64_t i = 0; i < n; ++i) {
        uint8_t st = 0;
        uint32_t ov = 0;
        uint32_t k = keys[i];
        if (k != 0) {
            switch (types[i]) {
                case 0:
                    if (!apply_mask || apply_mask[i]) {
                        auto r = m.insert_or_assign(k, vals[i]);
                        st = r.second ? 1 : 2;
                    }
                    break;
                case 1: {
                    auto it = m.find(k);
                    if (it != m.end()) { st = 1; ov = it->second; }
                    break;
                }
                case 2:
                    st = m.erase(k) ? 1 : 0;
                    break;
                case 3: {
                    auto it = m.find(k);
                    if (it != m.end()) { it->second += 1u; st = 1; ov = it->second; }
                    break;
                }
                default:
                    break;
            }
        }
        status[i] = st;
        out_vals[i] = ov;
    }
}

// The per-key serialisation check of a run of concurrent launches (see SerialSearch).
// ops: types / keys / vals with launch[i] = the index of the launch op i ran in; status /
// out_vals: what the table under test returned; fin_keys / fin_vals: its contents after the run,
// sorted by key.  The map holds the state before the run.  Key 0 is never stored, so its ops
// must all report status 0.  A key whose ops all ran in one launch and include no increment is
// decided by serial_closed_form, any other by the search.  Returns the number of keys with no
// valid order (a key whose launch holds more than 63 of its ops, or whose search exceeds 2^22
// steps, counts as one); *first_bad = the lowest op index of such a key.  When it returns 0 the
// map holds the final state of every key the run touched.
uint64_t hive_oracle_map_check_serial(void* h, const uint8_t* types, const uint32_t* keys, const uint32_t* vals,
                                      const uint32_t* launch, uint64_t n, const uint8_t* status,
                                      const uint32_t* out_vals, const uint32_t* fin_keys, const uint32_t* fin_vals,
                                      uint64_t n_fin, uint64_t* first_bad) {
    auto& m = ((ReplayMap*)h)->m;
    std::vector<uint64_t> idx(n);
    for (uint64_t i = 0; i < n; ++i) idx[i] = i;
    std::sort(idx.begin(), idx.end(), [&](uint64_t a, uint64_t b) {
        if (keys[a] != keys[b]) return keys[a] < keys[b];
        if (launch[a] != launch[b]) return launch[a] < launch[b];
        return a < b;
    });
    uint64_t bad = 0;
    if (first_bad) *first_bad = ~0ull;
    std::vector<std::pair<uint32_t, std::pair<bool, uint32_t>>> finals;
    std::vector<std::vector<SerialOp>> groups;
    for (uint64_t s = 0; s < n;) {
        const uint32_t k = keys[idx[s]];
        uint64_t e = s;
        uint64_t low = idx[s];
        groups.clear();
        while (e < n && keys[idx[e]] == k) {
            const uint64_t i = idx[e];
            low = std::min(low, i);
            if (e == s || launch[i] != launch[idx[e - 1]]) groups.emplace_back();
            groups.back().push_back(SerialOp{types[i], vals ? vals[i] : 0u, status[i], out_vals ? out_vals[i] : 0u});
            ++e;
        }
        bool ok = true;
        for (const auto& G : groups) ok = ok && G.size() <= 63;
        bool fin_present = false;
        uint32_t fin_value = 0;
        if (k != 0) {
            const uint32_t* it = std::lower_bound(fin_keys, fin_keys + n_fin, k);
            if (it != fin_keys + n_fin && *it == k) {
                fin_present = true;
                fin_value = fin_vals[it - fin_keys];
            }
        }
        bool present = false;
        uint32_t value = 0;
        if (k != 0) {
            auto mt = m.find(k);
            if (mt != m.end()) {
                present = true;
                value = mt->second;
            }
        }
        if (ok && groups.size() == 1 && !has_increment(groups[0])) {
            ok = serial_closed_form(groups[0], present, value, fin_present, fin_value) == 1;
        } else if (ok) {
            SerialSearch srch{&groups, fin_present, fin_value, 1ll << 22, {}};
            ok = srch.run(0, 0, present, value);
        }
        if (!ok) {
            ++bad;
            if (first_bad && low < *first_bad) *first_bad = low;
        } else if (k != 0) {
            finals.push_back({k, {fin_present, fin_value}});
        }
        s = e;
    }
    if (!bad)
        for (const auto& f : finals) {
            if (f.second.first) m[f.first] = f.second.second;
            else m.erase(f.first);
        }
    return bad;
}

// Self-test of the closed form against the search on random single-launch groups of up to
// max_ops ops without increments (random results: mostly inconsistent, plus results of a random
// order of the ops).  Returns the number of groups on which the two disagree.
uint64_t hive_oracle_serial_selftest(uint64_t seed, uint64_t trials, int max_ops) {
    uint64_t st = seed, disagree = 0;
    auto rnd = [&](uint64_t m) { return sm64(st) % m; };
    for (uint64_t t = 0; t < trials; ++t) {
        const int m = 1 + (int)rnd((uint64_t)max_ops);
        std::vector<SerialOp> G(m);
        bool present = rnd(2), fin_present;
        uint32_t value = 1 + (uint32_t)rnd(3), fin_value;
        for (auto& o : G) {
            o.type = (uint8_t)rnd(3);
            o.val = 1 + (uint32_t)rnd(3);
        }
        if (rnd(2)) {  // results of one random order
            std::vector<int> ord(m);
            for (int i = 0; i < m; ++i) ord[i] = i;
            for (int i = m - 1; i > 0; --i) std::swap(ord[i], ord[rnd((uint64_t)i + 1)]);
            bool p = present;
            uint32_t v = value;
            for (int i : ord) {
                SerialOp& o = G[i];
                o.ov = 0;
                if (o.type == 0) {
                    o.st = p ? 2 : 1;
                    p = true;
                    v = o.val;
                } else if (o.type == 1) {
                    o.st = p;
                    o.ov = p ? v : 0;
                } else {
                    o.st = p;
                    p = false;
                }
            }
            fin_present = p;
            fin_value = p ? v : 0;
        } else {  // arbitrary results
            for (auto& o : G) {
                o.st = (uint8_t)rnd(3);
                o.ov = o.type == 1 && o.st == 1 ? 1 + (uint32_t)rnd(3) : 0;
            }
            fin_present = rnd(2);
            fin_value = fin_present ? 1 + (uint32_t)rnd(3) : 0;
        }
        std::vector<std::vector<SerialOp>> groups{G};
        SerialSearch srch{&groups, fin_present, fin_value, 1ll << 30, {}};
        const bool a = srch.run(0, 0, present, value);
        const bool b = serial_closed_form(G, present, value, fin_present, fin_value) == 1;
        disagree += a != b;
    }
    return disagree;
}

// Writes the key->value set sorted by key; returns its size.
uint64_t hive_oracle_map_dump(void* h, uint32_t* keys, uint32_t* vals, uint64_t cap) {
    auto& m = ((ReplayMap*)h)->m;
    std::vector<std::pair<uint32_t, uint32_t>> v(m.begin(), m.end());
    std::sort(v.begin(), v.end());
    uint64_t n = std::min<uint64_t>(cap, v.size());
    for (uint64_t i = 0; i < n; ++i) { keys[i] = v[i].first; vals[i] = v[i].second; }
    return v.size();
}

// ---- 4. multithreaded CPU table -------------------------------------------------------------
void* hive_oracle_cpu_new(int policy, uint64_t capacity_slots, int max_evictions) {
    uint64_t nb = (capacity_slots + kSlots - 1) / kSlots;
    if (nb == 0) nb = 1;
    return new CpuTable(policy, (uint32_t)nb, max_evictions);
}
void hive_oracle_cpu_free(void* h) { delete (CpuTable*)h; }
uint64_t hive_oracle_cpu_failed(void* h) { return ((CpuTable*)h)->failed.load(); }

// Bulk insert with `threads` std::threads; returns wall seconds (steady_clock).
double hive_oracle_cpu_insert(void* h, const uint32_t* keys, const uint32_t* vals, uint64_t n,
                              uint8_t* status, int threads) {
    CpuTable* t = (CpuTable*)h;
    return run_threads(threads, n, [&](uint64_t i) {
        int r = t->insert(keys[i], vals[i]);
        if (status) status[i] = (uint8_t)r;
    });
}

double hive_oracle_cpu_find(void* h, const uint32_t* keys, uint64_t n, uint32_t* vals, uint8_t* found,
                            int threads) {
    CpuTable* t = (CpuTable*)h;
    return run_threads(threads, n, [&](uint64_t i) {
        uint32_t v = 0;
        bool f = t->find(keys[i], &v);
        if (vals) vals[i] = f ? v : 0;
        if (found) found[i] = f;
    });
}

}  // extern "C"
