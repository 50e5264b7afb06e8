// hive_workload.cpp -- seeded synthetic workloads for the Hive benchmarks (host C++).
//
// The reference generates its workloads in src/hashTableBenchmark.cc (keys from a
// std::random_device-seeded mt19937_64, so runs are not reproducible, :62-100, :156-272,
// :275-432).  These generators are deterministic instead, built on the SplitMix64 step of the
// reference's include/zipf_distribution.h:10-16:
//
//   key draw      k = 1 + (uint32)(sm64(state) % (2^32 - 3))   (0 and the top two values excluded)
//   unique keys   draw until n distinct keys are found; absent keys continue the same stream and
//                 skip every key drawn before
//   values        v(k) = low 32 bits of sm64(s) with s = k
//   shuffle       Fisher-Yates, i = n-1 .. 1, j = sm64(state) % (i + 1)
//   lookup set    partial Fisher-Yates picks n_present inserted keys (i = 0 .. n_present-1,
//                 j = i + sm64(state) % (n - i)), then the first n_absent absent keys are
//                 appended and the whole set is shuffled
//   batches       see hive_wl_mixed_batch
#include <algorithm>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <thread>
#include <unordered_set>
#include <vector>

namespace {

inline uint64_t sm64(uint64_t& x) {
    uint64_t z = (x += 0x9e3779b97f4a7c15ULL);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}

constexpr uint64_t kKeySpan = 4294967293ULL;
inline uint32_t draw_key(uint64_t& s) { return 1u + (uint32_t)(sm64(s) % kKeySpan); }

// Membership over the whole 32-bit key space: a 512 MiB bitmap for big draws, a hash set for
// small ones.
struct Seen {
    std::vector<uint64_t> bits;
    std::unordered_set<uint32_t> set;
    bool use_bits;
    explicit Seen(uint64_t expected) : use_bits(expected > (1u << 21)) {
        if (use_bits) bits.assign((1ull << 32) / 64, 0);
        else set.reserve(expected * 2);
    }
    bool insert(uint32_t k) {
        if (!use_bits) return set.insert(k).second;
        uint64_t& w = bits[k >> 6];
        const uint64_t m = 1ull << (k & 63);
        if (w & m) return false;
        w |= m;
        return true;
    }
};

template <typename F>
void parallel_for(uint64_t n, F&& f) {
    unsigned t = std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
    if (n < (1u << 16)) t = 1;
    std::vector<std::thread> pool;
    for (unsigned i = 0; i < t; ++i) {
        uint64_t lo = n * i / t, hi = n * (i + 1) / t;
        pool.emplace_back([lo, hi, &f] {
            for (uint64_t j = lo; j < hi; ++j) f(j);
        });
    }
    for (auto& p : pool) p.join();
}

}  // namespace

extern "C" {

uint64_t hive_wl_sm64(uint64_t* state) { return sm64(*state); }

uint64_t hive_wl_gen_keys(uint64_t seed, uint64_t n_present, uint64_t n_absent, uint32_t* present,
                          uint32_t* absent) {
    uint64_t s = seed;
    Seen seen(n_present + n_absent);
    for (uint64_t i = 0; i < n_present;) {
        uint32_t k = draw_key(s);
        if (seen.insert(k)) present[i++] = k;
    }
    for (uint64_t i = 0; i < n_absent;) {
        uint32_t k = draw_key(s);
        if (seen.insert(k)) absent[i++] = k;
    }
    return s;
}

void hive_wl_values(const uint32_t* keys, uint64_t n, uint32_t* vals) {
    parallel_for(n, [&](uint64_t i) {
        uint64_t s = keys[i];
        vals[i] = (uint32_t)sm64(s);
    });
}

void hive_wl_shuffle(uint32_t* a, uint64_t n, uint64_t* state) {
    if (n < 2) return;
    for (uint64_t i = n - 1; i > 0; --i) std::swap(a[i], a[sm64(*state) % (i + 1)]);
}

// out[0 .. n_present + n_absent): n_present keys sampled without replacement from
// inserted[0 .. n), then absent[0 .. n_absent), shuffled.  `inserted` is not modified.
void hive_wl_lookup_set(const uint32_t* inserted, uint64_t n, const uint32_t* absent, uint64_t n_present,
                        uint64_t n_absent, uint64_t* state, uint32_t* out) {
    std::vector<uint32_t> pick(inserted, inserted + n);
    for (uint64_t i = 0; i < n_present && i < n; ++i) std::swap(pick[i], pick[i + sm64(*state) % (n - i)]);
    std::memcpy(out, pick.data(), n_present * 4);
    std::memcpy(out + n_present, absent, n_absent * 4);
    hive_wl_shuffle(out, n_present + n_absent, state);
}

}  // extern "C"
