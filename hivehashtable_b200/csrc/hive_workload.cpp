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
#include <cmath>
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

// ---- mixed batches ---------------------------------------------------------------------------
// Keys of a mixed-batch stream are key(i) = mix(mix(i + s0) ^ s1) for an index i: mix is the
// MurmurHash3 32-bit finaliser, a bijection, so distinct indices give distinct keys with no
// membership test; indices whose key is 0, 2^32-2 or 2^32-1 are skipped.  Inserted keys take
// indices 0, 1, 2, ... in order (the prefill first); absent lookups take indices from 2^31 up,
// which are never inserted.  Batch sizes are floor(2^U), U uniform in [log_lo, log_hi), drawn
// from the size stream (state = seed); op contents come from the content stream
// (state = seed ^ 0xD1B54A32D192ED03).  A batch of size s holds s/2 inserts of new keys,
// 4s/10 lookups (round(0.8 * lookups) of live keys, the rest absent) and the remaining deletes
// of live keys; no key gets two ops in one batch and lookups and deletes are disjoint.  The
// batch is then shuffled (Fisher-Yates on the content stream).
}  // extern "C"

namespace {

inline uint32_t fmix32(uint32_t h) {
    h ^= h >> 16;
    h *= 0x85ebca6bu;
    h ^= h >> 13;
    h *= 0xc2b2ae35u;
    h ^= h >> 16;
    return h;
}

struct KeySpace {
    uint32_t s0, s1;
    explicit KeySpace(uint64_t seed) {
        uint64_t s = seed ^ 0x6A09E667F3BCC909ULL;
        s0 = (uint32_t)sm64(s);
        s1 = (uint32_t)sm64(s);
    }
    uint32_t key(uint32_t i) const { return fmix32(fmix32(i + s0) ^ s1); }
    static bool valid(uint32_t k) { return k != 0u && k < 0xFFFFFFFEu; }
};

// Index stream that skips indices mapping to a reserved key.
struct IndexStream {
    const KeySpace& ks;
    uint32_t next;
    IndexStream(const KeySpace& k, uint32_t start) : ks(k), next(start) {}
    uint32_t take() {
        while (!KeySpace::valid(ks.key(next))) ++next;
        return next++;
    }
};

uint64_t batch_size(uint64_t& s, double lo, double hi) {
    const double u = lo + (hi - lo) * ((sm64(s) >> 11) * (1.0 / 9007199254740992.0));
    uint64_t n = (uint64_t)std::floor(std::exp2(u));
    return n < 1 ? 1 : n;
}

}  // namespace

extern "C" {

// Sizes of n_batches batches; returns their sum.
uint64_t hive_wl_mixed_plan(uint64_t seed, uint64_t n_batches, double log_lo, double log_hi, uint64_t* sizes) {
    uint64_t s = seed, tot = 0;
    for (uint64_t b = 0; b < n_batches; ++b) {
        const uint64_t n = batch_size(s, log_lo, log_hi);
        if (sizes) sizes[b] = n;
        tot += n;
    }
    return tot;
}

}  // extern "C"

// ---- served requests ---------------------------------------------------------------------------
// Zipfian ranks with the closed-form sampler of Gray et al., "Quickly Generating Billion-Record
// Synthetic Databases" (SIGMOD 1994): with zeta(n) = sum_{i=1..n} i^-theta,
// alpha = 1/(1-theta), eta = (1 - (2/n)^(1-theta)) / (1 - zeta(2)/zeta(n)), a uniform u gives
// rank 0 if u*zeta(n) < 1, rank 1 if u*zeta(n) < 1 + 2^-theta, else floor(n * (eta*u - eta + 1)^alpha).
// Records are indices 0 .. n_records-1 of the key bijection above (seed) -- the preload; request
// mixes (mix): 0 = 50 % lookup / 50 % update, 1 = 95 / 5, 2 = 100 % lookup, 3 = 95 % lookup /
// 5 % inserts of new records with lookups Zipf-distributed over the records newest first.
// Types: 1 lookup, 0 insert (an update of an existing record or a new record); update values
// are the low 32 bits of sm64(key ^ (request index << 32)).
namespace {
struct Zipf {
    double theta, zetan, zeta2, alpha, eta, half_pow;
    uint64_t n;
    static double zeta(uint64_t n, double theta, double from = 0.0, uint64_t from_n = 0) {
        double z = from;
        for (uint64_t i = from_n + 1; i <= n; ++i) z += std::pow((double)i, -theta);
        return z;
    }
    Zipf(uint64_t n_, double th) : theta(th), n(n_) {
        zetan = zeta(n, theta);
        zeta2 = 1.0 + std::pow(2.0, -theta);
        alpha = 1.0 / (1.0 - theta);
        half_pow = std::pow(0.5, theta);
        set_eta();
    }
    void set_eta() { eta = (1.0 - std::pow(2.0 / (double)n, 1.0 - theta)) / (1.0 - zeta2 / zetan); }
    void grow_to(uint64_t n2) {  // zeta extended incrementally for the newest-first mix
        zetan = zeta(n2, theta, zetan, n);
        n = n2;
        set_eta();
    }
    uint64_t sample(double u) const {
        const double uz = u * zetan;
        if (uz < 1.0) return 0;
        if (uz < 1.0 + half_pow) return 1;
        uint64_t r = (uint64_t)((double)n * std::pow(eta * u - eta + 1.0, alpha));
        return r < n ? r : n - 1;
    }
};
inline double unit(uint64_t& s) { return (sm64(s) >> 11) * (1.0 / 9007199254740992.0); }
}  // namespace

extern "C" {

// preload_keys[n_records]; types/keys/vals[n_requests].
void hive_wl_served(uint64_t seed, uint64_t n_records, uint64_t n_requests, int mix, double theta,
                    uint32_t* preload_keys, uint8_t* types, uint32_t* keys, uint32_t* vals) {
    KeySpace ks(seed);
    IndexStream ins(ks, 0u);
    std::vector<uint32_t> rec(n_records);
    for (uint64_t r = 0; r < n_records; ++r) {
        rec[r] = ins.take();
        preload_keys[r] = ks.key(rec[r]);
    }
    Zipf z(n_records, theta);
    uint64_t st = seed ^ 0x9E3779B97F4A7C15ULL;
    const double read_frac = mix == 0 ? 0.5 : mix == 2 ? 1.0 : 0.95;
    uint64_t total = n_records;
    for (uint64_t i = 0; i < n_requests; ++i) {
        const bool read = unit(st) < read_frac;
        uint32_t key;
        if (mix == 3 && !read) {
            const uint32_t idx = ins.take();  // a new record
            rec.push_back(idx);
            ++total;
            z.grow_to(total);
            key = ks.key(idx);
            types[i] = 0;
        } else {
            const uint64_t rank = z.sample(unit(st));
            const uint64_t r = mix == 3 ? total - 1 - rank : rank;  // newest first for mix 3
            key = ks.key(rec[r]);
            types[i] = read ? 1 : 0;
        }
        keys[i] = key;
        uint64_t s = (uint64_t)key ^ (i << 32);
        vals[i] = (uint32_t)sm64(s);
    }
}

}  // extern "C"

extern "C" {

// prefill_keys[prefill_n]: the keys inserted before the batches (indices 0 .. prefill_n-1).
// types/keys/vals[total]: the batches back to back; offsets[n_batches + 1].
// Returns the number of live keys after the last batch.
uint64_t hive_wl_mixed_fill(uint64_t seed, uint64_t prefill_n, uint64_t n_batches, double log_lo, double log_hi,
                            uint32_t* prefill_keys, uint8_t* types, uint32_t* keys, uint32_t* vals,
                            uint64_t* offsets) {
    KeySpace ks(seed);
    IndexStream ins(ks, 0u), abs_(ks, 0x80000000u);
    uint64_t size_state = seed, st = seed ^ 0xD1B54A32D192ED03ULL;
    std::vector<uint32_t> live;      // indices of live keys
    std::vector<uint32_t> pos;       // pos[i] = position of index i in live
    std::vector<uint32_t> touched;   // touched[i] = 1 + last batch that used index i
    live.reserve(prefill_n);
    auto grow = [&](uint32_t i) {
        if (i >= pos.size()) {
            size_t n = std::max<size_t>((size_t)i + 1, pos.size() * 2);
            pos.resize(n, 0xFFFFFFFFu);
            touched.resize(n, 0u);
        }
    };
    for (uint64_t j = 0; j < prefill_n; ++j) {
        const uint32_t i = ins.take();
        grow(i);
        pos[i] = (uint32_t)live.size();
        live.push_back(i);
        prefill_keys[j] = ks.key(i);
    }
    uint64_t o = 0;
    offsets[0] = 0;
    for (uint64_t b = 0; b < n_batches; ++b) {
        const uint64_t n = batch_size(size_state, log_lo, log_hi);
        const uint64_t ni = n / 2, nl = n * 4 / 10, nd = n - ni - nl;
        const uint64_t nlp = (uint64_t)std::llround(0.8 * (double)nl);
        const uint32_t tag = (uint32_t)b + 1;
        const uint64_t start = o;
        auto pick_live = [&]() -> uint32_t {
            for (;;) {
                const uint32_t i = live[sm64(st) % live.size()];
                if (touched[i] != tag) {
                    touched[i] = tag;
                    return i;
                }
            }
        };
        std::vector<uint32_t> dels, news;
        for (uint64_t j = 0; j < nlp && !live.empty(); ++j) {
            types[o] = 1;
            keys[o++] = ks.key(pick_live());
        }
        for (uint64_t j = nlp; j < nl; ++j) {
            types[o] = 1;
            keys[o++] = ks.key(abs_.take());
        }
        for (uint64_t j = 0; j < nd && !live.empty(); ++j) {
            const uint32_t i = pick_live();
            dels.push_back(i);
            types[o] = 2;
            keys[o++] = ks.key(i);
        }
        for (uint64_t j = 0; j < ni; ++j) {
            const uint32_t i = ins.take();
            grow(i);
            touched[i] = tag;
            news.push_back(i);
            types[o] = 0;
            keys[o++] = ks.key(i);
        }
        // the batch's effect on the live set: deletes leave, inserts join
        for (uint32_t i : dels) {
            const uint32_t p = pos[i], last = live.back();
            live[p] = last;
            pos[last] = p;
            live.pop_back();
            pos[i] = 0xFFFFFFFFu;
        }
        for (uint32_t i : news) {
            pos[i] = (uint32_t)live.size();
            live.push_back(i);
        }
        // shuffle the batch (types and keys together), then attach values v(k)
        for (uint64_t j = o - start; j > 1; --j) {
            const uint64_t r = sm64(st) % j;
            std::swap(types[start + j - 1], types[start + r]);
            std::swap(keys[start + j - 1], keys[start + r]);
        }
        for (uint64_t j = start; j < o; ++j) {
            uint64_t s = keys[j];
            vals[j] = (uint32_t)sm64(s);
        }
        offsets[b + 1] = o;
    }
    return live.size();
}

}  // extern "C"
