// hive_serve.cpp -- an open-loop request loop with continuous batching over one Hive table.
//
// The reference has no serving path (its "YCSB" driver is one closed-loop bulk launch,
// src/hashTableBenchmark.cc:434-570).  This loop admits requests by arrival time and keeps the
// GPU fed with batches:
//
//   admit      every request whose arrival time has passed joins the pending queue
//   coalesce   a batch takes up to max_batch pending requests in arrival order and groups them
//              by key: a group whose first request is a lookup needs the key's value before the
//              batch (one device lookup); a group with writes needs one device upsert of its last
//              written value.  Lookups after a write in the same batch are answered from that
//              write, so every result equals the one a one-at-a-time replay in arrival order gives.
//              Each request's answer source (the write that answers it, or its key group) is fixed
//              while the batch is formed, so answering is one pass in request order
//   launch     pinned-host -> device copies on the slot's copy stream; the lookups, then the
//              upserts, on the single compute stream (batches therefore reach the table in
//              arrival order); the results back on the copy stream
//   pipeline   up to `depth` batches are in flight: while the GPU works on one, the next batch is
//              formed, copied and queued.  depth = 1 is the plain loop: one batch at a time
//   answer     a second host thread takes the batches in order as their results reach the host
//              and answers their requests, while this thread forms the next batch: a batch that
//              finishes on the GPU is answered at once instead of after the next formation
//   growth     the load is tracked without touching the device: keys known placed (from the
//              statuses of finished batches) plus every distinct write in flight counted as new.
//              Loads count against the slots of the unsplit level (8 n_lo; see level_slots).
//              Incremental (grow_start > 0): once the load could pass grow_start, the loop sets a
//              target of the next full level and, before each batch, splits the next run of buckets
//              toward it on the compute stream (hive_resize within the reservation queues the
//              split kernel and returns), so batches keep flowing; the run length makes the
//              doubling end within the batches that fit between grow_start and max_load.  At once
//              (fallback): before a batch that could push the load past max_load, the loop drains,
//              recounts, checks free device memory for the next level (cudaMemGetInfo) and
//              grows to it.  When memory does not allow growth, the batch's new keys are refused
//              (status 0) and existing keys still update
//
// Completion time of a request = when its batch's results are on the host and answered.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>

#include "hive_serve.h"

namespace {

using Clock = std::chrono::steady_clock;

// Key -> group index of one batch: open addressing with linear probing over a power-of-two table
// at least twice the batch size, one 16-byte entry per slot (key, group, batch stamp) so a probe
// touches one cache line.  An entry belongs to the current batch iff its stamp equals the batch's
// generation, so starting a batch costs one increment instead of a clear.
class GroupMap {
  public:
    explicit GroupMap(uint32_t max_keys) {
        uint32_t sz = 16;
        while (sz < 2u * max_keys) sz <<= 1;
        mask_ = sz - 1;
        e_.assign(sz, Entry{0u, 0, 0u, 0u});
    }
    void next_batch() {
        if (++gen_ == 0) {  // stamps wrapped: clear once every 2^32 batches
            for (auto& x : e_) x.stamp = 0u;
            gen_ = 1;
        }
    }
    // The group of key k; *added is true when k is new to the batch (its group is then `fresh`).
    int32_t find_or_add(uint32_t k, int32_t fresh, bool* added) {
        uint32_t h = k;
        h ^= h >> 16;
        h *= 0x85ebca6bu;
        h ^= h >> 13;
        h *= 0xc2b2ae35u;
        h ^= h >> 16;
        for (uint32_t i = h & mask_;; i = (i + 1) & mask_) {
            Entry& x = e_[i];
            if (x.stamp != gen_) {
                x = Entry{k, fresh, gen_, 0u};
                *added = true;
                return fresh;
            }
            if (x.key == k) {
                *added = false;
                return x.group;
            }
        }
    }

  private:
    struct Entry {
        uint32_t key;
        int32_t group;
        uint32_t stamp;
        uint32_t pad;
    };
    std::vector<Entry> e_;
    uint32_t mask_ = 0, gen_ = 0;
};

struct Slot {
    cudaStream_t copy = nullptr;
    cudaEvent_t staged = nullptr, done = nullptr;
    // pinned host staging
    uint32_t *h_fkeys = nullptr, *h_ukeys = nullptr, *h_uvals = nullptr, *h_fvals = nullptr;
    uint8_t *h_types = nullptr, *h_ftypes = nullptr, *h_found = nullptr, *h_ust = nullptr;
    // device
    uint32_t *d_fkeys = nullptr, *d_ukeys = nullptr, *d_uvals = nullptr, *d_fvals = nullptr;
    uint8_t *d_ftypes = nullptr, *d_utypes = nullptr, *d_found = nullptr, *d_ust = nullptr;
    // the batch: requests [first, first + count) in arrival order
    uint64_t first = 0, count = 0;
    // how each request is answered: >= 0, a lookup answered by that earlier write of the batch
    // (offset in the batch); < 0, -(g + 1) for key group g (a lookup: the group's device lookup;
    // a write: the group's device upsert)
    std::vector<int32_t> ans;
    std::vector<int32_t> fpos, upos;  // group -> position in the lookup / upsert list, or -1
    uint32_t nf = 0, nu = 0;
    uint64_t new_writes = 0;          // distinct written keys of the batch (possible new keys)
};

// Device bytes per bucket of a table allocation (8 slots, 8 stash entries, fingerprint word,
// lock byte, stash and full bits), rounded up.
constexpr double kBytesPerBucket = 140.0;

// Smallest split step of incremental growth (buckets): below this a step costs more in launch
// overhead than it moves.
constexpr uint64_t kMinGrowStep = 1u << 10;

// Mid-level, a bucket not yet split takes keys of 1/n_lo of the hash space, twice a split
// bucket's share, so the load that bounds placement is keys / (8 n_lo): the capacity that growth
// decisions count is that of the level, and growth targets the next full level (2 n_lo buckets).
uint64_t level_buckets(const hive_info& info) { return (uint64_t)info.base_buckets << info.level; }
double level_slots(const hive_info& info) { return 8.0 * (double)level_buckets(info); }

// Whether the table may grow to `target` buckets: within the reservation always; beyond it when
// free device memory holds the new allocation (the old one stays until the copy is done).
bool growth_admitted(const hive_info& info, uint64_t target) {
    if (target <= info.max_buckets) return true;
    size_t fr = 0, tot = 0;
    if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) return false;
    const double nb_cap = (double)std::max<uint64_t>(target, 2 * info.max_buckets);
    return (double)fr > nb_cap * kBytesPerBucket * 1.05;
}

int alloc_slot(Slot& s, uint32_t cap) {
    if (cudaStreamCreateWithFlags(&s.copy, cudaStreamNonBlocking) != cudaSuccess) return HIVE_ERR_CUDA;
    if (cudaEventCreateWithFlags(&s.staged, cudaEventDisableTiming) != cudaSuccess) return HIVE_ERR_CUDA;
    if (cudaEventCreateWithFlags(&s.done, cudaEventDisableTiming) != cudaSuccess) return HIVE_ERR_CUDA;
    const size_t w = (size_t)cap * 4, b = (size_t)cap;
    if (cudaMallocHost(&s.h_fkeys, w) || cudaMallocHost(&s.h_ukeys, w) || cudaMallocHost(&s.h_uvals, w) ||
        cudaMallocHost(&s.h_fvals, w) || cudaMallocHost(&s.h_types, b) || cudaMallocHost(&s.h_ftypes, b) ||
        cudaMallocHost(&s.h_found, b) || cudaMallocHost(&s.h_ust, b))
        return HIVE_ERR_OOM;
    if (cudaMalloc(&s.d_fkeys, w) || cudaMalloc(&s.d_ukeys, w) || cudaMalloc(&s.d_uvals, w) ||
        cudaMalloc(&s.d_fvals, w) || cudaMalloc(&s.d_ftypes, b) || cudaMalloc(&s.d_utypes, b) ||
        cudaMalloc(&s.d_found, b) || cudaMalloc(&s.d_ust, b))
        return HIVE_ERR_OOM;
    std::memset(s.h_ftypes, HIVE_OP_LOOKUP, b);
    std::memset(s.h_types, HIVE_OP_INSERT, b);
    if (cudaMemcpy(s.d_ftypes, s.h_ftypes, b, cudaMemcpyHostToDevice) ||
        cudaMemcpy(s.d_utypes, s.h_types, b, cudaMemcpyHostToDevice))
        return HIVE_ERR_CUDA;
    return HIVE_OK;
}

void free_slot(Slot& s) {
    cudaFreeHost(s.h_fkeys); cudaFreeHost(s.h_ukeys); cudaFreeHost(s.h_uvals); cudaFreeHost(s.h_fvals);
    cudaFreeHost(s.h_types); cudaFreeHost(s.h_ftypes); cudaFreeHost(s.h_found); cudaFreeHost(s.h_ust);
    cudaFree(s.d_fkeys); cudaFree(s.d_ukeys); cudaFree(s.d_uvals); cudaFree(s.d_fvals);
    cudaFree(s.d_ftypes); cudaFree(s.d_utypes); cudaFree(s.d_found); cudaFree(s.d_ust);
    if (s.staged) cudaEventDestroy(s.staged);
    if (s.done) cudaEventDestroy(s.done);
    if (s.copy) cudaStreamDestroy(s.copy);
}

}  // namespace

extern "C" {

int hive_serve_run(
    hive_table* t, const hive_serve_config* cfg, const uint8_t* types, const uint32_t* keys, const uint32_t* vals,
    const double* arrival_s, uint64_t n, uint32_t* out_vals, uint8_t* out_status, double* done_s,
    hive_serve_stats* stats) {
    if (!t || !cfg || !types || !keys || !vals || !arrival_s || !out_vals || !out_status || !done_s)
        return HIVE_ERR_INVALID_ARG;
    if (cfg->depth < 1 || cfg->depth > 64 || cfg->max_batch < 1) return HIVE_ERR_INVALID_ARG;
    if (!(cfg->grow_start >= 0.0) || (cfg->grow_start > 0.0 && !(cfg->grow_start < cfg->max_load)))
        return HIVE_ERR_INVALID_ARG;
    hive_serve_stats st{};
    const uint32_t cap = cfg->max_batch;
    std::vector<Slot> slots(cfg->depth);
    int rc = HIVE_OK;
    cudaStream_t compute = nullptr;
    if (cudaStreamCreateWithFlags(&compute, cudaStreamNonBlocking) != cudaSuccess) return HIVE_ERR_CUDA;
    for (auto& s : slots)
        if ((rc = alloc_slot(s, cap))) break;
    hive_info info{};
    // shared with the answering thread
    std::atomic<uint64_t> live_done{cfg->live_keys};  // keys in the table after the answered batches
    std::atomic<uint64_t> pending_new{0};             // possible new keys of the batches in flight
    std::atomic<uint64_t> launched{0}, answered{0};   // batches queued / answered (in order)
    std::atomic<uint64_t> finished{0};                // requests answered
    std::atomic<int> answer_rc{HIVE_OK};
    uint64_t grow_target = 0, grow_step = 0;  // incremental growth: target buckets, buckets per step
    uint64_t grow_refused_at = 0;             // bucket count at which growth found no memory

    GroupMap gid(cap);
    std::vector<uint32_t> g_key;    // group -> key
    std::vector<int32_t> g_lastw;   // group -> offset of its latest write so far, or -1
    std::vector<uint8_t> g_look;    // group -> its first request is a lookup
    // Requests are admitted in arrival order, so the pending ones are always [pend, next).
    uint64_t pend = 0, next = 0;
    const auto t0 = Clock::now();
    auto now_s = [&] { return std::chrono::duration<double>(Clock::now() - t0).count(); };

    auto finish = [&](Slot& s) {
        const double ta = now_s();
        // answers of the batch, in request order, from the sources fixed when it was formed
        for (uint64_t j = 0; j < s.count; ++j) {
            const uint64_t r = s.first + j;
            const int32_t a = s.ans[j];
            if (types[r] == HIVE_OP_LOOKUP) {
                if (a >= 0) {
                    out_vals[r] = vals[s.first + a];
                    out_status[r] = 1;
                } else {
                    const int32_t f = s.fpos[-a - 1];
                    out_status[r] = s.h_found[f];
                    out_vals[r] = s.h_found[f] ? s.h_fvals[f] : 0u;
                }
            } else {
                const uint8_t us = s.h_ust[s.upos[-a - 1]];
                out_status[r] = (us != HIVE_ST_FAIL && us != HIVE_ST_ERROR) ? 1 : 0;
                out_vals[r] = 0;
            }
        }
        uint64_t placed_new = 0;
        for (uint32_t u = 0; u < s.nu; ++u) placed_new += s.h_ust[u] == HIVE_ST_INSERTED || s.h_ust[u] == HIVE_ST_STASHED;
        live_done.fetch_add(placed_new);
        pending_new.fetch_sub(s.new_writes);
        const double td = now_s();
        std::fill(done_s + s.first, done_s + s.first + s.count, td);
        st.answer_s += now_s() - ta;
        finished.fetch_add(s.count, std::memory_order_release);
    };

    // The answering thread: takes the queued batches in order as their results reach the host and
    // answers them, while this thread forms and queues the next ones (different batches write
    // different output ranges).
    std::atomic<bool> stop{false};
    std::thread answerer([&] {
        for (;;) {
            const uint64_t a = answered.load(std::memory_order_acquire);
            if (a < launched.load(std::memory_order_acquire)) {
                Slot& s = slots[a % slots.size()];
                cudaError_t q;
                for (int spin = 0; (q = cudaEventQuery(s.done)) == cudaErrorNotReady; ++spin)
                    if ((spin & 63) == 63) std::this_thread::yield();
                if (q != cudaSuccess) {
                    answer_rc.store(HIVE_ERR_CUDA);
                    return;
                }
                finish(s);
                answered.store(a + 1, std::memory_order_release);
            } else if (stop.load(std::memory_order_acquire)) {
                return;
            } else {
                std::this_thread::yield();
            }
        }
    });

    auto drain = [&] {
        while (answered.load(std::memory_order_acquire) < launched.load(std::memory_order_relaxed))
            if (answer_rc.load()) return answer_rc.load();
        return answer_rc.load();
    };

    while (!rc && finished.load(std::memory_order_acquire) < n) {
        if ((rc = answer_rc.load())) break;
        // admit arrivals
        const double tn = now_s();
        while (next < n && arrival_s[next] <= tn) ++next;
        const uint64_t in_flight = launched.load(std::memory_order_relaxed) - answered.load(std::memory_order_acquire);
        if (pend == next || in_flight == slots.size()) {
            if (pend == next && next < n && in_flight == 0) {
                // idle until the next arrival
                while (now_s() < arrival_s[next]) {
                }
            }
            st.idle_s += now_s() - tn;
            continue;
        }
        // form a batch
        const double tf = now_s();
        Slot& s = slots[launched.load(std::memory_order_relaxed) % slots.size()];
        const uint64_t take = std::min<uint64_t>(next - pend, cap);
        s.first = pend;
        s.count = take;
        pend += take;
        // coalesce by key: a group whose first request is a lookup needs one device lookup; a group
        // with writes needs one device upsert of its last written value; a lookup after a write of
        // its key in the batch is answered from that write
        gid.next_batch();
        s.ans.resize(take);
        g_key.clear();
        g_lastw.clear();
        g_look.clear();
        uint64_t new_writes = 0;
        for (uint64_t j = 0; j < take; ++j) {
            const uint64_t r = s.first + j;
            bool added;
            const int32_t g = gid.find_or_add(keys[r], (int32_t)g_key.size(), &added);
            const bool lookup = types[r] == HIVE_OP_LOOKUP;
            if (added) {
                g_key.push_back(keys[r]);
                g_lastw.push_back(-1);
                g_look.push_back(lookup);
            }
            if (lookup) {
                s.ans[j] = g_lastw[g] >= 0 ? g_lastw[g] : -(g + 1);
            } else {
                if (g_lastw[g] < 0) ++new_writes;
                g_lastw[g] = (int32_t)j;
                s.ans[j] = -(g + 1);
            }
        }
        const size_t ng = g_key.size();
        s.fpos.resize(ng);
        s.upos.resize(ng);
        s.nf = s.nu = 0;
        for (size_t g = 0; g < ng; ++g) {
            if (g_look[g]) {
                s.h_fkeys[s.nf] = g_key[g];
                s.fpos[g] = (int32_t)s.nf++;
            } else {
                s.fpos[g] = -1;
            }
            if (g_lastw[g] >= 0) {
                s.h_ukeys[s.nu] = g_key[g];
                s.h_uvals[s.nu] = vals[s.first + g_lastw[g]];
                s.upos[g] = (int32_t)s.nu++;
            } else {
                s.upos[g] = -1;
            }
        }
        // growth: keep the load factor under max_load counting every write in flight as a new key
        if (cfg->max_load > 0.0 && new_writes) {
            hive_get_info(t, &info);
            const uint64_t est = live_done + pending_new + new_writes;
            if (cfg->grow_start > 0.0) {
                if (!grow_target && info.num_buckets != grow_refused_at &&
                    (double)est > cfg->grow_start * level_slots(info)) {
                    const uint64_t target = 2 * level_buckets(info);
                    if (growth_admitted(info, target)) {
                        // batches that fit between grow_start and max_load of the level; the
                        // doubling is spread over half of them
                        const double room = (cfg->max_load - cfg->grow_start) * level_slots(info);
                        const double batches = std::max(1.0, std::floor(room / (double)cap / 2.0));
                        grow_target = target;
                        grow_step = std::max<uint64_t>(kMinGrowStep,
                                                       (uint64_t)std::ceil((target - info.num_buckets) / batches));
                    } else {
                        grow_refused_at = info.num_buckets;
                    }
                }
                if (grow_target) {
                    const uint64_t to = std::min(grow_target, info.num_buckets + grow_step);
                    if ((rc = hive_resize(t, to * 8, compute))) {
                        if (rc == HIVE_ERR_CUDA) break;
                        rc = HIVE_OK;  // no memory for it after all: leave it to the check below
                        grow_refused_at = info.num_buckets;
                        grow_target = 0;
                    } else {
                        ++st.grow_steps;
                        if (to == grow_target) {
                            grow_target = 0;
                            ++st.resizes;
                        }
                    }
                    hive_get_info(t, &info);
                }
            }
            const double cap_slots = level_slots(info);
            if ((double)est > cfg->max_load * cap_slots) {
                if ((rc = drain())) break;
                uint64_t sz = 0;
                if ((rc = hive_size(t, &sz, compute))) break;
                live_done = sz;
                if ((double)(live_done + new_writes) > cfg->max_load * cap_slots) {
                    ++st.drains;
                    const uint64_t target = 2 * level_buckets(info);
                    if (info.num_buckets != grow_refused_at && growth_admitted(info, target) &&
                        hive_resize(t, target * 8, compute) == HIVE_OK) {
                        ++st.resizes;
                        grow_target = 0;
                    } else {
                        grow_refused_at = info.num_buckets;
                        st.refused += new_writes;  // the batch still runs; inserts that find no room fail
                    }
                }
            }
        }
        pending_new += new_writes;
        s.new_writes = new_writes;
        // launch
        const double tl = now_s();
        st.form_s += tl - tf;
        if (s.nf && cudaMemcpyAsync(s.d_fkeys, s.h_fkeys, (size_t)s.nf * 4, cudaMemcpyHostToDevice, s.copy)) rc = HIVE_ERR_CUDA;
        if (s.nu && (cudaMemcpyAsync(s.d_ukeys, s.h_ukeys, (size_t)s.nu * 4, cudaMemcpyHostToDevice, s.copy) ||
                     cudaMemcpyAsync(s.d_uvals, s.h_uvals, (size_t)s.nu * 4, cudaMemcpyHostToDevice, s.copy)))
            rc = HIVE_ERR_CUDA;
        if (rc) break;
        cudaEventRecord(s.staged, s.copy);
        cudaStreamWaitEvent(compute, s.staged, 0);
        // coalescing leaves each key once per list
        const uint32_t hints = HIVE_HINT_NO_DELETES | HIVE_HINT_UNIQUE_KEYS;
        if (s.nf && (rc = hive_apply_ops(t, s.d_ftypes, s.d_fkeys, nullptr, s.nf, s.d_found, s.d_fvals, hints,
                                         compute)))
            break;
        if (s.nu && (rc = hive_apply_ops(t, s.d_utypes, s.d_ukeys, s.d_uvals, s.nu, s.d_ust, nullptr, hints,
                                         compute)))
            break;
        cudaEventRecord(s.done, compute);
        cudaStreamWaitEvent(s.copy, s.done, 0);
        if (s.nf && (cudaMemcpyAsync(s.h_found, s.d_found, s.nf, cudaMemcpyDeviceToHost, s.copy) ||
                     cudaMemcpyAsync(s.h_fvals, s.d_fvals, (size_t)s.nf * 4, cudaMemcpyDeviceToHost, s.copy)))
            rc = HIVE_ERR_CUDA;
        if (s.nu && cudaMemcpyAsync(s.h_ust, s.d_ust, s.nu, cudaMemcpyDeviceToHost, s.copy)) rc = HIVE_ERR_CUDA;
        cudaEventRecord(s.done, s.copy);
        st.batches++;
        st.launch_s += now_s() - tl;
        st.device_lookups += s.nf;
        st.device_upserts += s.nu;
        launched.fetch_add(1, std::memory_order_release);
    }
    if (!rc) rc = drain();
    stop.store(true, std::memory_order_release);
    answerer.join();
    if (!rc) rc = answer_rc.load();
    if (!rc) rc = hive_check(t, compute);
    st.wall_s = now_s();
    if (stats) *stats = st;
    cudaStreamSynchronize(compute);
    for (auto& s : slots) free_slot(s);
    cudaStreamDestroy(compute);
    return rc;
}

}  // extern "C"
