// hash_kat_inc.cpp -- TEST INFRASTRUCTURE (oracle pin).  Prints the reference's own host-callable
// hash functions from its include/hash.hpp (compiled from the reference tree by oracle/build.py)
// for a deterministic key list, so the oracle's restatement can be checked against them.
//
// Output, one line per key:  key hash1(key) murmurhash(key, M_i)... cityhash(key, M_i)...
// with the moduli M listed on the first line.  hash2's host form in hash.hpp is inline PTX and
// cannot run on the CPU; it is pinned by hash_kat_uhf.cpp (plain-C form) and, on the GPU, by
// hash_dev_kat.cu.
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include "hash.hpp"

static uint64_t mix(uint64_t& x) {  // SplitMix64 step, only to spread the key list
    uint64_t z = (x += 0x9e3779b97f4a7c15ULL);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}

int main(int argc, char** argv) {
    const int n = argc > 1 ? atoi(argv[1]) : 4096;
    const uint32_t mods[] = {1u, 7u, 163840u, 8388608u, 294967291u, 4294967295u};
    const int nm = sizeof(mods) / sizeof(mods[0]);
    printf("M");
    for (int j = 0; j < nm; ++j) printf(" %u", mods[j]);
    printf("\n");
    uint64_t s = 2024;
    for (int i = 0; i < n; ++i) {
        uint32_t k;
        if (i < 8) {
            const uint32_t edge[8] = {0u, 1u, 2u, 3u, 0x7fffffffu, 0x80000000u, 0xfffffffeu, 0xffffffffu};
            k = edge[i];
        } else {
            k = (uint32_t)mix(s);
        }
        printf("%u %u", k, hash1(k));
        for (int j = 0; j < nm; ++j) printf(" %u", murmurhash(k, mods[j]));
        for (int j = 0; j < nm; ++j) printf(" %u", cityhash(k, mods[j]));
        printf("\n");
    }
    return 0;
}
