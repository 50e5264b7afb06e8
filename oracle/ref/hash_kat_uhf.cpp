// hash_kat_uhf.cpp -- TEST INFRASTRUCTURE (oracle pin).  Prints the reference's plain-C hash
// functions of UniformHashFunction/src/hash_function.cu (linked from the reference tree by
// oracle/build.py).  Each returns its hash modulo PRIME_N = 294967291
// (UniformHashFunction/include/hash_function.h:10); this pins hash2 on the CPU.
//
// Output, one line per key:  key hash1 hash2 cityhash murmurhash   (all mod PRIME_N)
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include "hash_function.h"

static uint64_t mix(uint64_t& x) {
    uint64_t z = (x += 0x9e3779b97f4a7c15ULL);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}

int main(int argc, char** argv) {
    const int n = argc > 1 ? atoi(argv[1]) : 4096;
    uint64_t s = 2024;
    for (int i = 0; i < n; ++i) {
        uint32_t k;
        if (i < 8) {
            const uint32_t edge[8] = {0u, 1u, 2u, 3u, 0x7fffffffu, 0x80000000u, 0xfffffffeu, 0xffffffffu};
            k = edge[i];
        } else {
            k = (uint32_t)mix(s);
        }
        printf("%u %u %u %u %u\n", k, hash1(k), hash2(k), cityhash(k), murmurhash(k));
    }
    return 0;
}
