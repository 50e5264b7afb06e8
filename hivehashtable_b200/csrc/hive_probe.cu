// hive_probe.cu -- random-bucket bandwidth probes for the roofline of the Hive kernels.
//
// The table's hot loop is a random 64 B bucket read (two 32 B sectors) followed, for an insert,
// by an 8 B CAS into that bucket.  These probes time exactly those access patterns over a buffer
// of the caller's size with no hashing, matching or control flow, so their throughput is the
// ceiling the table kernels are measured against (the plain copy bandwidth is not: sequential
// streams keep every DRAM page open, random 64 B reads do not).
//
//   mode 0  read one random 64 B bucket per thread
//   mode 1  read one random 64 B bucket, then CAS 8 B in it (value unchanged)
//   mode 2  read two random 64 B buckets per thread (dependent: the second address comes from the
//           first bucket's contents), the absent-key lookup pattern
//   mode 3  read one random 32 B sector (half a bucket) per thread
//   mode 4  read two random 64 B buckets per thread, both addresses known up front
//   mode 5  CAS 8 B in a random bucket with no read before it (value unchanged)
//   mode 6  read the random slot's 32 B sector, then CAS 8 B in it (value unchanged)
//   mode 7  read one random 64 B bucket per thread as one request shared by a lane pair (lane l
//           loads half l & 1 of the buckets of lanes 2(l >> 1)... : each thread's bucket is read
//           by two lanes, half each, in one of two load instructions per warp)
//   mode 8  mode 7, then CAS 8 B in the bucket (value unchanged)
#include <cuda_runtime.h>

#include <cstdint>

namespace {

__device__ __forceinline__ uint64_t mix64(uint64_t x) {
    x ^= x >> 33;
    x *= 0xff51afd7ed558ccdull;
    x ^= x >> 33;
    x *= 0xc4ceb9fe1a85ec53ull;
    x ^= x >> 33;
    return x;
}

__device__ __forceinline__ void ld64(const unsigned long long* p, unsigned long long (&v)[8]) {
    asm volatile("ld.global.nc.L1::no_allocate.v4.u64 {%0,%1,%2,%3}, [%4];"
                 : "=l"(v[0]), "=l"(v[1]), "=l"(v[2]), "=l"(v[3]) : "l"(p));
    asm volatile("ld.global.nc.L1::no_allocate.v4.u64 {%0,%1,%2,%3}, [%4];"
                 : "=l"(v[4]), "=l"(v[5]), "=l"(v[6]), "=l"(v[7]) : "l"(p + 4));
}

__device__ __forceinline__ void ld64_relaxed(const unsigned long long* p, unsigned long long (&v)[8]) {
    asm volatile("ld.relaxed.gpu.global.v4.u64 {%0,%1,%2,%3}, [%4];"
                 : "=l"(v[0]), "=l"(v[1]), "=l"(v[2]), "=l"(v[3]) : "l"(p) : "memory");
    asm volatile("ld.relaxed.gpu.global.v4.u64 {%0,%1,%2,%3}, [%4];"
                 : "=l"(v[4]), "=l"(v[5]), "=l"(v[6]), "=l"(v[7]) : "l"(p + 4) : "memory");
}

template <int kMode>
__global__ void __launch_bounds__(256) k_probe(unsigned long long* buf, uint64_t nb, uint64_t n, uint64_t seed,
                                               unsigned long long* sink) {
    const uint64_t i = (uint64_t)blockIdx.x * 256 + threadIdx.x;
    if (i >= n) return;
    const uint64_t b = mix64(i ^ seed) % nb;
    unsigned long long v[8];
    unsigned long long acc;
    if (kMode == 3) {
        asm volatile("ld.global.nc.L1::no_allocate.v4.u64 {%0,%1,%2,%3}, [%4];"
                     : "=l"(v[0]), "=l"(v[1]), "=l"(v[2]), "=l"(v[3])
                     : "l"(buf + b * 8 + (i & 1) * 4));
        acc = v[0] ^ v[1] ^ v[2] ^ v[3];
    } else if (kMode == 4) {
        unsigned long long w[8];
        const uint64_t b2 = mix64(i ^ ~seed) % nb;
        ld64(buf + b * 8, v);
        ld64(buf + b2 * 8, w);
        acc = v[0] ^ v[1] ^ v[2] ^ v[3] ^ v[4] ^ v[5] ^ v[6] ^ v[7] ^ w[0] ^ w[1] ^ w[2] ^ w[3] ^ w[4] ^ w[5] ^ w[6] ^
              w[7];
    } else if (kMode == 5) {
        const int j = (int)(i & 7);
        const unsigned long long g = (unsigned long long)(i * 0x9e3779b97f4a7c15ull);
        acc = atomicCAS(buf + b * 8 + j, g, g);
    } else if (kMode == 6) {
        const int j = (int)(i & 7);
        asm volatile("ld.relaxed.gpu.global.v4.u64 {%0,%1,%2,%3}, [%4];"
                     : "=l"(v[0]), "=l"(v[1]), "=l"(v[2]), "=l"(v[3])
                     : "l"(buf + b * 8 + (j & 4))
                     : "memory");
        unsigned long long cur = v[0];
#pragma unroll
        for (int q = 1; q < 4; ++q)
            if (q == (j & 3)) cur = v[q];
        acc = atomicCAS(buf + b * 8 + j, cur, cur);
    } else if (kMode == 1) {
        ld64_relaxed(buf + b * 8, v);
        const int j = (int)(i & 7);
        unsigned long long cur = v[0];
#pragma unroll
        for (int q = 1; q < 8; ++q)
            if (q == j) cur = v[q];
        acc = atomicCAS(buf + b * 8 + j, cur, cur);
    } else {
        ld64(buf + b * 8, v);
        acc = v[0] ^ v[1] ^ v[2] ^ v[3] ^ v[4] ^ v[5] ^ v[6] ^ v[7];
        if (kMode == 2) {
            const uint64_t b2 = mix64(acc ^ i) % nb;
            ld64(buf + b2 * 8, v);
            acc ^= v[0] ^ v[1] ^ v[2] ^ v[3] ^ v[4] ^ v[5] ^ v[6] ^ v[7];
        }
    }
    if (acc == 0x9e3779b97f4a7c15ull) *sink = acc;  // keeps the loads live; practically never taken
}

// Modes 7 and 8: in round r lane l reads half (l & 1) of the bucket of lane 16r + (l >> 1), so one
// warp instruction covers 16 buckets with one two-sector request each.  n must be a multiple of
// 256 (every lane of every warp takes part in the shuffles).
template <int kMode>
__global__ void __launch_bounds__(256) k_probe_pair(unsigned long long* buf, uint64_t nb, uint64_t seed,
                                                    unsigned long long* sink) {
    const uint64_t i = (uint64_t)blockIdx.x * 256 + threadIdx.x;
    const unsigned lane = threadIdx.x & 31;
    const uint64_t b = mix64(i ^ seed) % nb;
    unsigned long long acc = 0, mine = 0;
#pragma unroll
    for (int r = 0; r < 2; ++r) {
        const uint64_t bb = __shfl_sync(0xffffffffu, b, 16 * r + (int)(lane >> 1));
        unsigned long long v[4];
        asm volatile("ld.relaxed.gpu.global.v4.u64 {%0,%1,%2,%3}, [%4];"
                     : "=l"(v[0]), "=l"(v[1]), "=l"(v[2]), "=l"(v[3])
                     : "l"(buf + bb * 8 + (lane & 1) * 4)
                     : "memory");
        unsigned long long x = v[0] ^ v[1] ^ v[2] ^ v[3];
        x ^= __shfl_xor_sync(0xffffffffu, x, 1);
        const unsigned long long got = __shfl_sync(0xffffffffu, x, (int)((2 * lane) & 31u));
        if ((int)(lane >> 4) == r) mine = got;
    }
    acc = mine;
    if (kMode == 8) {
        const int j = (int)(i & 7);
        acc ^= atomicCAS(buf + b * 8 + j, 0ull, 0ull);  // the insert's claim of a free slot
    }
    if (acc == 0x9e3779b97f4a7c15ull) *sink = acc;  // keeps the loads live; practically never taken
}

}  // namespace

extern "C" {

// buf: device buffer of nb 64-byte buckets; n: buckets read (threads).  Returns a cudaError_t.
__attribute__((visibility("default"))) int hive_probe_random_buckets(void* buf, uint64_t nb, uint64_t n, int mode,
                                                                      uint64_t seed, void* sink, void* stream) {
    if (!buf || !nb || !sink || mode < 0 || mode > 8) return (int)cudaErrorInvalidValue;
    if (mode >= 7 && n % 256) return (int)cudaErrorInvalidValue;
    if (!n) return 0;
    const unsigned grid = (unsigned)((n + 255) / 256);
    cudaStream_t s = (cudaStream_t)stream;
    auto* p = (unsigned long long*)buf;
    auto* k = (unsigned long long*)sink;
    if (mode == 0) k_probe<0><<<grid, 256, 0, s>>>(p, nb, n, seed, k);
    else if (mode == 1) k_probe<1><<<grid, 256, 0, s>>>(p, nb, n, seed, k);
    else if (mode == 2) k_probe<2><<<grid, 256, 0, s>>>(p, nb, n, seed, k);
    else if (mode == 3) k_probe<3><<<grid, 256, 0, s>>>(p, nb, n, seed, k);
    else if (mode == 4) k_probe<4><<<grid, 256, 0, s>>>(p, nb, n, seed, k);
    else if (mode == 5) k_probe<5><<<grid, 256, 0, s>>>(p, nb, n, seed, k);
    else if (mode == 6) k_probe<6><<<grid, 256, 0, s>>>(p, nb, n, seed, k);
    else if (mode == 7) k_probe_pair<7><<<grid, 256, 0, s>>>(p, nb, seed, k);
    else k_probe_pair<8><<<grid, 256, 0, s>>>(p, nb, seed, k);
    return (int)cudaGetLastError();
}

}  // extern "C"
