// hive_shard.cu -- the exchange kernels of the hash-partitioned table (include/hive_shard.h).
//
// A batch submitted on one rank is split by owner rank (owner = (fmix32(key ^ 0x9E3779B9) * N) >>
// 32, a mixer independent of the table's bucket hashes) before one all-to-all exchange:
//   hive_shard_count    per block of 4096 ops, how many go to each rank;
//   hive_shard_scatter  with the exclusive prefix of those counts (rank-major), every op's key,
//                       value and type written at its place in destination order, and that place
//                       recorded per op;
//   hive_shard_gather   after the results come back in destination order, each op's status and
//                       value read from its recorded place, so they return in submission order.
// Ops inside one (block, rank) cell keep no particular order: ops of one batch are unordered, as
// in the reference's kernels.  The reference is single-GPU and has no counterpart.
#include <cuda_runtime.h>

#include <cstdint>

#include "hive_shard.h"

namespace {

constexpr int kBlock = 256;
constexpr int kPerThread = HIVE_SHARD_TILE / kBlock;

__device__ __forceinline__ uint32_t owner(uint32_t k, uint32_t world) {
    uint32_t h = k ^ 0x9E3779B9u;
    h ^= h >> 16;
    h *= 0x85ebca6bu;
    h ^= h >> 13;
    h *= 0xc2b2ae35u;
    h ^= h >> 16;
    return (uint32_t)(((uint64_t)h * world) >> 32);
}

__global__ void __launch_bounds__(kBlock) k_shard_count(const uint32_t* __restrict__ keys, uint64_t n, uint32_t world,
                                                        uint32_t* __restrict__ counts) {
    __shared__ uint32_t hist[HIVE_SHARD_MAX_RANKS];
    for (uint32_t r = threadIdx.x; r < world; r += kBlock) hist[r] = 0;
    __syncthreads();
    const uint64_t base = (uint64_t)blockIdx.x * HIVE_SHARD_TILE;
#pragma unroll
    for (int q = 0; q < kPerThread; ++q) {
        const uint64_t i = base + (uint64_t)q * kBlock + threadIdx.x;
        if (i < n) atomicAdd(&hist[owner(__ldg(keys + i), world)], 1u);
    }
    __syncthreads();
    // rank-major: counts[r * nblocks + block]
    for (uint32_t r = threadIdx.x; r < world; r += kBlock) counts[(uint64_t)r * gridDim.x + blockIdx.x] = hist[r];
}

__global__ void __launch_bounds__(kBlock) k_shard_scatter(const uint32_t* __restrict__ keys,
                                                          const uint32_t* __restrict__ vals,
                                                          const uint8_t* __restrict__ types, uint64_t n,
                                                          uint32_t world, const uint64_t* __restrict__ starts,
                                                          uint32_t* __restrict__ out_keys,
                                                          uint32_t* __restrict__ out_vals,
                                                          uint8_t* __restrict__ out_types,
                                                          uint64_t* __restrict__ pos) {
    __shared__ uint32_t cur[HIVE_SHARD_MAX_RANKS];
    for (uint32_t r = threadIdx.x; r < world; r += kBlock) cur[r] = 0;
    __syncthreads();
    const uint64_t base = (uint64_t)blockIdx.x * HIVE_SHARD_TILE;
#pragma unroll
    for (int q = 0; q < kPerThread; ++q) {
        const uint64_t i = base + (uint64_t)q * kBlock + threadIdx.x;
        if (i >= n) continue;
        const uint32_t k = __ldg(keys + i);
        const uint32_t r = owner(k, world);
        const uint64_t p = starts[(uint64_t)r * gridDim.x + blockIdx.x] + atomicAdd(&cur[r], 1u);
        out_keys[p] = k;
        if (vals) out_vals[p] = __ldg(vals + i);
        if (types) out_types[p] = __ldg(types + i);
        pos[i] = p;
    }
}

__global__ void __launch_bounds__(kBlock) k_shard_gather(const uint64_t* __restrict__ pos, uint64_t n,
                                                         const uint8_t* __restrict__ src_status,
                                                         const uint32_t* __restrict__ src_vals,
                                                         uint8_t* __restrict__ status, uint32_t* __restrict__ vals) {
    const uint64_t i = (uint64_t)blockIdx.x * kBlock + threadIdx.x;
    if (i >= n) return;
    const uint64_t p = __ldcs(pos + i);
    if (status) __stcs(status + i, src_status[p]);
    if (vals) __stcs(vals + i, src_vals[p]);
}

inline int launched() { return cudaGetLastError() == cudaSuccess ? 0 : 1; }

}  // namespace

extern "C" {

uint64_t hive_shard_blocks(uint64_t n) { return (n + HIVE_SHARD_TILE - 1) / HIVE_SHARD_TILE; }

int hive_shard_count(const uint32_t* keys, uint64_t n, uint32_t world, uint32_t* counts, void* stream) {
    if (!keys || !counts || world == 0 || world > HIVE_SHARD_MAX_RANKS) return 1;
    if (n == 0) return 0;
    const uint64_t nb = hive_shard_blocks(n);
    if (nb > 0x7FFFFFFFull) return 1;
    k_shard_count<<<(unsigned)nb, kBlock, 0, (cudaStream_t)stream>>>(keys, n, world, counts);
    return launched();
}

int hive_shard_scatter(const uint32_t* keys, const uint32_t* vals, const uint8_t* types, uint64_t n, uint32_t world,
                       const uint64_t* starts, uint32_t* out_keys, uint32_t* out_vals, uint8_t* out_types,
                       uint64_t* pos, void* stream) {
    if (!keys || !starts || !out_keys || !pos || world == 0 || world > HIVE_SHARD_MAX_RANKS) return 1;
    if ((vals && !out_vals) || (types && !out_types)) return 1;
    if (n == 0) return 0;
    const uint64_t nb = hive_shard_blocks(n);
    if (nb > 0x7FFFFFFFull) return 1;
    k_shard_scatter<<<(unsigned)nb, kBlock, 0, (cudaStream_t)stream>>>(keys, vals, types, n, world, starts, out_keys,
                                                                         out_vals, out_types, pos);
    return launched();
}

int hive_shard_gather(const uint64_t* pos, uint64_t n, const uint8_t* src_status, const uint32_t* src_vals,
                      uint8_t* status, uint32_t* vals, void* stream) {
    if (!pos || (status && !src_status) || (vals && !src_vals)) return 1;
    if (n == 0) return 0;
    k_shard_gather<<<(unsigned)((n + kBlock - 1) / kBlock), kBlock, 0, (cudaStream_t)stream>>>(pos, n, src_status,
                                                                                            src_vals, status, vals);
    return launched();
}

}  // extern "C"
