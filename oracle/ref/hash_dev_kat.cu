// hash_dev_kat.cu -- TEST INFRASTRUCTURE (oracle pin, GPU).  Evaluates the reference's own
// device hash policies (include/HashPolicies.cuh over include/hash.hpp, compiled from the
// reference tree by oracle/build.py for sm_100a) for a key array, so tests can check the
// oracle's restatement -- including hash2's inline-PTX steps -- against the reference itself.
#include <cstdint>
#include <cuda_runtime.h>
#include "HashPolicies.cuh"

template <typename Policy>
__global__ void ref_buckets_kernel(const uint32_t* keys, size_t n, uint32_t nb, uint32_t* b0, uint32_t* b1) {
    size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    b0[i] = Policy::get_bucket(0, keys[i], nb);
    b1[i] = Policy::get_bucket(1, keys[i], nb);
}

// policy 0 = Default2HashPolicy, 1 = MurmurCityHashPolicy.  Host arrays in and out.
// Returns 0 on success, else the cudaError_t.
extern "C" int ref_dev_buckets(int policy, const uint32_t* h_keys, size_t n, uint32_t nb, uint32_t* h_b0,
                               uint32_t* h_b1) {
    uint32_t *d_k = nullptr, *d_0 = nullptr, *d_1 = nullptr;
    cudaError_t e = cudaMalloc(&d_k, n * 4 * 3 + 16);
    if (e != cudaSuccess) return (int)e;
    d_0 = d_k + n;
    d_1 = d_0 + n;
    e = cudaMemcpy(d_k, h_keys, n * 4, cudaMemcpyHostToDevice);
    if (e == cudaSuccess && n) {
        unsigned grid = (unsigned)((n + 255) / 256);
        if (policy == 1) ref_buckets_kernel<MurmurCityHashPolicy><<<grid, 256>>>(d_k, n, nb, d_0, d_1);
        else ref_buckets_kernel<Default2HashPolicy><<<grid, 256>>>(d_k, n, nb, d_0, d_1);
        e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaDeviceSynchronize();
    }
    if (e == cudaSuccess) e = cudaMemcpy(h_b0, d_0, n * 4, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(h_b1, d_1, n * 4, cudaMemcpyDeviceToHost);
    cudaFree(d_k);
    return (int)e;
}
