// Order-sensitive 64-bit digests of device arrays, for checking that a result
// computed inside a busy server equals the same request run alone without
// copying the arrays back: digest = sum over i of mix(seed, i, a[i]) (mod 2^64),
// a sum of per-element hashes, so the reduction order does not matter.
#include <cuda_runtime.h>

#include <algorithm>

#include "ol_common.cuh"
#include "ol_kernels.h"

namespace ol {

__device__ __forceinline__ unsigned long long mix64(unsigned long long x) {
    // splitmix64 finaliser (Steele, Lea, Flood 2014)
    x ^= x >> 30;
    x *= 0xBF58476D1CE4E5B9ull;
    x ^= x >> 27;
    x *= 0x94D049BB133111EBull;
    x ^= x >> 31;
    return x;
}

template <class T>
__global__ void digest_kernel(const T *__restrict__ a, uint64_t n, uint32_t seed, unsigned long long *out) {
    unsigned long long acc = 0;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        acc += mix64(((unsigned long long)seed << 56) ^ (i << 24) ^ (unsigned long long)a[i] * 0x9E3779B97F4A7C15ull);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xFFFFFFFFu, acc, o);
    if ((threadIdx.x & 31) == 0 && acc) atomicAdd(out, acc);
}

cudaError_t launch_digest_u32(const uint32_t *a, uint64_t n, uint32_t seed, unsigned long long *out, cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    const uint32_t blocks = (uint32_t)std::min<uint64_t>((n + 255) / 256, 1024);
    digest_kernel<uint32_t><<<blocks, 256, 0, st>>>(a, n, seed, out); OL_LAUNCHED();
    return cudaGetLastError();
}

cudaError_t launch_digest_u8(const uint8_t *a, uint64_t n, uint32_t seed, unsigned long long *out, cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    const uint32_t blocks = (uint32_t)std::min<uint64_t>((n + 255) / 256, 1024);
    digest_kernel<uint8_t><<<blocks, 256, 0, st>>>(a, n, seed, out); OL_LAUNCHED();
    return cudaGetLastError();
}

}  // namespace ol
