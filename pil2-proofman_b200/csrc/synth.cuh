// Seeded synthetic Goldilocks data, identical on host and device.
// Element i of stream `seed` is the first output below p of splitmix64 keyed by (seed, i, j),
// j = 0, 1, ... (a rejection happens with probability ~2^-32, so j is almost always 0).
#pragma once
#include <stdint.h>

namespace synth {

__host__ __device__ __forceinline__ uint64_t mix64(uint64_t z)
{
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}

__host__ __device__ __forceinline__ uint64_t value(uint64_t seed, uint64_t i)
{
    uint64_t key = mix64(seed * 0x9e3779b97f4a7c15ULL + 0x632be59bd9b4e019ULL) ^ (i * 0x9e3779b97f4a7c15ULL);
    for (uint64_t j = 0;; j++) {
        uint64_t v = mix64(key + j * 0xd1b54a32d192ed03ULL);
        if (v < 0xFFFFFFFF00000001ULL) return v;
    }
}

__global__ void fill_kernel(uint64_t *__restrict__ out, uint64_t n, uint64_t seed)
{
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = value(seed, i);
}

}  // namespace synth
