// Minimal stand-in for cuda-utils' cudaExtIntrinsics.cuh (written for this project): byte
// increments and decrements in a 4-byte aligned, padded byte array (the reference's vote
// counters). Test infrastructure only.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
namespace cudapp {
__device__ __forceinline__ void atomicIncOne(uint8_t* p) {
    const uintptr_t a = reinterpret_cast<uintptr_t>(p);
    atomicAdd(reinterpret_cast<unsigned int*>(a & ~uintptr_t(3)), 1u << (8u * unsigned(a & 3u)));
}
__device__ __forceinline__ void atomicDecOne(uint8_t* p) {
    const uintptr_t a = reinterpret_cast<uintptr_t>(p);
    atomicSub(reinterpret_cast<unsigned int*>(a & ~uintptr_t(3)), 1u << (8u * unsigned(a & 3u)));
}
}  // namespace cudapp
