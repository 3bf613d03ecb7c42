// Minimal stand-in for cuda-utils' cuda_hint.cuh (written for this project).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

__device__ __forceinline__ uint32_t lane_id() {
    uint32_t l;
    asm("mov.u32 %0, %%laneid;" : "=r"(l));
    return l;
}
template <typename... Ts>
__host__ __device__ __forceinline__ void unused(const Ts&...) {}
__device__ __forceinline__ void prefetchL1(const void* p) {
    asm volatile("prefetch.global.L1 [%0];" ::"l"(p));
}
